"""NumPy stand-in for the slice of the JAX API that jht's on-grid modules touch.

JAX is not installed in this container and there is no network, so jht (which
is pure Python over JAX) cannot be imported as shipped.  Its on-grid code only
uses a small, well-defined part of the JAX surface (``jax.numpy`` array math,
functional ``.at[...].set/.add`` updates, ``jax.lax.scan``, ``jax.jit`` and the
CG solver), all of which have exact NumPy meanings.  Installing this shim makes
``jax`` resolve to NumPy so that the reference's own source executes unchanged
and its outputs can be frozen as golden fixtures (``make_golden.py``).

Test infrastructure only: nothing in the product imports this module.
"""

from __future__ import annotations

import sys
import types

import numpy as np


class _Arr(np.ndarray):
    """ndarray with JAX's functional ``.at[idx].set / .add`` update syntax."""

    @property
    def at(self):
        return _AtIndexer(self)


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtUpdate(self._arr, idx)


class _AtUpdate:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _copy(self):
        return np.array(self._arr, copy=True).view(_Arr)

    def set(self, values, **_kw):
        out = self._copy()
        out[self._idx] = np.asarray(values)
        return out

    def add(self, values, **_kw):
        # JAX scatter-add accumulates repeated indices, i.e. ufunc.at semantics.
        out = self._copy()
        np.add.at(out, self._idx, np.asarray(values))
        return out


def _zeros(shape, dtype=np.float64):
    return np.zeros(shape, dtype=dtype).view(_Arr)


def _zeros_like(a, dtype=None):
    return np.zeros_like(np.asarray(a), dtype=dtype).view(_Arr)


def _tree_index(tree, i):
    if tree is None:
        return None
    if isinstance(tree, (tuple, list)):
        return type(tree)(_tree_index(t, i) for t in tree)
    return np.asarray(tree)[i]


def _tree_len(tree):
    if isinstance(tree, (tuple, list)):
        for t in tree:
            n = _tree_len(t)
            if n is not None:
                return n
        return None
    if tree is None:
        return None
    return np.asarray(tree).shape[0]


def _tree_stack(items):
    first = items[0]
    if first is None:
        return None
    if isinstance(first, (tuple, list)):
        return type(first)(_tree_stack([it[k] for it in items]) for k in range(len(first)))
    return np.stack([np.asarray(it) for it in items])


def _scan(f, init, xs, length=None):
    """Sequential ``lax.scan``: loop over the leading axis of ``xs``."""
    n = _tree_len(xs) if xs is not None else length
    carry = init
    ys = []
    for i in range(n):
        carry, y = f(carry, _tree_index(xs, i))
        ys.append(y)
    return carry, (_tree_stack(ys) if ys else None)


def _vdot_real(a, b):
    return float(np.real(np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())))


def _cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """Conjugate gradient with JAX's stopping rule ``|r|^2 <= max(tol^2 |b|^2, atol^2)``.

    Standard Hestenes-Stiefel CG (unpreconditioned unless ``M`` is given);
    ``maxiter`` defaults to ten times the problem size, as in JAX.
    """
    b = np.asarray(b)
    x = np.zeros_like(b) if x0 is None else np.asarray(x0).copy()
    precond = (lambda v: v) if M is None else M
    if maxiter is None:
        maxiter = 10 * b.size
    thresh = max(tol * tol * _vdot_real(b, b), atol * atol)
    r = b - np.asarray(A(x))
    z = precond(r)
    p = z
    gamma = _vdot_real(r, z)
    k = 0
    while True:
        rs = gamma if M is None else _vdot_real(r, r)
        if not (rs > thresh and k < maxiter):
            break
        Ap = np.asarray(A(p))
        alpha = gamma / _vdot_real(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = precond(r)
        gamma_new = _vdot_real(r, z)
        p = z + (gamma_new / gamma) * p
        gamma = gamma_new
        k += 1
    return x, None


def _segment_sum(data, segment_ids, num_segments):
    data = np.asarray(data)
    out = np.zeros(num_segments, dtype=data.dtype)
    np.add.at(out, np.asarray(segment_ids), data)
    return out


class _Config:
    jax_enable_x64 = True

    def update(self, name, value):
        setattr(self, name, value)


def install() -> None:
    """Register ``jax`` / ``jax.numpy`` / ... in ``sys.modules`` (idempotent)."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "_is_numpy_shim", False):
        return
    jax = types.ModuleType("jax")
    jax._is_numpy_shim = True
    jax.config = _Config()
    jax.Array = np.ndarray
    jax.jit = lambda f=None, **_kw: (f if f is not None else (lambda g: g))

    jnp = types.ModuleType("jax.numpy")
    for name in (
        "abs", "arange", "broadcast_to", "clip", "concatenate", "conj", "exp", "imag",
        "log", "mod", "pad", "real", "sqrt", "stack", "sum", "tensordot", "transpose",
        "where", "float64", "complex128", "int64", "pi", "ceil", "full", "ones",
        "maximum", "minimum", "square", "dot", "vdot", "einsum", "isfinite", "sin", "cos",
    ):
        setattr(jnp, name, getattr(np, name))
    jnp.iscomplexobj = np.iscomplexobj
    jnp.asarray = lambda a, dtype=None: np.asarray(a, dtype=dtype)
    jnp.array = lambda a, dtype=None: np.array(a, dtype=dtype)
    jnp.zeros = _zeros
    jnp.zeros_like = _zeros_like
    jnp.fft = np.fft
    jnp.ndarray = np.ndarray

    lax = types.ModuleType("jax.lax")
    lax.scan = _scan
    lax.stop_gradient = lambda a: a

    ops = types.ModuleType("jax.ops")
    ops.segment_sum = _segment_sum

    scipy = types.ModuleType("jax.scipy")
    sparse = types.ModuleType("jax.scipy.sparse")
    linalg = types.ModuleType("jax.scipy.sparse.linalg")
    linalg.cg = _cg
    sparse.linalg = linalg
    scipy.sparse = sparse

    random = types.ModuleType("jax.random")

    jax.numpy = jnp
    jax.lax = lax
    jax.ops = ops
    jax.scipy = scipy
    jax.random = random
    for mod in (jax, jnp, lax, ops, scipy, sparse, linalg, random):
        sys.modules[mod.__name__] = mod


def import_reference(src_dir: str) -> types.ModuleType:
    """Import the reference ``jht`` package from ``src_dir`` without running its ``__init__``.

    The package ``__init__`` would pull in every module at once; the submodules
    are imported explicitly instead (the off-grid pair ``_nufft`` / ``offgrid`` too).
    """
    import importlib

    install()
    pkg = types.ModuleType("jht")
    pkg.__path__ = [f"{src_dir}/jht"]
    sys.modules["jht"] = pkg
    for sub in ("healpix", "_recursion", "_azimuth", "_analysis", "weights", "masked", "_reference", "_nufft",
                "offgrid"):
        setattr(pkg, sub, importlib.import_module(f"jht.{sub}"))
    return pkg
