"""Real-DOF isometry and the masked (cut-sky) operators on the B200.

Drop-in for the on-grid part of jht's ``masked`` module (src/jht/masked.py):
``alm_to_real`` / ``real_to_alm`` / ``n_dof`` (:117-175), ``pseudo_alm`` (:99-111),
the CG ``deconvolve`` (:278-314), the Wiener filter ``wiener`` (:320-372) and the
posterior draw ``constrained_realization`` (:375-439).  Extension: :func:`deconvolve_batch` solves
many right-hand sides at once (one batched S / S^T launch per CG iteration), with
FP64 residuals and inner products; ``precision`` selects the operator arithmetic.
"""

from __future__ import annotations

import math
from functools import lru_cache

import numpy as np
import torch

from . import _lib
from ._analysis import _pix_w_device, analysis
from .healpix import _adjoint_raw, _as_map, _check_spin, _synth_raw, alm_size

__all__ = ["alm_to_real", "real_to_alm", "n_dof", "pseudo_alm", "deconvolve", "deconvolve_batch", "wiener",
           "wiener_batch", "constrained_realization"]

_SQRT2 = math.sqrt(2.0)


@lru_cache(maxsize=None)
def _dof_layout(lmax: int, spin: int):
    ms = np.concatenate([np.full(lmax + 1 - m, m) for m in range(lmax + 1)])
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    act = ls >= abs(spin)
    idx = np.arange(alm_size(lmax))
    k_m0 = idx[act & (ms == 0)]
    k_mpos = idx[act & (ms > 0)]
    return k_m0, k_mpos, int(k_m0.size + 2 * k_mpos.size)


@lru_cache(maxsize=None)
def _dof_index(lmax: int, spin: int, device_index: int):
    k0, kp, _ = _dof_layout(lmax, spin)
    dev = torch.device("cuda", device_index) if device_index >= 0 else torch.device("cpu")
    return torch.as_tensor(k0, device=dev), torch.as_tensor(kp, device=dev)


def n_dof(lmax: int, spin: int = 0) -> int:
    """Length of the real DOF vector (both E, B channels for spin 2) (masked.py:140-143)."""
    nx = _dof_layout(lmax, spin)[2]
    return nx if spin == 0 else 2 * nx


def _tensor(a) -> torch.Tensor:
    return a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))


def _dev_index(t: torch.Tensor) -> int:
    return t.device.index if t.is_cuda else -1


def alm_to_real(alm, lmax: int, spin: int = 0) -> torch.Tensor:
    """``T``: a_lm -> x with ``||x||_2 = ||a||_G``: a_l0 -> a_l0, a_lm -> sqrt2 (Re, Im), l >= |spin|."""
    a = _tensor(alm)
    k0, kp = _dof_index(lmax, spin, _dev_index(a))

    def one(v):
        return torch.cat([v[k0].real, _SQRT2 * v[kp].real, _SQRT2 * v[kp].imag])

    return one(a) if spin == 0 else torch.cat([one(a[0]), one(a[1])])


def real_to_alm(x, lmax: int, spin: int = 0) -> torch.Tensor:
    """``T^-1``: x -> packed a_lm (l < |spin| modes zero)."""
    xv = _tensor(x).to(torch.float64)
    k0, kp = _dof_index(lmax, spin, _dev_index(xv))
    n0, npos = k0.numel(), kp.numel()
    K = alm_size(lmax)

    def one(v):
        a = torch.zeros(K, dtype=torch.complex128, device=v.device)
        a = a.index_copy(0, k0, v[:n0].to(torch.complex128))
        return a.index_copy(0, kp, torch.complex(v[n0 : n0 + npos], v[n0 + npos : n0 + 2 * npos]) / _SQRT2)

    if spin == 0:
        return one(xv)
    h = xv.shape[0] // 2
    return torch.stack([one(xv[:h]), one(xv[h:])])


def pseudo_alm(maps, mask, nside: int, lmax: int, spin: int = 0, niter: int = 3, use_weights: bool = True):
    """Masked pseudo-a_lm ``analysis(M * map)`` (masked.py:99-111)."""
    m = _as_map(maps)
    msk = _as_map(mask)
    return analysis((msk if spin == 0 else msk[None, :]) * m, nside, lmax, spin, niter, use_weights)


def _real_batch(a: torch.Tensor, lmax: int, spin: int) -> torch.Tensor:
    """(B, ncomp, K) complex -> (B, n_dof) real."""
    k0, kp = _dof_index(lmax, spin, _dev_index(a))
    parts = []
    for c in range(a.shape[1]):
        v = a[:, c]
        parts += [v[:, k0].real, _SQRT2 * v[:, kp].real, _SQRT2 * v[:, kp].imag]
    return torch.cat(parts, dim=1)


def _alm_batch(x: torch.Tensor, lmax: int, spin: int) -> torch.Tensor:
    """(B, n_dof) real -> (B, ncomp, K) complex."""
    k0, kp = _dof_index(lmax, spin, _dev_index(x))
    n0, npos = k0.numel(), kp.numel()
    ncomp = 1 if spin == 0 else 2
    nx = n0 + 2 * npos
    B = x.shape[0]
    out = torch.zeros((B, ncomp, alm_size(lmax)), dtype=torch.complex128, device=x.device)
    for c in range(ncomp):
        v = x[:, c * nx : (c + 1) * nx]
        out[:, c, k0] = v[:, :n0].to(torch.complex128)
        out[:, c, kp] = torch.complex(v[:, n0 : n0 + npos], v[:, n0 + npos :]) / _SQRT2
    return out


def _cg_batch(op, b: torch.Tensor, x: torch.Tensor, tol: float, max_iter: int, op_true=None,
              replace_every: int = 50):
    """Column-wise CG on (B, n) right-hand sides with JAX's stopping rule |r|^2 <= tol^2 |b|^2.

    Each column runs its own step sizes; converged columns are frozen.  Residual
    updates and inner products are FP64 (jax.scipy.sparse.linalg.cg as used at
    masked.py:313, :371, :438).  With ``op_true`` (the FP64 operator, when ``op`` is a
    mixed-precision one) the recursive residual is replaced by the true residual
    ``b - op_true(x)`` every ``replace_every`` steps and whenever the recursive one meets the
    test, so the stopping rule holds for the FP64 system (CG with residual replacement).
    """
    def true_residual(x):
        return b - op_true(x)

    if op_true is not None:
        r = true_residual(x) if bool(x.any()) else b.clone()
    else:
        r = b - op(x) if bool(x.any()) else b.clone()
    p = r.clone()
    gamma = (r * r).sum(dim=1)
    thresh = tol * tol * (b * b).sum(dim=1)
    active = gamma > thresh
    it, replaced = 0, 0
    while bool(active.any()) and it < max_iter:
        Ap = op(p)
        denom = (p * Ap).sum(dim=1)
        alpha = torch.where(active, gamma / torch.where(active, denom, torch.ones_like(denom)), torch.zeros_like(gamma))
        x = x + alpha[:, None] * p
        r = r - alpha[:, None] * Ap
        it += 1
        g2 = (r * r).sum(dim=1)
        if op_true is not None and (it % replace_every == 0 or not bool((active & (g2 > thresh)).any())):
            r = torch.where(active[:, None], true_residual(x), r)
            g2 = (r * r).sum(dim=1)
            replaced += 1
        beta = torch.where(active, g2 / torch.where(active, gamma, torch.ones_like(gamma)), torch.zeros_like(g2))
        p = torch.where(active[:, None], r + beta[:, None] * p, p)
        gamma = torch.where(active, g2, gamma)
        active = gamma > thresh
    info = {"iterations": it, "rel_residual": torch.sqrt(gamma / (b * b).sum(dim=1))}
    if op_true is not None:
        info["outer"] = replaced
    return x, info


def _weight_pix(nside: int, npix: int, device, inv_noise=None, mask=None, use_weights: bool = True) -> torch.Tensor:
    """Per-pixel CG weight (1, 1, Npix): N^-1 if given, else mask * W (masked.py:77-93)."""
    if inv_noise is not None:
        w = _as_map(inv_noise)
    elif mask is not None:
        w = _as_map(mask) * _pix_w_device(nside, use_weights, device.index)
    else:
        raise ValueError("provide either inv_noise (per-pixel N^-1) or mask")
    return w.reshape(1, 1, npix)


@lru_cache(maxsize=None)
def _prior_ell(lmax: int, spin: int) -> np.ndarray:
    k0, kp, _ = _dof_layout(lmax, spin)
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    return np.concatenate([ls[k0], ls[kp], ls[kp]])


def _prior_sqrt(signal_cl, lmax: int, spin: int, device) -> torch.Tensor:
    """x-space whitening sqrt(Cl) per real DOF, exactly 0 on zero-power multipoles (masked.py:181-227)."""
    ell = torch.as_tensor(_prior_ell(lmax, spin), device=device)

    def one(cl):
        c = _tensor(cl).to(device=device, dtype=torch.float64)
        if tuple(c.shape) != (lmax + 1,):
            raise ValueError(f"signal_cl channel must have shape (lmax+1,) = ({lmax + 1},), got {tuple(c.shape)}")
        c = c[ell]
        return torch.where(c > 0, torch.sqrt(torch.where(c > 0, c, torch.ones_like(c))), torch.zeros_like(c))

    if spin == 0:
        return one(signal_cl)
    c_ee, c_bb = signal_cl
    return torch.cat([one(c_ee), one(c_bb)])


def _normal(x, w, nside, lmax, spin, precision):
    """T S^T (w S T^-1 x) for (B, n_dof) columns."""
    s = _synth_raw(_alm_batch(x, lmax, spin), nside, lmax, spin, precision)
    return _real_batch(_adjoint_raw(w * s, nside, lmax, spin, precision), lmax, spin)


def deconvolve_batch(maps, mask, nside: int, lmax: int, spin: int = 0, *, max_iter: int = 200, tol: float = 1e-8,
                     reg: float = 0.0, use_weights: bool = True, x0=None, precision: str = "fp64",
                     return_info: bool = False):
    """CG on ``(T S^T (M W) S T^-1 + reg) x = T S^T (M W) m`` for B right-hand sides at once.

    ``maps``: ``(B, Npix)`` (spin 0) or ``(B, 2, Npix)``; ``mask``: ``(Npix,)``.  Each
    column runs its own CG (its own step sizes and stopping test, JAX's
    ``|r|^2 <= tol^2 |b|^2``); converged columns are frozen.  Residual updates and
    inner products are FP64.  With ``precision="bf16x3"`` the operator applications
    inside CG run on the tensor cores and the recursive residual is replaced by the true
    FP64 residual every 50 steps and before the stopping test is accepted, so the test
    holds on the FP64 system (CG with residual replacement).
    Returns ``(B, K)`` / ``(B, 2, K)`` a_lm.
    """
    _check_spin(spin)
    m = _as_map(maps)
    npix = 12 * nside * nside
    ncomp = 1 if spin == 0 else 2
    mb = m.reshape(m.shape[0], ncomp, npix)
    B = mb.shape[0]
    w = _weight_pix(nside, npix, mb.device, mask=mask, use_weights=use_weights)
    b = _real_batch(_adjoint_raw(w * mb, nside, lmax, spin, "fp64"), lmax, spin)
    x = torch.zeros_like(b) if x0 is None else _real_batch(torch.as_tensor(x0).reshape(B, ncomp, -1).to(b.device), lmax, spin)
    op64 = lambda v: _normal(v, w, nside, lmax, spin, "fp64") + reg * v  # noqa: E731
    if precision == "fp64":
        x, info = _cg_batch(op64, b, x, tol, max_iter)
    else:
        opmx = lambda v: _normal(v, w, nside, lmax, spin, precision) + reg * v  # noqa: E731
        x, info = _cg_batch(opmx, b, x, tol, max_iter, op_true=op64)
    a = _alm_batch(x, lmax, spin)
    a = a.reshape(B, alm_size(lmax)) if spin == 0 else a
    return (a, info) if return_info else a


def deconvolve(maps, mask, nside: int, lmax: int, spin: int = 0, *, max_iter: int = 200, tol: float = 1e-8,
               reg: float = 0.0, use_weights: bool = True, x0=None, precision: str = "fp64"):
    """Cut-sky CG deconvolution of one map (masked.py:278-314)."""
    m = _as_map(maps)
    out = deconvolve_batch(m[None], mask, nside, lmax, spin, max_iter=max_iter, tol=tol, reg=reg,
                           use_weights=use_weights, x0=None if x0 is None else _tensor(x0)[None], precision=precision)
    return out[0]


def _wiener_solve(mb, signal_cl, nside, lmax, spin, inv_noise, mask, max_iter, tol, use_weights, x0, precision,
                  source=None):
    """Prior-whitened CG (P A_x P + I) y = P b_x (+ source), x = P y, for (B, ncomp, Npix) maps."""
    npix = 12 * nside * nside
    B = mb.shape[0]
    ncomp = mb.shape[1]
    w = _weight_pix(nside, npix, mb.device, inv_noise=inv_noise, mask=mask, use_weights=use_weights)
    pw = _prior_sqrt(signal_cl, lmax, spin, mb.device)[None, :]
    rhs = pw * _real_batch(_adjoint_raw(w * mb, nside, lmax, spin, precision), lmax, spin)
    if source is not None:
        rhs = rhs + source(w, pw)
    if x0 is None:
        y = torch.zeros_like(rhs)
    else:  # warm start y0 = P^+ T(x0), 0 on pinned modes
        xv = _real_batch(_tensor(x0).reshape(B, ncomp, -1).to(mb.device), lmax, spin)
        y = torch.where(pw > 0, xv / torch.where(pw > 0, pw, torch.ones_like(pw)), torch.zeros_like(xv))
    y, info = _cg_batch(lambda v: pw * _normal(pw * v, w, nside, lmax, spin, precision) + v, rhs, y, tol, max_iter)
    a = _alm_batch(pw * y, lmax, spin)
    return (a.reshape(B, alm_size(lmax)) if spin == 0 else a), info


def wiener_batch(maps, signal_cl, nside: int, lmax: int, spin: int = 0, *, inv_noise=None, mask=None,
                 max_iter: int = 200, tol: float = 1e-8, use_weights: bool = True, x0=None, precision: str = "fp64",
                 return_info: bool = False):
    """Wiener-mean a_lm of B maps at once: ``(S^T N^-1 S + C^-1) a = S^T N^-1 m`` per column."""
    _check_spin(spin)
    m = _as_map(maps)
    ncomp = 1 if spin == 0 else 2
    mb = m.reshape(m.shape[0], ncomp, 12 * nside * nside)
    a, info = _wiener_solve(mb, signal_cl, nside, lmax, spin, inv_noise, mask, max_iter, tol, use_weights, x0,
                            precision)
    return (a, info) if return_info else a


def wiener(maps, signal_cl, nside: int, lmax: int, spin: int = 0, *, inv_noise=None, mask=None, max_iter: int = 200,
           tol: float = 1e-8, use_weights: bool = True, x0=None, precision: str = "fp64"):
    """Wiener filter / MAP a_lm (masked.py:320-372).

    Solves ``(S^T N^-1 S + C^-1) a = S^T N^-1 m`` by CG in prior-whitened real-DOF
    coordinates ``x = P y``, ``P = diag(sqrt(Cl))``; zero-power multipoles are pinned
    to 0 exactly.  ``signal_cl``: ``(lmax+1,)`` (spin 0) or ``(C_EE, C_BB)``;
    ``inv_noise`` (per-pixel N^-1, mask folded in) or else ``mask`` (weight M W).
    """
    m = _as_map(maps)
    a = wiener_batch(m[None], signal_cl, nside, lmax, spin, inv_noise=inv_noise, mask=mask, max_iter=max_iter,
                     tol=tol, use_weights=use_weights, x0=None if x0 is None else _tensor(x0)[None], precision=precision)
    return a[0]


def constrained_realization(maps, signal_cl, nside: int, lmax: int, key, spin: int = 0, *, inv_noise=None,
                            mask=None, max_iter: int = 200, tol: float = 1e-8, use_weights: bool = True, x0=None,
                            precision: str = "fp64"):
    """One posterior draw ``a ~ N(a_wiener, (S^T N^-1 S + C^-1)^-1)`` (masked.py:375-439).

    Same whitened system as :func:`wiener` with the source
    ``P T S^T (sqrt(N^-1) omega) + xi`` added to the right-hand side, ``omega ~ N(0, I)``
    per pixel and ``xi ~ N(0, I)`` per real DOF (0 on pinned modes).  ``key`` replaces
    jax's PRNG key: a ``torch.Generator`` on the maps' device, or an int seed; the
    draws are ``torch.randn`` of omega then xi, in that order, from it.
    """
    _check_spin(spin)
    m = _as_map(maps)
    ncomp = 1 if spin == 0 else 2
    npix = 12 * nside * nside
    mb = m.reshape(1, ncomp, npix)
    if isinstance(key, torch.Generator):
        gen = key
    else:
        gen = torch.Generator(device=mb.device)
        gen.manual_seed(int(key))
    omega = torch.randn((1, ncomp, npix), dtype=torch.float64, device=mb.device, generator=gen)
    xi = torch.randn((1, n_dof(lmax, spin)), dtype=torch.float64, device=mb.device, generator=gen)

    def source(w, pw):
        s1 = _real_batch(_adjoint_raw(torch.sqrt(w) * omega, nside, lmax, spin, precision), lmax, spin)
        return pw * s1 + torch.where(pw > 0, xi, torch.zeros_like(xi))

    a, _ = _wiener_solve(mb, signal_cl, nside, lmax, spin, inv_noise, mask, max_iter, tol, use_weights,
                         None if x0 is None else _tensor(x0)[None], precision, source=source)
    return a[0]
