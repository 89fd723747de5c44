"""HEALPix RING geometry and the on-grid transforms S and S^T on the B200.

Drop-in for jht's ``healpix`` module (src/jht/healpix.py): same names, argument
meaning, shapes, conventions (healpy m-major a_lm packing, orthonormal
Condon-Shortley Y_lm, COSMO Q/U, RING order) and error behaviour (ValueError on a
wrong alm/map shape, NotImplementedError for spin not in {0, 2}, one UserWarning
per geometry above the lmax <= 1.5 nside ceiling).  Inputs may be NumPy arrays or
torch tensors; results are torch tensors on the current CUDA device (complex128
alm, float64 maps).  Both transforms are differentiable (torch.autograd): the
gradient of S is built from S^T and vice versa.
"""

from __future__ import annotations

import threading
import warnings
from functools import lru_cache

import numpy as np
import torch

from . import _lib

__all__ = [
    "alm_size",
    "alm_column_base",
    "alm_metric_weight",
    "RingInfo",
    "synthesis",
    "adjoint_synthesis",
    "synthesis_batch",
    "adjoint_synthesis_batch",
]


def alm_size(lmax: int) -> int:
    """Number of packed coefficients, ``(lmax+1)(lmax+2)/2`` (healpix.py:49-50)."""
    return (lmax + 1) * (lmax + 2) // 2


def alm_column_base(m: int, lmax: int) -> int:
    """Index of a_{m,m}, the start of the contiguous column l = m..lmax (healpix.py:53-55)."""
    return m * (2 * lmax + 1 - m) // 2 + m


@lru_cache(maxsize=None)
def alm_metric_weight(lmax: int) -> np.ndarray:
    """``2 - delta_{m0}`` per packed coefficient: the metric in which S^T is the transpose of S.

    ``<S a, v>_map == sum G Re(conj(a) S^T v)`` (healpix.py:58-74).
    """
    ms = np.concatenate([np.full(lmax + 1 - m, m) for m in range(lmax + 1)])
    w = np.where(ms == 0, 1.0, 2.0)
    w.setflags(write=False)
    return w


class RingInfo:
    """Per-ring z = cos(theta), pixel count, first-pixel azimuth and start pixel (healpix.py:107-140)."""

    def __init__(self, nside: int):
        i = np.arange(1, 4 * nside, dtype=np.int64)
        npr = np.empty(i.shape, dtype=np.int64)
        z = np.empty(i.shape)
        phi0 = np.empty(i.shape)
        north, south = i < nside, i > 3 * nside
        belt = ~north & ~south
        npr[north] = 4 * i[north]
        z[north] = 1.0 - i[north] ** 2 / (3.0 * nside**2)
        phi0[north] = np.pi / (4.0 * i[north])
        ii = 4 * nside - i[south]
        npr[south] = 4 * ii
        z[south] = -(1.0 - ii**2 / (3.0 * nside**2))
        phi0[south] = np.pi / (4.0 * ii)
        ib = i[belt]
        npr[belt] = 4 * nside
        z[belt] = 4.0 / 3.0 - 2.0 * ib / (3.0 * nside)
        phi0[belt] = np.where((ib - nside) % 2 == 0, np.pi / (4.0 * nside), 0.0)
        self.nside = nside
        self.npix = 12 * nside**2
        self.z = z
        self.npix_ring = npr
        self.phi0 = phi0
        self.startpix = np.concatenate([[0], np.cumsum(npr)[:-1]])
        self.nrings = int(i.size)


# ---------------------------------------------------------------------------------------
# validation and warnings (healpix.py:191-207, :380-386, :404-411)
# ---------------------------------------------------------------------------------------
_warned: set[tuple[int, int, int]] = set()
_warn_lock = threading.Lock()


def _check_spin(spin: int) -> None:
    if spin not in (0, 2):
        raise NotImplementedError(f"spin={spin} unsupported (only 0 and 2)")


def _ceiling_warning(nside: int, lmax: int, spin: int) -> None:
    if 2 * lmax > 3 * nside:
        key = (nside, lmax, spin)
        with _warn_lock:
            if key in _warned:
                return
            _warned.add(key)
        warnings.warn(
            f"jht_b200: lmax={lmax} exceeds the HEALPix band-limit ceiling 1.5*nside "
            f"(= {1.5 * nside:g} for nside={nside}); the transform is exact as a linear operator but "
            "the quadrature (analysis) is unvalidated above the ceiling.",
            stacklevel=3,
        )


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("jht_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def _host_tensor(x) -> torch.Tensor:
    """``x`` as a tensor where it lies (array-likes wrap host memory without a copy), so
    shapes are checked before any device transfer."""
    return x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x))


def _as_alm(alm) -> torch.Tensor:
    t = _host_tensor(alm)
    if not t.is_complex():
        t = t.to(torch.float64)
    return t.to(device=_device(), dtype=torch.complex128)


def _as_map(m) -> torch.Tensor:
    t = _host_tensor(m)
    if t.is_complex():
        raise TypeError("maps must be real")
    return t.to(device=_device(), dtype=torch.float64)


# ---------------------------------------------------------------------------------------
# raw (non-autograd) calls into the C ABI; batch axis leading
# ---------------------------------------------------------------------------------------
def _synth_raw(alm: torch.Tensor, nside: int, lmax: int, spin: int, precision: str) -> torch.Tensor:
    """alm (B, ncomp, K) complex128 contiguous -> maps (B, ncomp, npix) float64."""
    B = alm.shape[0]
    plan = _lib.get_plan(nside, lmax, spin, precision, B)
    alm = alm.contiguous()
    out = torch.empty((B, plan.ncomp, plan.npix), dtype=torch.float64, device=alm.device)
    if B:
        st = plan.lib.jhtb_synthesis(plan.handle, alm.data_ptr(), out.data_ptr(), B, _lib.stream_ptr())
        _lib.check(st, "jhtb_synthesis")
    return out


def _adjoint_raw(maps: torch.Tensor, nside: int, lmax: int, spin: int, precision: str) -> torch.Tensor:
    """maps (B, ncomp, npix) float64 contiguous -> alm (B, ncomp, K) complex128."""
    B = maps.shape[0]
    plan = _lib.get_plan(nside, lmax, spin, precision, B)
    maps = maps.contiguous()
    out = torch.empty((B, plan.ncomp, plan.K), dtype=torch.complex128, device=maps.device)
    if B:
        st = plan.lib.jhtb_adjoint_synthesis(plan.handle, maps.data_ptr(), out.data_ptr(), B, _lib.stream_ptr())
        _lib.check(st, "jhtb_adjoint_synthesis")
    return out


@lru_cache(maxsize=None)
def _m0_mask(lmax: int, device_index: int) -> torch.Tensor:
    return torch.zeros(alm_size(lmax), dtype=torch.bool, device=torch.device("cuda", device_index)).index_fill_(
        0, torch.arange(lmax + 1, device=torch.device("cuda", device_index)), True
    )


@lru_cache(maxsize=None)
def _metric(lmax: int, device_index: int) -> torch.Tensor:
    return torch.as_tensor(np.array(alm_metric_weight(lmax)), device=torch.device("cuda", device_index))


def _synthesis_cotangent(b: torch.Tensor, lmax: int, spin: int) -> torch.Tensor:
    """torch gradient w.r.t. complex alm of <g, S a>, given b = S^T g  (B, ncomp, K).

    torch's complex gradient is dL/dRe + i dL/dIm.  For m > 0 it is G b; at m = 0
    spin 0 depends only on Re a (b real there), while spin 2 mixes the imaginary
    part of E with B and vice versa through -(E +- iB):
    grad E_l0 = Re bE + i Re bB, grad B_l0 = Re bB - i Re bE.
    (The complex conjugate of jht's JAX cotangent, test_grad.py:134-147.)
    """
    dev = b.device.index
    g = b * _metric(lmax, dev)
    if spin == 2:
        m0 = _m0_mask(lmax, dev)
        bE, bB = b[:, 0].real, b[:, 1].real
        gE = torch.where(m0, torch.complex(bE, bB), g[:, 0])
        gB = torch.where(m0, torch.complex(bB, -bE), g[:, 1])
        g = torch.stack([gE, gB], dim=1)
    return g


def _adjoint_cotangent_input(ga: torch.Tensor, lmax: int, spin: int) -> torch.Tensor:
    """alm to synthesise for the gradient of <ga, S^T v> w.r.t. the real map v.

    dL/dv = S(ga / G) with the m = 0 imaginary parts dropped (S^T v is real at m = 0).
    """
    dev = ga.device.index
    a = ga / _metric(lmax, dev)
    m0 = _m0_mask(lmax, dev)
    return torch.where(m0, torch.complex(a.real, torch.zeros_like(a.real)), a)


class _Synthesis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alm, nside, lmax, spin, precision):
        ctx.geom = (nside, lmax, spin, precision)
        return _synth_raw(alm, nside, lmax, spin, precision)

    @staticmethod
    def backward(ctx, g):
        nside, lmax, spin, precision = ctx.geom
        b = _Adjoint.apply(g.contiguous(), nside, lmax, spin, precision)
        return _synthesis_cotangent(b, lmax, spin), None, None, None, None


class _Adjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, maps, nside, lmax, spin, precision):
        ctx.geom = (nside, lmax, spin, precision)
        return _adjoint_raw(maps, nside, lmax, spin, precision)

    @staticmethod
    def backward(ctx, ga):
        nside, lmax, spin, precision = ctx.geom
        a = _adjoint_cotangent_input(ga.contiguous(), lmax, spin)
        return _Synthesis.apply(a, nside, lmax, spin, precision), None, None, None, None


# ---------------------------------------------------------------------------------------
# public transforms
# ---------------------------------------------------------------------------------------
def synthesis(alm, nside: int, lmax: int, spin: int = 0, *, precision: str = "fp64") -> torch.Tensor:
    """``S: a_lm -> map`` on the HEALPix RING grid (healpix.py:363-387).

    alm: packed complex, ``(alm_size(lmax),)`` for spin 0 or ``(2, alm_size(lmax))``
    (E, B) for spin 2.  Returns ``(12 nside^2,)`` or ``(2, 12 nside^2)`` (Q, U).
    ``precision`` selects the contraction arithmetic ("fp64" plain or "fp32").
    """
    a = _host_tensor(alm)
    expect = (alm_size(lmax),) if spin == 0 else (2, alm_size(lmax))
    if tuple(a.shape) != expect:
        raise ValueError(
            f"alm shape {tuple(a.shape)} != expected {expect} for lmax={lmax}, spin={spin} "
            "(a wrong-size alm would otherwise be silently misread)"
        )
    _check_spin(spin)
    _ceiling_warning(nside, lmax, spin)
    a = _as_alm(a)
    out = _Synthesis.apply(a.reshape(1, -1, alm_size(lmax)), nside, lmax, spin, precision)
    return out.reshape((12 * nside * nside,) if spin == 0 else (2, 12 * nside * nside))


def adjoint_synthesis(m, nside: int, lmax: int, spin: int = 0, *, precision: str = "fp64") -> torch.Tensor:
    """``S^T``: the exact transpose of :func:`synthesis` (healpix.py:390-412).

    ``<S a, v>_map == sum (2 - delta_m0) Re(conj(a) S^T v)``; equals
    ``(Npix / 4 pi) healpy.map2alm(v, iter=0)``.  Input ``(Npix,)`` or ``(2, Npix)``.
    """
    m = _host_tensor(m)
    npix = 12 * nside * nside
    expect = (npix,) if spin == 0 else (2, npix)
    if tuple(m.shape) != expect:
        raise ValueError(
            f"map shape {tuple(m.shape)} != expected {expect} for nside={nside}, spin={spin} "
            "(a wrong-size map would otherwise be silently misread)"
        )
    _check_spin(spin)
    _ceiling_warning(nside, lmax, spin)
    m = _as_map(m)
    out = _Adjoint.apply(m.reshape(1, -1, npix), nside, lmax, spin, precision)
    return out.reshape((alm_size(lmax),) if spin == 0 else (2, alm_size(lmax)))


def synthesis_batch(alm, nside: int, lmax: int, spin: int = 0, *, precision: str = "fp64") -> torch.Tensor:
    """Batched :func:`synthesis`: alm ``(B, K)`` or ``(B, 2, K)`` -> ``(B, Npix)`` / ``(B, 2, Npix)``.

    One launch for the whole batch (jht reaches the same result with ``jax.vmap``).
    """
    a = _as_alm(alm)
    K = alm_size(lmax)
    if (spin == 0 and (a.dim() != 2 or a.shape[1] != K)) or (spin == 2 and (a.dim() != 3 or tuple(a.shape[1:]) != (2, K))):
        raise ValueError(f"batched alm shape {tuple(a.shape)} invalid for lmax={lmax}, spin={spin}")
    _check_spin(spin)
    _ceiling_warning(nside, lmax, spin)
    B = a.shape[0]
    out = _Synthesis.apply(a.reshape(B, -1, K), nside, lmax, spin, precision)
    return out.reshape((B, 12 * nside * nside) if spin == 0 else (B, 2, 12 * nside * nside))


def adjoint_synthesis_batch(maps, nside: int, lmax: int, spin: int = 0, *, precision: str = "fp64") -> torch.Tensor:
    """Batched :func:`adjoint_synthesis`: ``(B, Npix)`` / ``(B, 2, Npix)`` -> ``(B, K)`` / ``(B, 2, K)``."""
    m = _as_map(maps)
    npix = 12 * nside * nside
    if (spin == 0 and (m.dim() != 2 or m.shape[1] != npix)) or (spin == 2 and (m.dim() != 3 or tuple(m.shape[1:]) != (2, npix))):
        raise ValueError(f"batched map shape {tuple(m.shape)} invalid for nside={nside}, spin={spin}")
    _check_spin(spin)
    _ceiling_warning(nside, lmax, spin)
    B = m.shape[0]
    out = _Adjoint.apply(m.reshape(B, -1, npix), nside, lmax, spin, precision)
    K = alm_size(lmax)
    return out.reshape((B, K) if spin == 0 else (B, 2, K))
