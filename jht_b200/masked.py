"""Real-DOF isometry and the masked (cut-sky) operators on the B200.

Drop-in for the on-grid part of jht's ``masked`` module (src/jht/masked.py):
``alm_to_real`` / ``real_to_alm`` / ``n_dof`` (:117-175), ``pseudo_alm`` (:99-111)
and the CG ``deconvolve`` (:278-314).  Extension: :func:`deconvolve_batch` solves
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

__all__ = ["alm_to_real", "real_to_alm", "n_dof", "pseudo_alm", "deconvolve", "deconvolve_batch"]

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


def deconvolve_batch(maps, mask, nside: int, lmax: int, spin: int = 0, *, max_iter: int = 200, tol: float = 1e-8,
                     reg: float = 0.0, use_weights: bool = True, x0=None, precision: str = "fp64",
                     return_info: bool = False):
    """CG on ``(T S^T (M W) S T^-1 + reg) x = T S^T (M W) m`` for B right-hand sides at once.

    ``maps``: ``(B, Npix)`` (spin 0) or ``(B, 2, Npix)``; ``mask``: ``(Npix,)``.  Each
    column runs its own CG (its own step sizes and stopping test, JAX's
    ``|r|^2 <= tol^2 |b|^2``); converged columns are frozen.  Residual updates and
    inner products are FP64.  Returns ``(B, K)`` / ``(B, 2, K)`` a_lm.
    """
    _check_spin(spin)
    m = _as_map(maps)
    npix = 12 * nside * nside
    ncomp = 1 if spin == 0 else 2
    mb = m.reshape(m.shape[0], ncomp, npix)
    B = mb.shape[0]
    w = _as_map(mask) * _pix_w_device(nside, use_weights, mb.device.index)
    w = w.reshape(1, 1, npix)

    def op(x):
        a = _alm_batch(x, lmax, spin)
        s = _synth_raw(a, nside, lmax, spin, precision)
        return _real_batch(_adjoint_raw(w * s, nside, lmax, spin, precision), lmax, spin) + reg * x

    b = _real_batch(_adjoint_raw(w * mb, nside, lmax, spin, precision), lmax, spin)
    x = torch.zeros_like(b) if x0 is None else _real_batch(torch.as_tensor(x0).reshape(B, ncomp, -1).to(b.device), lmax, spin)
    r = b - op(x)
    p = r.clone()
    gamma = (r * r).sum(dim=1)
    thresh = tol * tol * (b * b).sum(dim=1)
    active = gamma > thresh
    it = 0
    while bool(active.any()) and it < max_iter:
        Ap = op(p)
        denom = (p * Ap).sum(dim=1)
        alpha = torch.where(active, gamma / torch.where(active, denom, torch.ones_like(denom)), torch.zeros_like(gamma))
        x = x + alpha[:, None] * p
        r = r - alpha[:, None] * Ap
        g2 = (r * r).sum(dim=1)
        beta = torch.where(active, g2 / torch.where(active, gamma, torch.ones_like(gamma)), torch.zeros_like(g2))
        p = torch.where(active[:, None], r + beta[:, None] * p, p)
        gamma = torch.where(active, g2, gamma)
        active = gamma > thresh
        it += 1
    a = _alm_batch(x, lmax, spin)
    a = a.reshape(B, alm_size(lmax)) if spin == 0 else a
    if return_info:
        return a, {"iterations": it, "rel_residual": torch.sqrt(gamma / (b * b).sum(dim=1))}
    return a


def deconvolve(maps, mask, nside: int, lmax: int, spin: int = 0, *, max_iter: int = 200, tol: float = 1e-8,
               reg: float = 0.0, use_weights: bool = True, x0=None, precision: str = "fp64"):
    """Cut-sky CG deconvolution of one map (masked.py:278-314)."""
    m = _as_map(maps)
    out = deconvolve_batch(m[None], mask, nside, lmax, spin, max_iter=max_iter, tol=tol, reg=reg,
                           use_weights=use_weights, x0=None if x0 is None else _tensor(x0)[None], precision=precision)
    return out[0]
