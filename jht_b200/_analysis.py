"""Analysis (map -> a_lm, the approximate inverse) on the B200.

Drop-in for jht's ``_analysis`` module (src/jht/_analysis.py:49-67):
``A0 = S^T W`` and ``niter`` Jacobi steps ``a += A0 (m - S a)``.  The weighted
residual ``W (m - S a)`` runs as one FP64 kernel (``jhtb_weighted_residual``).

``precision`` (extension) selects the arithmetic of the A0 applications: with
``"bf16x3"`` they run as the batched tensor-core adjoint (split-BF16 products, FP32
sums folded into FP64), while the residual synthesis ``S a`` and ``W (m - S a)``
stay FP64, so each Jacobi step corrects the previous steps' rounding and the result
approaches the FP64 analysis.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np
import torch

from . import _lib
from .healpix import (
    _adjoint_raw,
    _as_map,
    _check_spin,
    _ceiling_warning,
    _synth_raw,
    adjoint_synthesis,
    alm_size,
    synthesis,
)
from .weights import pixel_weights, ring_weights

__all__ = ["bare_analysis", "analysis", "map2alm"]


@lru_cache(maxsize=None)
def _ring_w_device(nside: int, device_index: int) -> torch.Tensor:
    return torch.as_tensor(np.array(ring_weights(nside)), device=torch.device("cuda", device_index))


@lru_cache(maxsize=None)
def _pix_w_device(nside: int, use_weights: bool, device_index: int) -> torch.Tensor:
    return torch.as_tensor(np.asarray(pixel_weights(nside, use_weights)), device=torch.device("cuda", device_index))


def _weighted(maps: torch.Tensor, synth: torch.Tensor | None, nside: int, lmax: int, spin: int,
              use_weights: bool) -> torch.Tensor:
    """W (maps - synth) through the C ABI (no autograd); shapes (B, ncomp, npix)."""
    plan = _lib.get_plan(nside, lmax, spin, "fp64", maps.shape[0])
    out = torch.empty_like(maps)
    rw = _ring_w_device(nside, maps.device.index).data_ptr() if use_weights else None
    st = plan.lib.jhtb_weighted_residual(
        plan.handle, maps.data_ptr(), synth.data_ptr() if synth is not None else None, rw, out.data_ptr(),
        maps.shape[0], _lib.stream_ptr(),
    )
    _lib.check(st, "jhtb_weighted_residual")
    return out


def _needs_grad(t: torch.Tensor) -> bool:
    return torch.is_grad_enabled() and t.requires_grad


def bare_analysis(maps, nside: int, lmax: int, spin: int = 0, use_weights: bool = True, *,
                  precision: str = "fp64") -> torch.Tensor:
    """``A0 = S^T W`` (_analysis.py:49-52)."""
    m = _as_map(maps)
    if _needs_grad(m):
        w = _pix_w_device(nside, use_weights, m.device.index)
        return adjoint_synthesis(w * m if spin == 0 else w[None, :] * m, nside, lmax, spin, precision=precision)
    _check_spin(spin)
    npix = 12 * nside * nside
    expect = (npix,) if spin == 0 else (2, npix)
    if tuple(m.shape) != expect:
        raise ValueError(f"map shape {tuple(m.shape)} != expected {expect} for nside={nside}, spin={spin}")
    _ceiling_warning(nside, lmax, spin)
    mb = m.reshape(1, -1, npix).contiguous()
    a = _adjoint_raw(_weighted(mb, None, nside, lmax, spin, use_weights), nside, lmax, spin, precision)
    return a.reshape((alm_size(lmax),) if spin == 0 else (2, alm_size(lmax)))


def analysis(maps, nside: int, lmax: int, spin: int = 0, niter: int = 3, use_weights: bool = True, *,
             precision: str = "fp64") -> torch.Tensor:
    """A0 followed by ``niter`` Jacobi refinements (_analysis.py:55-63)."""
    m = _as_map(maps)
    if _needs_grad(m):
        a = bare_analysis(m, nside, lmax, spin, use_weights, precision=precision)
        for _ in range(niter):
            r = m - synthesis(a, nside, lmax, spin)
            a = a + bare_analysis(r, nside, lmax, spin, use_weights, precision=precision)
        return a
    _check_spin(spin)
    npix = 12 * nside * nside
    expect = (npix,) if spin == 0 else (2, npix)
    if tuple(m.shape) != expect:
        raise ValueError(f"map shape {tuple(m.shape)} != expected {expect} for nside={nside}, spin={spin}")
    _ceiling_warning(nside, lmax, spin)
    mb = m.reshape(1, -1, npix).contiguous()
    a = analysis_batch_raw(mb, nside, lmax, spin, niter, use_weights, precision)
    return a.reshape((alm_size(lmax),) if spin == 0 else (2, alm_size(lmax)))


def analysis_batch_raw(mb: torch.Tensor, nside: int, lmax: int, spin: int, niter: int, use_weights: bool,
                       precision: str = "fp64") -> torch.Tensor:
    """Jacobi analysis of a (B, ncomp, npix) batch, no autograd."""
    a = _adjoint_raw(_weighted(mb, None, nside, lmax, spin, use_weights), nside, lmax, spin, precision)
    for _ in range(niter):
        s = _synth_raw(a, nside, lmax, spin, "fp64")
        a += _adjoint_raw(_weighted(mb, s, nside, lmax, spin, use_weights), nside, lmax, spin, precision)
    return a


map2alm = analysis
