"""HEALPix ring quadrature weights (host FP64, computed once per nside).

Drop-in for jht's ``weights`` module (src/jht/weights.py:60-106): jht's own
minimum-norm weights making the m=0 colatitude quadrature exact for even
Legendre polynomials to degree 2*nside.  Solved on the host with LAPACK
(``numpy.linalg.lstsq``); the result is uploaded once and used by the weighted
residual kernel on the GPU.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np
from numpy.polynomial.legendre import legvander

from .healpix import RingInfo

__all__ = ["ring_weights", "pixel_weights"]


@lru_cache(maxsize=None)
def ring_weights(nside: int) -> np.ndarray:
    """Per-ring weight deviations ``w_i`` (length 2*nside, north half + equator).

    The per-pixel weight of ring i is ``(4 pi / Npix)(1 + w_i)``; southern rings use
    their north partner's weight.  ``w`` is the minimum-norm solution of
    ``sum_i c_i n_i (1 + w_i) P_l(z_i) = Npix delta_{l0}`` for even l <= 2*nside,
    with ``c_i = 2`` (N/S pair) or 1 (equator).
    """
    geo = RingInfo(nside)
    T = 2 * nside
    z = geo.z[:T]
    n = geo.npix_ring[:T].astype(np.float64)
    mult = np.full(T, 2.0)
    mult[-1] = 1.0
    P = legvander(z, 2 * nside)[:, ::2]
    A = ((mult * n)[:, None] * P).T
    rhs = -A.sum(axis=1)
    rhs[0] += geo.npix
    w, *_ = np.linalg.lstsq(A, rhs, rcond=None)
    w.setflags(write=False)
    return w


@lru_cache(maxsize=None)
def pixel_weights(nside: int, use_weights: bool = True) -> np.ndarray:
    """Per-pixel quadrature weights in RING order (``4 pi / Npix`` when ``use_weights=False``)."""
    geo = RingInfo(nside)
    base = 4.0 * np.pi / geo.npix
    if not use_weights:
        wv = np.full(geo.npix, base)
    else:
        w = ring_weights(nside)
        r = np.arange(geo.nrings)
        half = np.where(r < 2 * nside, r, 4 * nside - 2 - r)
        wv = base * (1.0 + np.repeat(w[half], geo.npix_ring))
    wv.setflags(write=False)
    return wv
