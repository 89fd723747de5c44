"""Complex FP64 FFTs on the device (jhtb_fft_c2c), for the off-grid transforms.

jht runs the off-grid path's theta FFT and the FFTs of the oversampled torus grid as
``jnp.fft`` inside XLA (_nufft.py:164-191); here they are this library's kernel: batched
transforms of 2,3,5-smooth lengths along either axis of a row-major 2-D array, held in
shared memory up to SM_MAX points and composed from two batched calls (four-step) above.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np
import torch

from . import _lib

SM_MAX = 10240  # longest transform one CTA holds in shared memory (kFftSmMax in fft.cu)


def _smooth(n: int) -> bool:
    for f in (2, 3, 5):
        while n % f == 0:
            n //= f
    return n == 1


def _split(n: int) -> tuple[int, int]:
    """n = n1 * n2 with both factors 2,3,5-smooth and <= SM_MAX, n1 as close to sqrt(n) as possible."""
    best = None
    d = 1
    while d * d <= n:
        if n % d == 0:
            for n1 in (d, n // d):
                n2 = n // n1
                if n1 <= SM_MAX and n2 <= SM_MAX and _smooth(n1) and _smooth(n2):
                    if best is None or abs(n1 - n2) < abs(best[0] - best[1]):
                        best = (n1, n2)
        d += 1
    if best is None:
        raise ValueError(f"FFT length {n} has no factorisation into two smooth lengths <= {SM_MAX}")
    return best


_PI_LD = np.longdouble("3.14159265358979323846264338327950288")


def _roots_host(n: int) -> np.ndarray:
    """e^{-2 pi i k / n} for k < n as complex128.  The angle is folded to the first octant in
    integers: with r = min(k, n - k) it is pi b / (2 n), b = 4 r in [0, 2 n]; b > n reflects
    about pi / 2 (the cosine changes sign), then 2 b > n about pi / 4 (cosine and sine swap).
    The octant's cosine and sine are taken in the host's extended precision (x86: 64-bit
    mantissa) before rounding to FP64, so each entry is within about half an FP64 ulp, and
    the multiples of pi / 2 come out exactly."""
    k = np.arange(n, dtype=np.int64)
    b = 4 * np.minimum(k, n - k)
    flip = b > n
    b = np.where(flip, 2 * n - b, b)
    swap = 2 * b > n
    b = np.where(swap, n - b, b)
    ang = _PI_LD * b.astype(np.longdouble) / (2 * n)
    c, s = np.cos(ang).astype(np.float64), np.sin(ang).astype(np.float64)
    c, s = np.where(swap, s, c), np.where(swap, c, s)
    c = np.where(flip, -c, c)
    s = np.where(k <= n // 2, s, -s)
    return c - 1j * s


@lru_cache(maxsize=None)
def _roots(n: int, device: int) -> torch.Tensor:
    """The table of _roots_host(n) on the device (built once per length and device)."""
    return torch.as_tensor(_roots_host(n), dtype=torch.complex128, device=torch.device("cuda", device))


def _call(x, out, n, howmany, inner, in_stride, in_do, in_di, out_stride, out_do, out_di, sign, scale, tw):
    lib = _lib.load_library()
    roots = _roots(n, x.device.index)
    _lib.check(lib.jhtb_fft_c2c(x.data_ptr(), out.data_ptr(), n, howmany, inner, in_stride, in_do, in_di, out_stride,
                                out_do, out_di, sign, float(scale), tw, roots.data_ptr(), _lib.stream_ptr()),
               "jhtb_fft_c2c")


def fft(x: torch.Tensor, dim: int, sign: int, scale: float = 1.0) -> torch.Tensor:
    """``scale * sum_i x[.., i, ..] e^{sign 2 pi i i k / n}`` along ``dim`` (0 or 1) of a 2-D
    complex128 CUDA tensor (a new tensor; sign -1 is numpy's fft, +1 its unscaled inverse)."""
    if x.dim() != 2 or x.dtype != torch.complex128 or not x.is_cuda:
        raise ValueError("fft: expects a 2-D complex128 CUDA tensor")
    if dim not in (0, 1) or sign not in (1, -1):
        raise ValueError("fft: dim must be 0 or 1 and sign +1 or -1")
    x = x.contiguous()
    rows, cols = x.shape
    out = torch.empty_like(x)
    n = x.shape[dim]
    if x.numel() == 0:
        return out
    if not _smooth(n):
        raise ValueError(f"fft: length {n} is not 2,3,5-smooth")
    # element i of transform o at o * dist + i * s
    s, howmany, dist = (1, rows, cols) if dim == 1 else (cols, cols, 1)
    if n <= SM_MAX:
        _call(x, out, n, howmany, 1, s, dist, 0, s, dist, 0, sign, scale, 0)
        return out
    # four-step, n = n1 n2, i = n2 i1 + i2, k = k1 + n1 k2: length-n1 transforms over i1 for
    # every i2, times e^{sign 2 pi i i2 k1 / n}; then length-n2 transforms over i2 for every
    # k1, written to k1 + n1 k2
    n1, n2 = _split(n)
    tmp = torch.empty_like(x)
    _call(x, tmp, n1, howmany * n2, n2, n2 * s, dist, s, n2 * s, dist, s, sign, 1.0, n)
    _call(tmp, out, n2, howmany * n1, n1, s, dist, n2 * s, n1 * s, dist, s, sign, scale, 0)
    return out
