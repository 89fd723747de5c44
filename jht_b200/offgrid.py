"""Off-grid synthesis and its exact adjoint on the B200 (jht's offgrid.py / _nufft.py).

``synthesis_general(alm, loc, spin=, lmax=, epsilon=)`` evaluates the band-limited field
at arbitrary points ``loc = [[theta, phi], ...]``; ``adjoint_synthesis_general`` is its
exact transpose in the (2 - delta_m0) alm metric.  The algorithm is jht's (which
matches ducc's ``sphere_interpol``), mapped onto the device:

1. the Legendre stage at ``ns`` Clenshaw-Curtis rings ``theta_j = j pi / (ns - 1)``,
   both poles included (offgrid.py:60-88, :155-160): the library's FP64 recursion
   kernels on a ring-set plan (``jhtb_plan_create_rings`` + ``jhtb_legendre_synthesis``);
2. the double-Fourier-sphere extension to the 2 pi theta period and a theta FFT
   (offgrid.py:113-129), then the deconvolution by the kernel's Fourier transform and an
   inverse 2D FFT onto the oversampled torus grid (_nufft.py:164-174) -- gathers and the
   library's FFT kernel (``jhtb_fft_c2c``, 2,3,5-smooth lengths; the 2-D transform skips
   the grid's all-zero rows);
3. the W x W exponential-of-semicircle window sums at the points
   (``jhtb_nufft_interp``, _nufft.py:150-178).

The adjoint runs the transposes in reverse order (``jhtb_nufft_spread`` with FP64
atomics, forward FFT, transposed extension, ``jhtb_legendre_adjoint``).

Accuracy is set by ``epsilon`` through jht's kernel table (W = 14 at the default 1e-10);
torch autograd gives the alm gradient (the adjoint, jht's VJP convention) and the
pointing gradient d field / d (theta, phi) from the kernel's derivative weights.
Spin 0 and 2 (jht also covers spin 1 and 3: ``NotImplementedError`` here).
"""

from __future__ import annotations

import ctypes
import math
from functools import lru_cache

import numpy as np
import torch

from . import _lib
from . import _fft
from .healpix import (
    _adjoint_cotangent_input,
    _as_alm,
    _device,
    _host_tensor,
    _synthesis_cotangent,
    alm_metric_weight,
    alm_size,
)

__all__ = ["synthesis_general", "adjoint_synthesis_general"]

# achievable accuracy -> (kernel width W, oversampling sigma): jht's table (_nufft.py:33-39)
_KERNELS = {1e-4: (6, 2.0), 1e-6: (8, 2.0), 1e-8: (10, 2.0), 1e-10: (14, 2.0), 1e-12: (16, 2.0)}


def _kernel_for(eps: float) -> tuple[int, float]:
    ok = [e for e in _KERNELS if e <= eps * 1.0000001]
    return _KERNELS[max(ok)] if ok else _KERNELS[min(_KERNELS)]


def _fft_size(n: float) -> int:
    """Smallest even 2,3,5-smooth integer >= n."""
    k = int(math.ceil(n))
    k += k % 2
    while True:
        r = k
        for f in (2, 3, 5):
            while r % f == 0:
                r //= f
        if r == 1:
            return k
        k += 2


def _kernel_ft(N: int, n: int, W: int, beta: float) -> np.ndarray:
    """Fourier transform of the window at the N centered modes of an n-point axis
    (Gauss-Legendre quadrature, 2W + 24 nodes, as _nufft.py:87-94)."""
    k = np.arange(-(N // 2), -(N // 2) + N)
    t, w = np.polynomial.legendre.leggauss(2 * W + 24)
    t, w = t * (W / 2.0), w * (W / 2.0)
    psi = np.exp(beta * (np.sqrt(np.clip(1.0 - (2.0 * t / W) ** 2, 0.0, 1.0)) - 1.0))
    return np.cos(np.outer(k, t) * (2.0 * np.pi / n)) @ (psi * w)


class _Geometry:
    """Per (lmax, spin, epsilon, device): the ring-set plan and the NUFFT tables."""

    def __init__(self, lmax: int, spin: int, eps: float, device: int):
        self.lmax, self.spin, self.ncomp = lmax, spin, 1 if spin == 0 else 2
        self.ns = _fft_size(lmax + 1) + 1
        self.nd = 2 * self.ns - 2
        theta = np.arange(self.ns) * np.pi / (self.ns - 1)
        x = np.cos(theta[: (self.ns + 1) // 2])
        x[-1] = max(x[-1], 0.0)  # the equator ring (cos(pi/2) = 6e-17 in FP64)
        self.W, sigma = _kernel_for(eps)
        self.Nm = 2 * lmax + 1
        self.nk, self.nm = _fft_size(sigma * self.nd), _fft_size(sigma * self.Nm)
        self.beta = float(np.pi * self.W * (1.0 - 0.5 / sigma))
        self.tiles_m = self.nm // _TILE + 2
        dev = torch.device("cuda", device)
        ck = _kernel_ft(self.nd, self.nk, self.W, self.beta)
        cm = _kernel_ft(self.Nm, self.nm, self.W, self.beta)
        self.inv_corr = torch.as_tensor(1.0 / np.outer(ck, cm), device=dev)  # (nd, Nm) centered
        self.kpos = torch.as_tensor(np.arange(-(self.nd // 2), -(self.nd // 2) + self.nd) % self.nk, device=dev)
        self.mpos = torch.as_tensor(np.arange(-lmax, lmax + 1) % self.nm, device=dev)
        mv = np.arange(-lmax, lmax + 1)
        self.sign_m = torch.as_tensor(((-1.0) ** np.abs(mv)) * ((-1.0) ** spin), device=dev)
        self.south = torch.arange(self.ns, self.nd, device=dev)
        self.refl = self.nd - self.south
        self.metric = torch.as_tensor(np.array(alm_metric_weight(lmax)), device=dev)
        with torch.cuda.device(device):
            self.plan = _lib.Plan(0, lmax, spin, "fp64", 1, device=device, rings=(self.ns, x))


@lru_cache(maxsize=None)
def _geometry(lmax: int, spin: int, eps: float, device: int) -> _Geometry:
    return _Geometry(lmax, spin, eps, device)


def _stream():
    return _lib.stream_ptr()


_SORT_MIN_POINTS = 1 << 16  # below this the window reads of unsorted points stay in cache


_TILE = 32  # grid cells per tile edge (kTile in nufft.cu)
_SEG_POINTS = 1024  # points per spread segment


def _tile_keys(g: "_Geometry", theta: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
    two_pi = 2.0 * math.pi
    kb = torch.floor(torch.remainder(torch.nan_to_num(theta), two_pi) * (g.nk / (_TILE * two_pi)))
    mb = torch.floor(torch.remainder(torch.nan_to_num(phi), two_pi) * (g.nm / (_TILE * two_pi)))
    return kb.to(torch.int64) * g.tiles_m + mb.to(torch.int64)


def _point_order(g: "_Geometry", theta: torch.Tensor, phi: torch.Tensor):
    """(permutation, sorted tile keys) grouping the points by 32 x 32-cell tiles of the
    torus grid, so neighbouring threads' windows overlap in L1 / L2 (the grid of a large
    lmax is GBs); None for small point sets."""
    if theta.numel() < _SORT_MIN_POINTS:
        return None
    key = _tile_keys(g, theta, phi)
    ks, order = torch.sort(key)
    return order, ks


def _segments(sorted_keys: torch.Tensor):
    """Segments of at most _SEG_POINTS consecutive sorted points within one tile:
    (first point, count, tile key)."""
    tiles, counts = torch.unique_consecutive(sorted_keys, return_counts=True)
    starts = torch.cumsum(counts, 0) - counts
    nseg = (counts + _SEG_POINTS - 1) // _SEG_POINTS
    seg_tile = torch.repeat_interleave(tiles, nseg)
    first_seg = torch.cumsum(nseg, 0) - nseg
    within = torch.arange(seg_tile.numel(), device=sorted_keys.device) - torch.repeat_interleave(first_seg, nseg)
    seg_start = torch.repeat_interleave(starts, nseg) + within * _SEG_POINTS
    seg_end = torch.repeat_interleave(starts + counts, nseg)
    seg_count = torch.minimum(seg_end - seg_start, torch.full_like(seg_start, _SEG_POINTS)).to(torch.int32)
    return seg_start.contiguous(), seg_count.contiguous(), seg_tile.contiguous()


# ---------------------------------------------------------------------------------------
# forward: alm -> oversampled grid -> points
# ---------------------------------------------------------------------------------------
def _ring_coeffs(g: _Geometry, alm: torch.Tensor) -> torch.Tensor:
    """(ncomp, K) alm -> (ncomp, ns, lmax+1) ring coefficients (+spin, -spin channels)."""
    out = torch.empty((g.ncomp, g.ns, g.lmax + 1), dtype=torch.complex128, device=alm.device)
    st = g.plan.lib.jhtb_legendre_synthesis(g.plan.handle, alm.contiguous().data_ptr(), out.data_ptr(), 1, _stream())
    _lib.check(st, "jhtb_legendre_synthesis")
    return out


def _torus_grid(g: _Geometry, F: torch.Tensor) -> torch.Tensor:
    """Ring coefficients -> samples of the field's torus extension on the nk x nm grid,
    deconvolved by the window's transform (offgrid.py:126-139, _nufft.py:164-174)."""
    L, ns, nd = g.lmax, g.ns, g.nd
    Fp, Fm = F[0], F[-1]
    cols = torch.zeros((nd, g.Nm), dtype=torch.complex128, device=F.device)
    cols[:ns, L:] = Fp
    cols[:ns, :L] = torch.conj(torch.flip(Fm[:, 1:], dims=(1,)))
    cols[g.south] = g.sign_m[None, :] * cols[g.refl]
    # theta FFT (1/nd scaled, as norm="forward"), centred: the shift of an even length is a roll
    Fk = torch.roll(_fft.fft(cols, 0, -1, 1.0 / nd), nd // 2, dims=0)
    # the unscaled inverse 2-D FFT of the zero-padded grid: rows first, only the nd non-zero
    # rows (the other rows stay zero), then every column
    Crow = torch.zeros((nd, g.nm), dtype=torch.complex128, device=F.device)
    Crow[:, g.mpos] = Fk * g.inv_corr
    C = torch.zeros((g.nk, g.nm), dtype=torch.complex128, device=F.device)
    C[g.kpos] = _fft.fft(Crow, 1, +1)
    return _fft.fft(C, 0, +1)


def _interp(g: _Geometry, grid: torch.Tensor, theta: torch.Tensor, phi: torch.Tensor, deriv: bool):
    po = _point_order(g, theta, phi)
    if po is not None:
        order = po[0]
        out = _interp_raw(g, grid, theta[order], phi[order], deriv)
        res = []
        for t in out:
            if t is None:
                res.append(None)
                continue
            r = torch.empty_like(t)
            r[order] = t
            res.append(r)
        return tuple(res)
    return _interp_raw(g, grid, theta, phi, deriv)


def _interp_raw(g: _Geometry, grid: torch.Tensor, theta: torch.Tensor, phi: torch.Tensor, deriv: bool):
    n = theta.numel()
    out = torch.empty(n, dtype=torch.complex128, device=theta.device)
    dth = torch.empty_like(out) if deriv else None
    dph = torch.empty_like(out) if deriv else None
    st = g.plan.lib.jhtb_nufft_interp(
        grid.contiguous().data_ptr(), g.nk, g.nm, g.W, ctypes.c_double(g.beta), theta.data_ptr(), phi.data_ptr(), n,
        out.data_ptr(), dth.data_ptr() if deriv else None, dph.data_ptr() if deriv else None, _stream())
    _lib.check(st, "jhtb_nufft_interp")
    return out, dth, dph


def _forward(g: _Geometry, alm: torch.Tensor, theta, phi, deriv: bool):
    grid = _torus_grid(g, _ring_coeffs(g, alm))
    return _interp(g, grid, theta, phi, deriv)


def _field_of(g: _Geometry, f: torch.Tensor) -> torch.Tensor:
    return f.real.contiguous() if g.spin == 0 else torch.stack([f.real, f.imag])


# ---------------------------------------------------------------------------------------
# adjoint: points -> grid -> ring coefficients -> alm
# ---------------------------------------------------------------------------------------
def _adjoint(g: _Geometry, fc: torch.Tensor, theta: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
    """Complex point values -> (ncomp, K) alm, the transpose of _forward's value path
    divided by the metric (offgrid.py:223-243)."""
    L, ns, nd = g.lmax, g.ns, g.nd
    grid = torch.zeros((g.nk, g.nm), dtype=torch.complex128, device=fc.device)
    po = _point_order(g, theta, phi)
    if po is not None:
        order, keys = po
        fc, theta, phi = fc[order].contiguous(), theta[order].contiguous(), phi[order].contiguous()
        seg_start, seg_count, seg_tile = _segments(keys)
        st = g.plan.lib.jhtb_nufft_spread_tiles(
            fc.data_ptr(), theta.data_ptr(), phi.data_ptr(), theta.numel(), seg_start.numel(), seg_start.data_ptr(),
            seg_count.data_ptr(), seg_tile.data_ptr(), g.tiles_m, g.nk, g.nm, g.W, ctypes.c_double(g.beta),
            grid.data_ptr(), _stream())
        _lib.check(st, "jhtb_nufft_spread_tiles")
    else:
        st = g.plan.lib.jhtb_nufft_spread(fc.contiguous().data_ptr(), theta.data_ptr(), phi.data_ptr(), theta.numel(),
                                          g.nk, g.nm, g.W, ctypes.c_double(g.beta), grid.data_ptr(), _stream())
        _lib.check(st, "jhtb_nufft_spread")
    # the forward 2-D FFT restricted to the nd x Nm centred modes: every column, then the
    # nd rows that are kept; then the scaled inverse theta FFT of the uncentred columns
    G = _fft.fft(_fft.fft(grid, 0, -1)[g.kpos], 1, -1)[:, g.mpos] * g.inv_corr
    d = _fft.fft(torch.roll(G, -(nd // 2), dims=0), 0, +1, 1.0 / nd)
    top = d[:ns].clone()
    top.index_add_(0, g.refl, g.sign_m[None, :] * d[g.south])
    V = torch.zeros((g.ncomp, ns, L + 1), dtype=torch.complex128, device=fc.device)
    Vm = torch.zeros((ns, L + 1), dtype=torch.complex128, device=fc.device)
    Vm[:, 1:] = torch.conj(torch.flip(top[:, :L], dims=(1,)))
    if g.spin == 0:
        V[0] = top[:, L:] + Vm
    else:
        V[0] = top[:, L:]
        V[1] = Vm
    a = torch.empty((g.ncomp, alm_size(L)), dtype=torch.complex128, device=fc.device)
    st = g.plan.lib.jhtb_legendre_adjoint(g.plan.handle, V.data_ptr(), a.data_ptr(), 1, _stream())
    _lib.check(st, "jhtb_legendre_adjoint")
    # the library's spin-2 form is (1/2)(-p - n), (i/2)(p - n); jht's off-grid one has no 1/2
    return (a if g.spin == 0 else 2.0 * a) / g.metric


# ---------------------------------------------------------------------------------------
# autograd
# ---------------------------------------------------------------------------------------
class _SynthesisGeneral(torch.autograd.Function):
    """(ncomp, K) alm, point coordinates -> real field; gradients in alm and in the points."""

    @staticmethod
    def forward(ctx, alm, theta, phi, g):
        deriv = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        f, dth, dph = _forward(g, alm, theta, phi, deriv)
        ctx.g = g
        ctx.save_for_backward(theta, phi, *((dth, dph) if deriv else ()))
        return _field_of(g, f)

    @staticmethod
    def backward(ctx, gf):
        g = ctx.g
        theta, phi, *d = ctx.saved_tensors
        gf = gf.contiguous()
        galm = gth = gph = None
        if ctx.needs_input_grad[0]:
            # same convention as the on-grid synthesis: G-weighted adjoint, m = 0 handled
            # as jht's real / E-B structure requires
            b = _AdjointGeneral.apply(gf, theta, phi, g)
            galm = _synthesis_cotangent(b[None], g.lmax, g.spin)[0]
        if d:
            dth, dph = d
            if g.spin == 0:
                gth, gph = gf * dth.real, gf * dph.real
            else:
                gth = gf[0] * dth.real + gf[1] * dth.imag
                gph = gf[0] * dph.real + gf[1] * dph.imag
        return galm, gth, gph, None


class _AdjointGeneral(torch.autograd.Function):
    """Real field -> (ncomp, K) alm, differentiable in the field."""

    @staticmethod
    def forward(ctx, field, theta, phi, g):
        ctx.g = g
        ctx.save_for_backward(theta, phi)
        fc = torch.complex(field, torch.zeros_like(field)) if g.spin == 0 else torch.complex(field[0], field[1])
        return _adjoint(g, fc, theta, phi)

    @staticmethod
    def backward(ctx, ga):
        g = ctx.g
        theta, phi = ctx.saved_tensors
        a = _adjoint_cotangent_input(ga.contiguous()[None], g.lmax, g.spin)[0]
        f, _, _ = _forward(g, a, theta, phi, False)
        return _field_of(g, f), None, None, None


# ---------------------------------------------------------------------------------------
# public API
# ---------------------------------------------------------------------------------------
def _check_loc(loc) -> torch.Tensor:
    """``loc`` as a tensor where it lies, its shape checked (moved to the device later)."""
    t = _host_tensor(loc)
    if t.dim() != 2 or t.shape[-1] != 2:
        raise ValueError(f"loc must have shape (npts, 2) [theta, phi]; got {tuple(t.shape)}")
    return t


def _check_spin(spin: int) -> None:
    if spin not in (0, 1, 2, 3):
        raise NotImplementedError(f"spin={spin} unsupported (0, 1, 2, 3)")
    if spin not in (0, 2):
        raise NotImplementedError(f"spin={spin}: the off-grid transforms are implemented for spin 0 and 2")


def synthesis_general(alm, loc, *, spin: int = 0, lmax: int, epsilon: float = 1e-10) -> torch.Tensor:
    """``a_lm -> field`` at the points ``loc`` (offgrid.py:181-220).

    ``alm``: ``(alm_size(lmax),)`` (spin 0) or ``(2, alm_size(lmax))`` (E, B);
    ``loc``: ``(npts, 2)`` with ``loc[:, 0] = theta`` (colatitude) and ``loc[:, 1] = phi``,
    evaluated on the 2 pi torus extension (no range check, as jht).  Returns ``(npts,)``
    or ``(2, npts)`` (Q, U).  Differentiable in ``alm`` and in ``loc``.
    """
    _check_spin(spin)
    t = _check_loc(loc)
    a = _host_tensor(alm)
    expect = (alm_size(lmax),) if spin == 0 else (2, alm_size(lmax))
    if tuple(a.shape) != expect:
        raise ValueError(
            f"alm shape {tuple(a.shape)} != expected {expect} for lmax={lmax}, spin={spin} "
            "(a wrong-size alm would otherwise be silently clamped by the gather)"
        )
    a = _as_alm(a)
    t = t.to(device=a.device, dtype=torch.float64)
    g = _geometry(int(lmax), int(spin), float(epsilon), a.device.index)
    theta, phi = t[:, 0].contiguous(), t[:, 1].contiguous()
    return _SynthesisGeneral.apply(a.reshape(g.ncomp, -1), theta, phi, g)


def adjoint_synthesis_general(field, loc, *, spin: int = 0, lmax: int, epsilon: float = 1e-10) -> torch.Tensor:
    """Exact transpose of :func:`synthesis_general`: ``<S_g a, v> = <a, S_g^T v>_G``
    (offgrid.py:223-243).  ``field``: real ``(npts,)`` (spin 0) or ``(2, npts)`` (Q, U)."""
    _check_spin(spin)
    t = _check_loc(loc)
    f = _host_tensor(field)
    if f.is_complex():
        raise TypeError(
            "field must be real ((npts,) for spin=0; (2, npts) real Q/U planes for spin>0); "
            "a complex field would be silently mis-folded"
        )
    npts = t.shape[0]
    expect = (npts,) if spin == 0 else (2, npts)
    if tuple(f.shape) != expect:
        raise ValueError(f"field shape {tuple(f.shape)} != expected {expect} for {npts} points")
    t = t.to(device=_device(), dtype=torch.float64)
    f = f.to(device=t.device, dtype=torch.float64).contiguous()
    g = _geometry(int(lmax), int(spin), float(epsilon), t.device.index)
    theta, phi = t[:, 0].contiguous(), t[:, 1].contiguous()
    out = _AdjointGeneral.apply(f, theta, phi, g)
    return out.reshape(-1) if spin == 0 else out
