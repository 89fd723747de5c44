"""CPU restatement of jht's off-grid transforms (test infrastructure only).

jht's ``synthesis_general`` / ``adjoint_synthesis_general`` (src/jht/offgrid.py) evaluate a
band-limited field at arbitrary points: the Legendre step at a Clenshaw-Curtis theta grid
(offgrid.py:60-88, :155-168), the double-Fourier-sphere extension and a theta FFT
(:113-129), then a 2D type-2 NUFFT with the "exponential of semicircle" kernel
(_nufft.py:83-181).  The adjoint is the exact transpose (type-1 NUFFT, transposed
extension, adjoint contraction), divided by the (2 - delta_m0) metric (offgrid.py:243).

This module restates those steps in NumPy so the CUDA path can be checked against it, and
``direct_field`` sums a_lm sY_lm(theta, phi) point by point as the exact answer.  Only
``tests/`` import it.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

from . import jht_oracle as O

TWO_PI = 2.0 * np.pi

# achievable accuracy -> (kernel width W, oversampling sigma)  (_nufft.py:33-39)
KERNEL_TABLE = {1e-4: (6, 2.0), 1e-6: (8, 2.0), 1e-8: (10, 2.0), 1e-10: (14, 2.0), 1e-12: (16, 2.0)}


def kernel_params(eps: float) -> tuple[int, float]:
    """Cheapest table entry whose accuracy meets ``eps`` (_nufft.py:42-47)."""
    meets = [e for e in KERNEL_TABLE if e <= eps * 1.0000001]
    return KERNEL_TABLE[max(meets)] if meets else KERNEL_TABLE[min(KERNEL_TABLE)]


def smooth_even_size(n: float) -> int:
    """Smallest even 2,3,5-smooth integer >= n (_nufft.py:50-62)."""
    k = int(np.ceil(n))
    k += k % 2
    while True:
        r = k
        for f in (2, 3, 5):
            while r % f == 0:
                r //= f
        if r == 1:
            return k
        k += 2


def es_beta(W: int, sigma: float) -> float:
    return float(np.pi * W * (1.0 - 0.5 / sigma))  # _nufft.py:65-66


def es_kernel(t, beta: float, W: int):
    """exp(beta (sqrt(1 - (2t/W)^2) - 1)) on |t| < W/2, else 0 (_nufft.py:69-84)."""
    z2 = (2.0 * np.asarray(t) / W) ** 2
    inside = z2 < 1.0
    return np.where(inside, np.exp(beta * (np.sqrt(np.where(inside, 1.0 - z2, 1.0)) - 1.0)), 0.0)


def deconv_factor(N: int, n: int, W: int, beta: float) -> np.ndarray:
    """Fourier transform of the kernel at the centered modes of an N-mode axis sampled on n
    points, by Gauss-Legendre quadrature with 2W + 24 nodes (_nufft.py:87-94)."""
    k = np.arange(-(N // 2), -(N // 2) + N)
    nodes, wts = np.polynomial.legendre.leggauss(2 * W + 24)
    t = nodes * (W / 2.0)
    w = wts * (W / 2.0)
    psi = np.exp(beta * (np.sqrt(np.clip(1.0 - (2.0 * t / W) ** 2, 0.0, 1.0)) - 1.0))
    return np.cos(np.outer(k, t) * (TWO_PI / n)) @ (psi * w)


class NufftTables:
    """Sizes and deconvolution factors of a 2D NUFFT with Nk x Nm centered modes (_nufft.py:97-147)."""

    def __init__(self, Nk: int, Nm: int, eps: float):
        self.W, sigma = kernel_params(eps)
        self.Nk, self.Nm = Nk, Nm
        self.nk, self.nm = smooth_even_size(sigma * Nk), smooth_even_size(sigma * Nm)
        self.beta = es_beta(self.W, sigma)
        self.corr_k = deconv_factor(Nk, self.nk, self.W, self.beta)
        self.corr_m = deconv_factor(Nm, self.nm, self.W, self.beta)
        self.kpos = np.arange(-(Nk // 2), -(Nk // 2) + Nk) % self.nk
        self.mpos = np.arange(-(Nm // 2), -(Nm // 2) + Nm) % self.nm


def _window(coord, n: int, W: int, beta: float):
    """Grid indices (mod n) and kernel weights of the W-point window of each coordinate
    (_nufft.py:150-161): the window starts at ceil(u - W/2), u = coord n / 2pi."""
    u = np.asarray(coord, dtype=np.float64) * n / TWO_PI
    first = np.ceil(u - W / 2.0).astype(np.int64)
    idx = first[:, None] + np.arange(W)[None, :]
    return idx % n, es_kernel(u[:, None] - idx, beta, W)


def nufft_type2(tab: NufftTables, coeffs: np.ndarray, theta, phi) -> np.ndarray:
    """f_j = sum_{k,m} coeffs[k, m] e^{i (k theta_j + m phi_j)} (_nufft.py:164-178)."""
    grid = np.zeros((tab.nk, tab.nm), np.complex128)
    grid[np.ix_(tab.kpos, tab.mpos)] = coeffs / tab.corr_k[:, None] / tab.corr_m[None, :]
    g = np.fft.ifft2(grid) * (tab.nk * tab.nm)
    ik, wk = _window(theta, tab.nk, tab.W, tab.beta)
    im, wm = _window(phi, tab.nm, tab.W, tab.beta)
    vals = g[ik[:, :, None], im[:, None, :]]
    return np.einsum("pa,pb,pab->p", wk, wm, vals)


def nufft_type1(tab: NufftTables, vals, theta, phi) -> np.ndarray:
    """coeffs[k, m] = sum_j vals_j e^{-i (k theta_j + m phi_j)}, the transpose of type 2
    (_nufft.py:181-191)."""
    ik, wk = _window(theta, tab.nk, tab.W, tab.beta)
    im, wm = _window(phi, tab.nm, tab.W, tab.beta)
    g = np.zeros((tab.nk, tab.nm), np.complex128)
    contrib = wk[:, :, None] * wm[:, None, :] * np.asarray(vals)[:, None, None]
    np.add.at(g, (ik[:, :, None], im[:, None, :]), contrib)
    C = np.fft.fft2(g)
    return C[np.ix_(tab.kpos, tab.mpos)] / tab.corr_k[:, None] / tab.corr_m[None, :]


class OffgridGeometry:
    """Clenshaw-Curtis theta rings (both poles included) and the NUFFT tables (offgrid.py:60-88)."""

    def __init__(self, lmax: int, spin: int, eps: float):
        if spin not in (0, 2):
            raise NotImplementedError("the restatement covers spin 0 and 2")
        self.lmax, self.spin = lmax, spin
        self.ns = smooth_even_size(lmax + 1) + 1  # rings on [0, pi]
        self.nd = 2 * self.ns - 2  # period of the doubled theta grid
        self.theta = np.arange(self.ns) * np.pi / (self.ns - 1)
        self.x = np.cos(self.theta)
        self.nufft = NufftTables(self.nd, 2 * lmax + 1, eps)
        mv = np.arange(-lmax, lmax + 1)
        self.sign_m = ((-1.0) ** np.abs(mv)) * ((-1.0) ** spin)


@lru_cache(maxsize=None)
def geometry(lmax: int, spin: int, eps: float) -> OffgridGeometry:
    return OffgridGeometry(lmax, spin, eps)


def _ring_coeffs(tab: O.Tables, dense: np.ndarray) -> np.ndarray:
    """C[m, ring] = sum_l pref_l a_lm lambda_lm(x_ring) on every ring (no N/S folding)."""
    M, nr = tab.seed_log.shape
    C = np.zeros((M, nr), np.complex128)
    for l, lam in O._recursion_rows(tab):
        C += (dense[:, l] * tab.pref[l])[:, None] * lam
    return C


def _ring_adjoint(tab: O.Tables, V: np.ndarray) -> np.ndarray:
    """Transpose of :func:`_ring_coeffs`: dense b[m, l] = pref_l sum_ring lambda V."""
    M, _ = tab.seed_log.shape
    b = np.zeros((M, tab.lmax + 1), np.complex128)
    for l, lam in O._recursion_rows(tab):
        b[:, l] = tab.pref[l] * np.sum(lam * V, axis=1)
    return b


def _channels(geo: OffgridGeometry, alm):
    """(+spin, -spin) dense inputs (offgrid.py:96-108)."""
    L = geo.lmax
    if geo.spin == 0:
        d = O.tri_to_dense(np.asarray(alm), L)  # [m, l]
        return d, d
    aE = O.tri_to_dense(np.asarray(alm[0]), L)
    aB = O.tri_to_dense(np.asarray(alm[1]), L)
    return -(aE + 1j * aB), -(aE - 1j * aB)


def fourier_coeffs(geo: OffgridGeometry, Cpos: np.ndarray, Cneg: np.ndarray) -> np.ndarray:
    """Per-m ring coefficients -> centered 2D Fourier coefficients F[k, m] of the doubled
    sphere (offgrid.py:126-139): m < 0 columns are conj(-spin, |m|), theta > pi rows are
    the reflected rows times (-1)^(m + spin); then an FFT over the doubled theta period."""
    L, ns, nd = geo.lmax, geo.ns, geo.nd
    cols = np.zeros((nd, 2 * L + 1), np.complex128)
    cols[:ns, L:] = Cpos.T
    cols[:ns, :L] = np.conj(Cneg[1:][::-1]).T
    j = np.arange(ns, nd)
    cols[j] = geo.sign_m[None, :] * cols[nd - j]
    return np.fft.fftshift(np.fft.fft(cols, axis=0), axes=0) / nd


def fourier_coeffs_adjoint(geo: OffgridGeometry, G: np.ndarray):
    """Transpose of :func:`fourier_coeffs` (offgrid.py:142-152): (Cpos_cot, Cneg_cot)."""
    L, ns, nd = geo.lmax, geo.ns, geo.nd
    d = np.fft.ifft(np.fft.ifftshift(G, axes=0), axis=0)
    top = d[:ns].copy()
    j = np.arange(ns, nd)
    np.add.at(top, nd - j, geo.sign_m[None, :] * d[j])
    cpos = top[:, L:].T
    cneg = np.zeros((L + 1, ns), np.complex128)
    cneg[1:] = np.conj(top[:, :L].T[::-1])
    return cpos, cneg


def _tables(geo: OffgridGeometry):
    tp = O.Tables(geo.x, geo.spin, geo.lmax)
    tm = tp if geo.spin == 0 else O.Tables(geo.x, -geo.spin, geo.lmax)
    return tp, tm


def synthesis_general(alm, loc, lmax: int, spin: int = 0, eps: float = 1e-10) -> np.ndarray:
    """Field at the points ``loc = [[theta, phi], ...]`` (offgrid.py:181-220)."""
    geo = geometry(lmax, spin, eps)
    tp, tm = _tables(geo)
    a, b = _channels(geo, alm)
    cpos = _ring_coeffs(tp, a)
    cneg = cpos if spin == 0 else _ring_coeffs(tm, b)
    f = nufft_type2(geo.nufft, fourier_coeffs(geo, cpos, cneg), loc[:, 0], loc[:, 1])
    return f.real if spin == 0 else np.stack([f.real, f.imag])


def adjoint_synthesis_general(field, loc, lmax: int, spin: int = 0, eps: float = 1e-10) -> np.ndarray:
    """Exact transpose of :func:`synthesis_general` in the (2 - delta_m0) metric (offgrid.py:223-243)."""
    geo = geometry(lmax, spin, eps)
    tp, tm = _tables(geo)
    fc = np.asarray(field, np.complex128) if spin == 0 else field[0] + 1j * field[1]
    G = nufft_type1(geo.nufft, fc, loc[:, 0], loc[:, 1])
    cpos, cneg = fourier_coeffs_adjoint(geo, G)
    pc = _ring_adjoint(tp, cpos)
    nc = _ring_adjoint(tm, cneg)
    gm = O.metric_weight(lmax)
    if spin == 0:
        return O.dense_to_tri(pc + nc, lmax) / gm
    aE = O.dense_to_tri(-(pc + nc), lmax)
    aB = O.dense_to_tri(1j * (pc - nc), lmax)
    return np.stack([aE, aB]) / gm[None, :]


def direct_field(alm, loc, lmax: int, spin: int = 0) -> np.ndarray:
    """sum_lm a_lm sY_lm(theta_j, phi_j) point by point: the exact answer the NUFFT approximates."""
    th, ph = np.asarray(loc[:, 0]), np.asarray(loc[:, 1])
    x = np.cos(th)
    if spin == 0:
        f = np.zeros(x.shape)
        for m in range(lmax + 1):
            b = O.alm_base(m, lmax)
            Fm = np.asarray(alm)[b : b + lmax + 1 - m] @ O.lambda_column(x, m, lmax)
            f += Fm.real if m == 0 else 2.0 * (Fm * np.exp(1j * m * ph)).real
        return f
    aE, aB = np.asarray(alm[0]), np.asarray(alm[1])
    out = np.zeros(x.shape, np.complex128)
    for m in range(lmax + 1):
        lmin = max(m, spin)
        b = O.alm_base(m, lmax) + (lmin - m)
        e, bb = aE[b : O.alm_base(m, lmax) + lmax + 1 - m], aB[b : O.alm_base(m, lmax) + lmax + 1 - m]
        lp = O.spin_lambda_column(x, m, spin, lmax)
        lm = O.spin_lambda_column(x, m, -spin, lmax)
        fp = (-(e + 1j * bb)) @ lp
        fm = (-(e - 1j * bb)) @ lm
        out += fp * np.exp(1j * m * ph)
        if m >= 1:
            out += np.conj(fm) * np.exp(-1j * m * ph)
    return np.stack([out.real, out.imag])
