"""CPU oracle for jht's on-grid HEALPix spherical-harmonic transform (FP64, NumPy).

TEST INFRASTRUCTURE ONLY.  This module restates, in plain NumPy, the algorithm
of the reference implementation (jht v0.2.0, ``src/jht``) so that the CUDA path
in ``jht_b200`` can be checked against it.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it;
the product never does.

Pinning.  The restatement is pinned against golden vectors produced by running
the reference's own source (``tests/golden/make_golden.py``), against the
closed-form Y_lm for l <= 2, ``scipy.special.sph_harm_y`` to l = 512, the
explicit Wigner-d sum and a 50-digit mpmath recursion (``tests/test_oracle.py``).

Each function cites the reference lines it follows.  The heavy recursion +
contraction loop also exists as C (``legendre_ref.c``) for large sizes; the
Python and C versions implement the same per-step log-renormalised recursion.
"""

from __future__ import annotations

import math
from functools import lru_cache

import numpy as np
from numpy.polynomial.legendre import legvander

# --------------------------------------------------------------------------------------
# a_lm layout (healpix.py:49-101)
# --------------------------------------------------------------------------------------


def alm_size(lmax: int) -> int:
    """Number of m>=0 coefficients, healpy packing (healpix.py:49-50)."""
    return (lmax + 1) * (lmax + 2) // 2


def alm_base(m: int, lmax: int) -> int:
    """Flat index of a_{m,m}; a_{l,m} sits at ``alm_base(m) + l - m`` (healpix.py:53-55)."""
    return m * (2 * lmax + 1 - m) // 2 + m


@lru_cache(maxsize=None)
def lm_of_index(lmax: int) -> tuple[np.ndarray, np.ndarray]:
    ells = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    ms = np.concatenate([np.full(lmax + 1 - m, m) for m in range(lmax + 1)])
    return ells, ms


def metric_weight(lmax: int) -> np.ndarray:
    """``2 - delta_{m0}`` per packed coefficient (healpix.py:58-74)."""
    _, ms = lm_of_index(lmax)
    return np.where(ms == 0, 1.0, 2.0)


def tri_to_dense(alm: np.ndarray, lmax: int) -> np.ndarray:
    """Packed (K,) -> dense (M, lmax+1) with zeros for l < m (healpix.py:77-101, :260-261)."""
    M = lmax + 1
    dense = np.zeros((M, M), dtype=np.complex128)
    for m in range(M):
        b = alm_base(m, lmax)
        dense[m, m:] = alm[b : b + lmax + 1 - m]
    return dense


def dense_to_tri(dense: np.ndarray, lmax: int) -> np.ndarray:
    """Dense (M, lmax+1) -> packed (K,) (healpix.py:263-264)."""
    out = np.empty(alm_size(lmax), dtype=np.complex128)
    for m in range(lmax + 1):
        b = alm_base(m, lmax)
        out[b : b + lmax + 1 - m] = dense[m, m:]
    return out


# --------------------------------------------------------------------------------------
# RING geometry (healpix.py:107-140)
# --------------------------------------------------------------------------------------


class Rings:
    """Per-ring z = cos(theta), pixel count, first-pixel azimuth and start pixel."""

    def __init__(self, nside: int):
        idx = np.arange(1, 4 * nside, dtype=np.int64)  # 1-based ring number
        n = np.empty_like(idx)
        z = np.empty(idx.shape)
        phi0 = np.empty(idx.shape)
        north = idx < nside
        south = idx > 3 * nside
        belt = ~north & ~south
        n[north] = 4 * idx[north]
        z[north] = 1.0 - idx[north] ** 2 / (3.0 * nside**2)
        phi0[north] = np.pi / (4.0 * idx[north])
        j = 4 * nside - idx[south]
        n[south] = 4 * j
        z[south] = -(1.0 - j**2 / (3.0 * nside**2))
        phi0[south] = np.pi / (4.0 * j)
        k = idx[belt]
        n[belt] = 4 * nside
        z[belt] = 4.0 / 3.0 - 2.0 * k / (3.0 * nside)
        phi0[belt] = np.where((k - nside) % 2 == 0, np.pi / (4.0 * nside), 0.0)
        self.nside = nside
        self.npix = 12 * nside * nside
        self.nrings = idx.size
        self.z = z
        self.nring = n
        self.phi0 = phi0
        self.start = np.concatenate([[0], np.cumsum(n)[:-1]])


# --------------------------------------------------------------------------------------
# recursion coefficients and seeds (_recursion.py:37-56, :136-188, :277-335)
# --------------------------------------------------------------------------------------


def legendre_ab(m: int, lmax: int) -> tuple[np.ndarray, np.ndarray]:
    """``lambda_l = a_l x lambda_{l-1} - b_l lambda_{l-2}`` for l = m+1..lmax (_recursion.py:37-50)."""
    l = np.arange(m + 1, lmax + 1, dtype=np.float64)
    a = np.sqrt((2 * l - 1) * (2 * l + 1) / ((l - m) * (l + m)))
    b = np.sqrt((2 * l + 1) * ((l - 1) ** 2 - m * m) / ((2 * l - 3) * (l - m) * (l + m)))
    return a, b


def sectoral_log_const(m: int) -> float:
    """theta-independent part of log|lambda_mm| (_recursion.py:53-56)."""
    k = np.arange(1, m + 1, dtype=np.float64)
    return float(-0.5 * np.log(4 * np.pi) + 0.5 * np.sum(np.log((2 * k + 1) / (2 * k))))


def wigner_acb(M: int, Mp: int, lmin: int, lmax: int):
    """A_l, C_l, B_l for l = lmin..lmax-1, producing d^{l+1}_{M,M'} (_recursion.py:136-143)."""
    l = np.arange(lmin, lmax, dtype=np.float64)
    D = l * np.sqrt(((l + 1) ** 2 - M * M) * ((l + 1) ** 2 - Mp * Mp))
    A = (2 * l + 1) * l * (l + 1) / D
    C = -(2 * l + 1) * M * Mp / D
    B = (l + 1) * np.sqrt((l * l - M * M) * (l * l - Mp * Mp)) / D
    return A, C, B


def wigner_seed(x: np.ndarray, M: int, Mp: int, lmin: int) -> tuple[float, np.ndarray]:
    """Single-term d^{lmin}_{M,M'}: (sign, log|d|) (_recursion.py:166-188)."""
    k0 = max(0, M - Mp)
    lg = math.lgamma
    logc = 0.5 * (lg(lmin + M + 1) + lg(lmin - M + 1) + lg(lmin + Mp + 1) + lg(lmin - Mp + 1)) - (
        lg(k0 + 1) + lg(lmin + M - k0 + 1) + lg(lmin - Mp - k0 + 1) + lg(k0 - M + Mp + 1)
    )
    sign = -1.0 if k0 % 2 else 1.0
    pc = 2 * lmin - 2 * k0 + M - Mp
    ps = 2 * k0 - M + Mp
    ch = np.sqrt(np.clip((1 + x) / 2, 0, 1))
    sh = np.sqrt(np.clip((1 - x) / 2, 0, 1))
    logd = np.full(x.shape, logc, dtype=np.float64)
    with np.errstate(divide="ignore"):
        if pc > 0:
            logd = logd + pc * np.log(ch)
        if ps > 0:
            logd = logd + ps * np.log(sh)
    return sign, logd


class Tables:
    """Dense all-m recursion tables for one spin (_recursion.py:257-335).

    ``A, B, C, pref`` are (lmax+1, M) l-major grids; ``seed_sign`` (M,),
    ``seed_log`` (M, T); ``lmin[m] = max(m, |spin|)``.
    """

    def __init__(self, x: np.ndarray, spin: int, lmax: int):
        x = np.asarray(x, dtype=np.float64)
        M = lmax + 1
        self.spin, self.lmax, self.x = spin, lmax, x
        self.lmin = np.maximum(np.arange(M), abs(spin))
        self.A = np.zeros((M, M))
        self.B = np.zeros((M, M))
        self.C = np.zeros((M, M))
        self.seed_sign = np.zeros(M)
        self.seed_log = np.zeros((M, x.size))
        if spin == 0:
            self.pref = np.ones((M, M))
            sin_t = np.sqrt(np.clip(1 - x * x, 0, 1))
            with np.errstate(divide="ignore"):
                logsin = np.log(sin_t)
            for m in range(M):
                a, b = legendre_ab(m, lmax)
                self.A[m + 1 :, m] = a
                self.B[m + 1 :, m] = b
                self.seed_sign[m] = 1.0 if m % 2 == 0 else -1.0
                c = sectoral_log_const(m)
                self.seed_log[m] = c if m == 0 else c + m * logsin
        else:
            ell = np.arange(M, dtype=np.float64)
            self.pref = ((-1.0) ** np.arange(M))[None, :] * np.sqrt((2 * ell + 1) / (4 * np.pi))[:, None]
            for m in range(M):
                lm = int(self.lmin[m])
                if lm < lmax:
                    A, C, B = wigner_acb(-m, spin, lm, lmax)
                    self.A[lm + 1 :, m] = A
                    self.C[lm + 1 :, m] = C
                    self.B[lm + 1 :, m] = B
                self.seed_sign[m], self.seed_log[m] = wigner_seed(x, -m, spin, lm)


def _recursion_rows(tab: Tables):
    """Yield ``(l, lam)`` with lam the (M, T) row lambda_{l,m}(x) (no pref), l = 0..lmax.

    One log-renormalised step per l for all m at once (_recursion.py:352-369):
    the carried pair is rescaled to unit norm and the log of the scale is kept.
    """
    M, T = tab.seed_log.shape
    x = tab.x[None, :]
    p = np.zeros((M, T))
    q = np.zeros((M, T))
    s = np.zeros((M, T))
    for l in range(tab.lmax + 1):
        raw = (tab.A[l][:, None] * x + tab.C[l][:, None]) * p - tab.B[l][:, None] * q
        r = np.sqrt(raw * raw + p * p)
        r = np.where(r == 0.0, 1.0, r)
        with np.errstate(divide="ignore"):
            rp, rq, rs = raw / r, p / r, s + np.log(r)
        seed = (tab.lmin == l)[:, None]
        active = (tab.lmin <= l)[:, None]
        recur = active & ~seed
        p = np.where(seed, tab.seed_sign[:, None], np.where(recur, rp, p))
        q = np.where(seed, 0.0, np.where(recur, rq, q))
        s = np.where(seed, tab.seed_log, np.where(recur, rs, s))
        with np.errstate(under="ignore", over="ignore"):
            lam = np.where(active, p * np.exp(s), 0.0)
        yield l, lam


def synth_contract(tab: Tables, alm_dense: np.ndarray):
    """Half-grid synthesis, spin 0: ``(F_total, F_signed)`` (_recursion.py:441-469)."""
    M, T = tab.seed_log.shape
    Ft = np.zeros((M, T), np.complex128)
    Fs = np.zeros((M, T), np.complex128)
    for l, lam in _recursion_rows(tab):
        c = (alm_dense[:, l] * tab.pref[l])[:, None] * lam
        Ft += c
        Fs += c if l % 2 == 0 else -c
    return Ft, Fs


def adjoint_contract(tab: Tables, Vn: np.ndarray, Vs: np.ndarray) -> np.ndarray:
    """Half-grid adjoint, spin 0: dense b (_recursion.py:472-497)."""
    M, _ = tab.seed_log.shape
    b = np.zeros((M, tab.lmax + 1), np.complex128)
    for l, lam in _recursion_rows(tab):
        par = 1.0 if l % 2 == 0 else -1.0
        b[:, l] = tab.pref[l] * (np.sum(lam * Vn, axis=1) + par * np.sum(lam * Vs, axis=1))
    return b


def synth_contract_spin2(tp: Tables, tm: Tables, bp: np.ndarray, bm: np.ndarray):
    """Two-state +-2 half-grid synthesis: (FpN, FpS, FmN, FmS) (_recursion.py:512-543)."""
    M, T = tp.seed_log.shape
    FpN, FpS, FmN, FmS = (np.zeros((M, T), np.complex128) for _ in range(4))
    for (l, lp), (_, lm) in zip(_recursion_rows(tp), _recursion_rows(tm)):
        par = 1.0 if l % 2 == 0 else -1.0
        cp = (bp[:, l] * tp.pref[l])[:, None]
        cm = (bm[:, l] * tp.pref[l])[:, None]
        FpN += cp * lp
        FpS += par * cp * lm
        FmN += cm * lm
        FmS += par * cm * lp
    return FpN, FpS, FmN, FmS


def adjoint_contract_spin2(tp: Tables, tm: Tables, Vpn, Sp, Vmn, Sm):
    """Two-state +-2 half-grid adjoint: dense (p2, m2) (_recursion.py:546-572)."""
    M, _ = tp.seed_log.shape
    p2 = np.zeros((M, tp.lmax + 1), np.complex128)
    m2 = np.zeros((M, tp.lmax + 1), np.complex128)
    for (l, lp), (_, lm) in zip(_recursion_rows(tp), _recursion_rows(tm)):
        par = 1.0 if l % 2 == 0 else -1.0
        p2[:, l] = tp.pref[l] * (np.sum(lp * Vpn, axis=1) + par * np.sum(lm * Sp, axis=1))
        m2[:, l] = tp.pref[l] * (np.sum(lm * Vmn, axis=1) + par * np.sum(lp * Sm, axis=1))
    return p2, m2


# --------------------------------------------------------------------------------------
# C acceleration of the same recursion (optional; used at large sizes)
# --------------------------------------------------------------------------------------


def _clib():
    from . import _cref  # local import: only when a large case asks for it

    return _cref.load()


# --------------------------------------------------------------------------------------
# north/south fold and the azimuthal stage (healpix.py:241-258, :280-357)
# --------------------------------------------------------------------------------------


def _build_full(geo: Rings, Fn: np.ndarray, Fs: np.ndarray) -> np.ndarray:
    """(M, T) north + signed south -> (M, nrings) with the (-1)^m mirror (healpix.py:250-253)."""
    M, T = Fn.shape
    F = np.zeros((M, geo.nrings), np.complex128)
    F[:, :T] = Fn
    src = np.arange(T - 1)
    sign_m = ((-1.0) ** np.arange(M))[:, None]
    F[:, 4 * geo.nside - 2 - src] = sign_m * Fs[:, src]
    return F


def _fold_south(geo: Rings, V: np.ndarray):
    """(M, nrings) -> (Vn, (-1)^m V_south) on the half grid (healpix.py:255-258)."""
    M = V.shape[0]
    T = 2 * geo.nside
    src = np.arange(T - 1)
    Vs = np.zeros((M, T), np.complex128)
    Vs[:, src] = V[:, 4 * geo.nside - 2 - src]
    return V[:, :T], ((-1.0) ** np.arange(M))[:, None] * Vs


def rings_synth(geo: Rings, Gp: np.ndarray, Gm: np.ndarray, lmax: int) -> np.ndarray:
    """Per ring: fold +m and conj(-m) columns mod N, inverse DFT times N (healpix.py:283-291, :319-330).

    ``Gp, Gm`` are (M, nrings) already multiplied by exp(i m phi0).  Returns
    complex ring samples in RING pixel order.
    """
    m = np.arange(lmax + 1)
    out = np.empty(geo.npix, np.complex128)
    for N in np.unique(geo.nring):
        rows = np.flatnonzero(geo.nring == N)
        D = np.zeros((rows.size, N), np.complex128)
        np.add.at(D, (slice(None), m % N), Gp[:, rows].T)
        np.add.at(D, (slice(None), (-m[1:]) % N), np.conj(Gm[1:, rows].T))
        y = np.fft.ifft(D, axis=1) * N
        for k, r in enumerate(rows):
            out[geo.start[r] : geo.start[r] + N] = y[k]
    return out


def rings_adjoint(geo: Rings, ring_data: np.ndarray, lmax: int):
    """Per ring: forward DFT, gather columns m mod N and (-m) mod N (healpix.py:299-303, :343-349).

    Returns ``(Wp, Wm)`` of shape (M, nrings) *before* the conjugate phase:
    ``Wp[m] = W[m mod N]`` and ``Wm[m] = conj(W[(-m) mod N])``.
    """
    m = np.arange(lmax + 1)
    Wp = np.zeros((lmax + 1, geo.nrings), np.complex128)
    Wm = np.zeros((lmax + 1, geo.nrings), np.complex128)
    for N in np.unique(geo.nring):
        rows = np.flatnonzero(geo.nring == N)
        pix = geo.start[rows][:, None] + np.arange(N)[None, :]
        W = np.fft.fft(ring_data[pix], axis=1)
        Wp[:, rows] = W[:, m % N].T
        Wm[:, rows] = np.conj(W[:, (-m) % N]).T
    return Wp, Wm


def _phase(geo: Rings, lmax: int) -> np.ndarray:
    """exp(i m phi0_r), (M, nrings) (healpix.py:222-225)."""
    return np.exp(1j * np.arange(lmax + 1)[:, None] * geo.phi0[None, :])


# --------------------------------------------------------------------------------------
# public transforms (healpix.py:363-412)
# --------------------------------------------------------------------------------------


def _check_spin(spin: int) -> None:
    if spin not in (0, 2):
        raise NotImplementedError(f"spin={spin} unsupported (only 0 and 2)")


def synthesis(alm, nside: int, lmax: int, spin: int = 0, use_c: bool | None = None) -> np.ndarray:
    """S: packed alm -> RING map; (K,) -> (Npix,) spin 0, (2, K) -> (2, Npix) spin 2."""
    _check_spin(spin)
    alm = np.asarray(alm, dtype=np.complex128)
    geo = Rings(nside)
    T = 2 * nside
    x = geo.z[:T]
    if use_c is None:
        use_c = (lmax + 1) * T > 200_000
    if spin == 0:
        if use_c:
            Ft, Fs = _clib().synth(0, lmax, x, alm[None, :])
        else:
            Ft, Fs = synth_contract(Tables(x, 0, lmax), tri_to_dense(alm, lmax))
        G = _build_full(geo, Ft, Fs) * _phase(geo, lmax)
        return np.real(rings_synth(geo, G, G, lmax))
    if use_c:
        FpN, FpS, FmN, FmS = _clib().synth(2, lmax, x, alm)
    else:
        aE, aB = tri_to_dense(alm[0], lmax), tri_to_dense(alm[1], lmax)
        FpN, FpS, FmN, FmS = synth_contract_spin2(
            Tables(x, 2, lmax), Tables(x, -2, lmax), -(aE + 1j * aB), -(aE - 1j * aB)
        )
    ph = _phase(geo, lmax)
    qu = rings_synth(geo, _build_full(geo, FpN, FpS) * ph, _build_full(geo, FmN, FmS) * ph, lmax)
    return np.stack([qu.real, qu.imag])


def adjoint_synthesis(maps, nside: int, lmax: int, spin: int = 0, use_c: bool | None = None) -> np.ndarray:
    """S^T: RING map -> packed alm, the exact transpose of :func:`synthesis`."""
    _check_spin(spin)
    maps = np.asarray(maps, dtype=np.float64)
    geo = Rings(nside)
    T = 2 * nside
    x = geo.z[:T]
    cph = np.conj(_phase(geo, lmax))
    if use_c is None:
        use_c = (lmax + 1) * T > 200_000
    if spin == 0:
        Wp, _ = rings_adjoint(geo, maps.astype(np.complex128), lmax)
        Vn, Vs = _fold_south(geo, Wp * cph)
        if use_c:
            return _clib().adjoint(0, lmax, x, [Vn, Vs])[0]
        return dense_to_tri(adjoint_contract(Tables(x, 0, lmax), Vn, Vs), lmax)
    Wp, Wm = rings_adjoint(geo, maps[0] + 1j * maps[1], lmax)
    Vpn, Sp = _fold_south(geo, Wp * cph)
    Vmn, Sm = _fold_south(geo, Wm * cph)
    if use_c:
        p2, m2 = _clib().adjoint(2, lmax, x, [Vpn, Sp, Vmn, Sm])
    else:
        p2d, m2d = adjoint_contract_spin2(Tables(x, 2, lmax), Tables(x, -2, lmax), Vpn, Sp, Vmn, Sm)
        p2, m2 = dense_to_tri(p2d, lmax), dense_to_tri(m2d, lmax)
    return np.stack([0.5 * (-p2 - m2), 0.5 * (1j * p2 - 1j * m2)])


# --------------------------------------------------------------------------------------
# eager per-m / per-ring forms (_reference.py:22-143) and per-m lambda columns
# --------------------------------------------------------------------------------------


def lambda_column(x, m: int, lmax: int) -> np.ndarray:
    """lambda_{l,m}(x), l = m..lmax, one log-renormalised scan (_recursion.py:59-117)."""
    x = np.asarray(x, dtype=np.float64)
    sin_t = np.sqrt(np.clip(1 - x * x, 0, 1))
    c = sectoral_log_const(m)
    if m == 0:
        s = np.full(x.shape, c)
    else:
        with np.errstate(divide="ignore"):
            s = c + m * np.log(sin_t)
    p = np.full(x.shape, 1.0 if m % 2 == 0 else -1.0)
    q = np.zeros_like(x)
    rows = [p * np.exp(s)]
    a, b = legendre_ab(m, lmax)
    for i in range(a.size):
        raw = a[i] * x * p - b[i] * q
        r = np.sqrt(raw * raw + p * p)
        r = np.where(r == 0, 1.0, r)
        p, q, s = raw / r, p / r, s + np.log(r)
        rows.append(p * np.exp(s))
    return np.array(rows)


def wigner_column(x, M: int, Mp: int, lmax: int) -> np.ndarray:
    """d^l_{M,M'}(x), l = max(|M|,|M'|)..lmax (_recursion.py:191-221)."""
    x = np.asarray(x, dtype=np.float64)
    lmin = max(abs(M), abs(Mp))
    sign, s = wigner_seed(x, M, Mp, lmin)
    p = np.full(x.shape, sign)
    q = np.zeros_like(x)
    with np.errstate(under="ignore"):
        rows = [p * np.exp(s)]
    if lmax > lmin:
        A, C, B = wigner_acb(M, Mp, lmin, lmax)
        for i in range(A.size):
            raw = (A[i] * x + C[i]) * p - B[i] * q
            r = np.sqrt(raw * raw + p * p)
            r = np.where(r == 0, 1.0, r)
            p, q, s = raw / r, p / r, s + np.log(r)
            with np.errstate(under="ignore"):
                rows.append(p * np.exp(s))
    return np.array(rows)


def spin_lambda_column(x, m: int, spin: int, lmax: int) -> np.ndarray:
    """{}_s lambda_{l,m}, l = max(m,|s|)..lmax (_recursion.py:224-235)."""
    lmin = max(m, abs(spin))
    d = wigner_column(x, -m, spin, lmax)
    ell = np.arange(lmin, lmax + 1, dtype=np.float64)
    return (((-1.0) ** m) * np.sqrt((2 * ell + 1) / (4 * np.pi)))[:, None] * d


def synthesis_eager(alm, nside: int, lmax: int, spin: int = 0) -> np.ndarray:
    """Per-m / per-ring synthesis (_reference.py:106-120, :55-70)."""
    geo = Rings(nside)
    x = geo.z
    mm = np.arange(lmax + 1)
    alm = np.asarray(alm, dtype=np.complex128)
    if spin == 0:
        F = np.array([alm[alm_base(m, lmax) : alm_base(m, lmax) + lmax + 1 - m] @ lambda_column(x, m, lmax) for m in mm])
        out = []
        for r in range(geo.nrings):
            N = int(geo.nring[r])
            g = F[:, r] * np.exp(1j * mm * geo.phi0[r])
            D = np.zeros(N, np.complex128)
            np.add.at(D, mm % N, g)
            np.add.at(D, (-mm[1:]) % N, np.conj(g[1:]))
            out.append(np.real(np.fft.ifft(D) * N))
        return np.concatenate(out)
    Fp, Fm = [], []
    for m in mm:
        lmin = max(m, 2)
        b = alm_base(m, lmax) + lmin - m
        e, bb = alm[0, b : alm_base(m, lmax) + lmax + 1 - m], alm[1, b : alm_base(m, lmax) + lmax + 1 - m]
        Fp.append(-(e + 1j * bb) @ spin_lambda_column(x, m, 2, lmax))
        Fm.append(-(e - 1j * bb) @ spin_lambda_column(x, m, -2, lmax))
    Fp, Fm = np.array(Fp), np.array(Fm)
    q, u = [], []
    for r in range(geo.nrings):
        N = int(geo.nring[r])
        ph = np.exp(1j * mm * geo.phi0[r])
        D = np.zeros(N, np.complex128)
        np.add.at(D, mm % N, Fp[:, r] * ph)
        np.add.at(D, (-mm[1:]) % N, np.conj(Fm[1:, r] * ph[1:]))
        y = np.fft.ifft(D) * N
        q.append(y.real)
        u.append(y.imag)
    return np.stack([np.concatenate(q), np.concatenate(u)])


def adjoint_eager(maps, nside: int, lmax: int, spin: int = 0) -> np.ndarray:
    """Per-ring / per-m adjoint (_reference.py:123-143, :73-103)."""
    geo = Rings(nside)
    x = geo.z
    mm = np.arange(lmax + 1)
    maps = np.asarray(maps, dtype=np.float64)
    if spin == 0:
        cols = []
        for r in range(geo.nrings):
            N = int(geo.nring[r])
            f = np.fft.fft(maps[geo.start[r] : geo.start[r] + N])
            cols.append(f[mm % N] * np.exp(-1j * mm * geo.phi0[r]))
        V = np.stack(cols, axis=1)
        return np.concatenate([lambda_column(x, m, lmax) @ V[m] for m in mm])
    fp, fm = [], []
    for r in range(geo.nrings):
        N = int(geo.nring[r])
        s = geo.start[r]
        W = np.fft.fft(maps[0][s : s + N] + 1j * maps[1][s : s + N])
        ph = np.exp(-1j * mm * geo.phi0[r])
        fp.append(W[mm % N] * ph)
        fm.append(np.conj(W[(-mm) % N]) * ph)
    Fp, Fm = np.stack(fp, axis=1), np.stack(fm, axis=1)
    aE, aB = [], []
    for m in mm:
        lmin = max(m, 2)
        p2 = spin_lambda_column(x, m, 2, lmax) @ Fp[m]
        m2 = spin_lambda_column(x, m, -2, lmax) @ Fm[m]
        e, b = 0.5 * (-p2 - m2), 0.5 * (1j * p2 - 1j * m2)
        pad = np.zeros(lmin - m, np.complex128)
        aE.append(np.concatenate([pad, e]))
        aB.append(np.concatenate([pad, b]))
    return np.stack([np.concatenate(aE), np.concatenate(aB)])


# --------------------------------------------------------------------------------------
# quadrature weights (weights.py:60-106) and analysis (_analysis.py:34-67)
# --------------------------------------------------------------------------------------


@lru_cache(maxsize=None)
def ring_weights(nside: int) -> np.ndarray:
    """Min-norm per-ring weight deviations w (length 2*nside) (weights.py:60-83)."""
    geo = Rings(nside)
    T = 2 * nside
    z = geo.z[:T]
    n = geo.nring[:T].astype(np.float64)
    mult = np.full(T, 2.0)
    mult[-1] = 1.0
    P = legvander(z, 2 * nside)[:, ::2]
    A = ((mult * n)[:, None] * P).T
    rhs = -A.sum(axis=1)
    rhs[0] += geo.npix
    w, *_ = np.linalg.lstsq(A, rhs, rcond=None)
    return w


@lru_cache(maxsize=None)
def pixel_weights(nside: int, use_weights: bool = True) -> np.ndarray:
    """Per-pixel quadrature weights in RING order (weights.py:86-106)."""
    geo = Rings(nside)
    base = 4 * np.pi / geo.npix
    if not use_weights:
        return np.full(geo.npix, base)
    w = ring_weights(nside)
    r = np.arange(geo.nrings)
    half = np.where(r < 2 * nside, r, 4 * nside - 2 - r)
    return base * (1.0 + np.repeat(w[half], geo.nring))


def bare_analysis(maps, nside, lmax, spin=0, use_weights=True, use_c=None):
    """A0 = S^T W (_analysis.py:49-52)."""
    return adjoint_synthesis(pixel_weights(nside, use_weights) * np.asarray(maps), nside, lmax, spin, use_c)


def analysis(maps, nside, lmax, spin=0, niter=3, use_weights=True, use_c=None):
    """A0 then ``niter`` Jacobi steps a += A0(m - S a) (_analysis.py:55-63)."""
    maps = np.asarray(maps, dtype=np.float64)
    a = bare_analysis(maps, nside, lmax, spin, use_weights, use_c)
    for _ in range(niter):
        r = maps - synthesis(a, nside, lmax, spin, use_c)
        a = a + bare_analysis(r, nside, lmax, spin, use_weights, use_c)
    return a


# --------------------------------------------------------------------------------------
# real-DOF isometry (masked.py:117-175) and CG deconvolution (masked.py:234-314)
# --------------------------------------------------------------------------------------


def _dof_idx(lmax: int, spin: int):
    ells, ms = lm_of_index(lmax)
    act = ells >= abs(spin)
    idx = np.arange(alm_size(lmax))
    return idx[act & (ms == 0)], idx[act & (ms > 0)]


def n_dof(lmax: int, spin: int = 0) -> int:
    k0, kp = _dof_idx(lmax, spin)
    n = k0.size + 2 * kp.size
    return n if spin == 0 else 2 * n


def alm_to_real(alm, lmax: int, spin: int = 0) -> np.ndarray:
    k0, kp = _dof_idx(lmax, spin)
    r2 = math.sqrt(2.0)

    def one(a):
        return np.concatenate([a[k0].real, r2 * a[kp].real, r2 * a[kp].imag])

    a = np.asarray(alm)
    return one(a) if spin == 0 else np.concatenate([one(a[0]), one(a[1])])


def real_to_alm(x, lmax: int, spin: int = 0) -> np.ndarray:
    k0, kp = _dof_idx(lmax, spin)
    r2 = math.sqrt(2.0)

    def one(v):
        a = np.zeros(alm_size(lmax), np.complex128)
        a[k0] = v[: k0.size]
        a[kp] = (v[k0.size : k0.size + kp.size] + 1j * v[k0.size + kp.size :]) / r2
        return a

    x = np.asarray(x, dtype=np.float64)
    if spin == 0:
        return one(x)
    h = x.size // 2
    return np.stack([one(x[:h]), one(x[h:])])


def cg(A, b, x0=None, tol=1e-5, maxiter=None):
    """Plain CG, stop when |r|^2 <= tol^2 |b|^2 (jax.scipy.sparse.linalg.cg rule)."""
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    maxiter = 10 * b.size if maxiter is None else maxiter
    thr = tol * tol * float(b @ b)
    r = b - A(x)
    p = r.copy()
    g = float(r @ r)
    k = 0
    while g > thr and k < maxiter:
        Ap = A(p)
        al = g / float(p @ Ap)
        x = x + al * p
        r = r - al * Ap
        g2 = float(r @ r)
        p = r + (g2 / g) * p
        g = g2
        k += 1
    return x, k


def deconvolve(maps, mask, nside, lmax, spin=0, *, max_iter=200, tol=1e-8, reg=0.0, use_weights=True, x0=None):
    """CG on S^T(MW)S a = S^T(MW) m in real-DOF coordinates (masked.py:278-314)."""
    w = np.asarray(mask) * pixel_weights(nside, use_weights)
    w = w if spin == 0 else w[None, :]
    b = alm_to_real(adjoint_synthesis(w * np.asarray(maps), nside, lmax, spin), lmax, spin)

    def op(x):
        a = real_to_alm(x, lmax, spin)
        return alm_to_real(adjoint_synthesis(w * synthesis(a, nside, lmax, spin), nside, lmax, spin), lmax, spin) + reg * x

    xi = None if x0 is None else alm_to_real(x0, lmax, spin)
    xs, _ = cg(op, b, xi, tol=tol, maxiter=max_iter)
    return real_to_alm(xs, lmax, spin)


def weight_pix(nside, spin, *, inv_noise=None, mask=None, use_weights=True):
    """Per-pixel CG weight: N^-1 if given, else mask * W (masked.py:77-93)."""
    if inv_noise is not None:
        w = np.asarray(inv_noise, dtype=np.float64)
    elif mask is not None:
        w = np.asarray(mask, dtype=np.float64) * pixel_weights(nside, use_weights)
    else:
        raise ValueError("provide either inv_noise (per-pixel N^-1) or mask")
    return w if spin == 0 else w[None, :]


def prior_sqrt(signal_cl, lmax, spin):
    """x-space whitening sqrt(Cl) per real DOF, exactly 0 on zero-power multipoles (masked.py:181-227)."""
    ms, ls = [], []
    for m in range(lmax + 1):
        ms.append(np.full(lmax + 1 - m, m))
        ls.append(np.arange(m, lmax + 1))
    ms, ls = np.concatenate(ms), np.concatenate(ls)
    act = ls >= abs(spin)
    ell = np.concatenate([ls[act & (ms == 0)], ls[act & (ms > 0)], ls[act & (ms > 0)]])

    def one(cl):
        c = np.asarray(cl, dtype=np.float64)[ell]
        return np.where(c > 0, np.sqrt(np.where(c > 0, c, 1.0)), 0.0)

    return one(signal_cl) if spin == 0 else np.concatenate([one(signal_cl[0]), one(signal_cl[1])])


def _whitened_system(maps, w, pw, nside, lmax, spin):
    b = pw * alm_to_real(adjoint_synthesis(w * np.asarray(maps), nside, lmax, spin), lmax, spin)

    def op(y):
        a = real_to_alm(pw * y, lmax, spin)
        return pw * alm_to_real(adjoint_synthesis(w * synthesis(a, nside, lmax, spin), nside, lmax, spin),
                                lmax, spin) + y

    return b, op


def wiener(maps, signal_cl, nside, lmax, spin=0, *, inv_noise=None, mask=None, max_iter=200, tol=1e-8,
           use_weights=True):
    """Wiener mean: CG on (P A_x P + I) y = P b_x, a = T^-1 P y (masked.py:320-372)."""
    w = weight_pix(nside, spin, inv_noise=inv_noise, mask=mask, use_weights=use_weights)
    pw = prior_sqrt(signal_cl, lmax, spin)
    b, op = _whitened_system(maps, w, pw, nside, lmax, spin)
    y, _ = cg(op, b, tol=tol, maxiter=max_iter)
    return real_to_alm(pw * y, lmax, spin)


def constrained_realization(maps, signal_cl, nside, lmax, omega, xi, spin=0, *, inv_noise=None, mask=None,
                            max_iter=200, tol=1e-8, use_weights=True):
    """Posterior draw for given sources omega (pixel space) and xi (x space) (masked.py:375-439)."""
    w = weight_pix(nside, spin, inv_noise=inv_noise, mask=mask, use_weights=use_weights)
    pw = prior_sqrt(signal_cl, lmax, spin)
    b, op = _whitened_system(maps, w, pw, nside, lmax, spin)
    s1 = alm_to_real(adjoint_synthesis(np.sqrt(w) * np.asarray(omega), nside, lmax, spin), lmax, spin)
    rhs = b + pw * s1 + np.where(pw > 0, np.asarray(xi), 0.0)
    y, _ = cg(op, rhs, tol=tol, maxiter=max_iter)
    return real_to_alm(pw * y, lmax, spin)


def bandpower(alm, lmax: int, spin: int = 0) -> np.ndarray:
    """C_l = (2l+1)^-1 sum_m (2 - delta_m0)|a_lm|^2 (diff.py:119-138)."""
    ells, _ = lm_of_index(lmax)
    w = metric_weight(lmax)

    def one(a):
        return np.bincount(ells, weights=w * np.abs(a) ** 2, minlength=lmax + 1) / (2 * np.arange(lmax + 1) + 1.0)

    a = np.asarray(alm)
    return one(a) if spin == 0 else np.stack([one(a[0]), one(a[1])])
