"""Pin the CPU oracle before trusting it (CPU only).

* golden vectors from running the reference's own code (tests/golden/make_golden.py);
* closed-form Y_lm for l <= 2 and scipy's sph_harm_y to l = 512 (test_recursion.py:85-120);
* explicit Wigner-d sum for spin 2 (test_recursion.py:161-191);
* a 40-digit mpmath evaluation of the same recursion (scripts/exploratory/highL_mpmath_ref.py);
* the N/S-folded fused scans against the per-m / per-ring eager forms (test_vectorized.py);
* the inner-product identity and weight moments (test_grad.py:105-128, test_weights.py:26-67).
"""

from __future__ import annotations

import numpy as np
import pytest
from numpy.polynomial.legendre import legvander
from scipy.special import gammaln, sph_harm_y

from conftest import TRANSFORM_TAGS, parse_tag, relerr
from oracle import jht_oracle as O


# ------------------------------------------------------------------------------------
# golden vectors (reference's own outputs)
# ------------------------------------------------------------------------------------
@pytest.mark.parametrize("tag", TRANSFORM_TAGS)
def test_oracle_transforms_match_golden(golden, tag):
    spin, nside, lmax = parse_tag(tag)
    a, v = golden[f"{tag}/alm"], golden[f"{tag}/v"]
    assert relerr(O.synthesis(a, nside, lmax, spin, use_c=False), golden[f"{tag}/map"]) <= 1e-14
    assert relerr(O.adjoint_synthesis(v, nside, lmax, spin, use_c=False), golden[f"{tag}/adj"]) <= 1e-14


@pytest.mark.parametrize("tag", TRANSFORM_TAGS)
def test_c_oracle_matches_golden(golden, tag):
    spin, nside, lmax = parse_tag(tag)
    a, v = golden[f"{tag}/alm"], golden[f"{tag}/v"]
    assert relerr(O.synthesis(a, nside, lmax, spin, use_c=True), golden[f"{tag}/map"]) <= 1e-12
    assert relerr(O.adjoint_synthesis(v, nside, lmax, spin, use_c=True), golden[f"{tag}/adj"]) <= 1e-12


@pytest.mark.parametrize("tag", ["s0_n8_l12", "s0_n16_l24", "s2_n8_l12", "s2_n16_l24", "s0_n4_l16"])
def test_eager_forms_match_golden(golden, tag):
    spin, nside, lmax = parse_tag(tag)
    assert relerr(O.synthesis_eager(golden[f"{tag}/alm"], nside, lmax, spin), golden[f"{tag}/map"]) <= 1e-12
    assert relerr(O.adjoint_eager(golden[f"{tag}/v"], nside, lmax, spin), golden[f"{tag}/adj"]) <= 1e-12


def test_complex_m0_is_projected_like_reference(golden):
    a = golden["s0_n8_l12_cplx0/alm"]
    assert relerr(O.synthesis(a, 8, 12, 0, use_c=False), golden["s0_n8_l12_cplx0/map"]) <= 1e-14


@pytest.mark.parametrize(
    "tag,nside,lmax,spin,niter,use_w",
    [
        ("ana_s0_n16_l24", 16, 24, 0, 3, True),
        ("ana_s2_n16_l24", 16, 24, 2, 3, True),
        ("ana_s0_n8_l12_bare", 8, 12, 0, 0, False),
        ("ana_s0_n16_l32_noise", 16, 32, 0, 3, True),
        ("ana_s2_n8_l16_it2", 8, 16, 2, 2, True),
    ],
)
def test_oracle_analysis_matches_golden(golden, tag, nside, lmax, spin, niter, use_w):
    out = O.analysis(golden[f"{tag}/map"], nside, lmax, spin, niter=niter, use_weights=use_w, use_c=False)
    assert relerr(out, golden[f"{tag}/alm"]) <= 1e-13


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 12, 16, 32, 64])
def test_oracle_ring_weights_match_golden(golden, nside):
    np.testing.assert_allclose(O.ring_weights(nside), golden[f"weights/ring_n{nside}"], rtol=0, atol=1e-14)


def test_oracle_pixel_weights_match_golden(golden):
    np.testing.assert_allclose(O.pixel_weights(8, True), golden["weights/pix_n8"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("m", [0, 1, 5, 31, 64])
def test_lambda_columns_match_golden(golden, m):
    x = golden["lambda/x"]
    np.testing.assert_allclose(O.lambda_column(x, m, 64), golden[f"lambda/s0_m{m}"], rtol=0, atol=1e-14)
    for s in (2, -2):
        np.testing.assert_allclose(
            O.spin_lambda_column(x, m, s, 64), golden[f"lambda/s{s}_m{m}"], rtol=0, atol=1e-14
        )


def test_real_dof_matches_golden(golden):
    np.testing.assert_array_equal(O.alm_to_real(golden["real/a0"], 12, 0), golden["real/x0"])
    np.testing.assert_array_equal(O.alm_to_real(golden["real/a2"], 12, 2), golden["real/x2"])
    np.testing.assert_allclose(O.real_to_alm(golden["real/x0"], 12, 0), golden["real/a0"], atol=1e-15)
    np.testing.assert_allclose(O.real_to_alm(golden["real/x2"], 12, 2), golden["real/a2"], atol=1e-15)
    assert O.n_dof(12, 0) == golden["real/x0"].size
    assert O.n_dof(12, 2) == golden["real/x2"].size


def test_cg_deconvolve_matches_golden(golden):
    out = O.deconvolve(golden["cg/data"], golden["cg/mask"], 8, 12, 0, tol=1e-8, reg=1e-6)
    assert relerr(out, golden["cg/alm"]) <= 1e-9


# ------------------------------------------------------------------------------------
# independent known-answer tests (analytic, scipy, Wigner sum, mpmath)
# ------------------------------------------------------------------------------------
def _analytic(theta):
    c, s = np.cos(theta), np.sin(theta)
    return {
        (0, 0): np.full_like(theta, np.sqrt(1 / (4 * np.pi))),
        (1, 0): np.sqrt(3 / (4 * np.pi)) * c,
        (1, 1): -np.sqrt(3 / (8 * np.pi)) * s,
        (2, 0): np.sqrt(5 / (16 * np.pi)) * (3 * c * c - 1),
        (2, 1): -np.sqrt(15 / (8 * np.pi)) * s * c,
        (2, 2): np.sqrt(15 / (32 * np.pi)) * s * s,
    }


def test_lambda_matches_closed_form_low_l():
    theta = np.linspace(0.05, np.pi - 0.05, 13)
    ana = _analytic(theta)
    for m in (0, 1, 2):
        lam = O.lambda_column(np.cos(theta), m, 2)
        for ell in range(m, 3):
            np.testing.assert_allclose(lam[ell - m], ana[(ell, m)], rtol=0, atol=1e-13)


@pytest.mark.parametrize("m", [0, 1, 2, 5, 10, 50, 100])
def test_lambda_matches_scipy_to_512(m):
    lmax = 512
    theta = np.linspace(0.03, np.pi - 0.03, 23)
    lam = O.lambda_column(np.cos(theta), m, lmax)
    worst = 0.0
    for ell in range(m, lmax + 1):
        ref = np.real(sph_harm_y(ell, m, theta, 0.0))
        worst = max(worst, np.max(np.abs(lam[ell - m] - ref)) / max(np.max(np.abs(ref)), 1.0))
    assert worst <= 1e-12


def _wigner_explicit(ell, M, Mp, beta):
    c, s = np.cos(beta / 2), np.sin(beta / 2)
    kmin, kmax = max(0, M - Mp), min(ell + M, ell - Mp)
    pref = 0.5 * (gammaln(ell + M + 1) + gammaln(ell - M + 1) + gammaln(ell + Mp + 1) + gammaln(ell - Mp + 1))
    tot = np.zeros_like(beta)
    for k in range(kmin, kmax + 1):
        lc = pref - (gammaln(k + 1) + gammaln(ell + M - k + 1) + gammaln(ell - Mp - k + 1) + gammaln(k - M + Mp + 1))
        tot += (-1) ** k * np.exp(lc) * c ** (2 * ell - 2 * k + M - Mp) * s ** (2 * k - M + Mp)
    return tot


@pytest.mark.parametrize("m", [0, 1, 2, 5, 10])
@pytest.mark.parametrize("spin", [2, -2])
def test_wigner_matches_explicit_sum(m, spin):
    theta = np.linspace(0.1, np.pi - 0.1, 15)
    lmin = max(m, 2)
    d = O.wigner_column(np.cos(theta), -m, spin, 12)
    for ell in range(lmin, 13):
        np.testing.assert_allclose(d[ell - lmin], _wigner_explicit(ell, -m, spin, theta), rtol=0, atol=1e-11)


@pytest.mark.parametrize("m,spin", [(0, 0), (7, 0), (300, 0), (3, 2), (250, 2)])
def test_recursion_matches_mpmath(m, spin):
    """40-digit three-term recursion (no renormalisation needed at arbitrary exponent)."""
    mpmath = pytest.importorskip("mpmath")
    mp = mpmath.mp
    mp.dps = 40
    lmax = 700
    thetas = [0.2, 1.1, 2.5]
    ours = (
        O.lambda_column(np.cos(thetas), m, lmax)
        if spin == 0
        else O.spin_lambda_column(np.cos(thetas), m, spin, lmax)
    )
    for j, th in enumerate(thetas):
        th = mp.mpf(th)
        x = mp.cos(th)
        if spin == 0:
            c = -mp.mpf(0.5) * mp.log(4 * mp.pi)
            for k in range(1, m + 1):
                c += mp.mpf(0.5) * mp.log(mp.mpf(2 * k + 1) / (2 * k))
            cur = (-1) ** m * mp.e**c * mp.sin(th) ** m
            prev = mp.mpf(0)
            vals = [cur]
            for ell in range(m + 1, lmax + 1):
                L = mp.mpf(ell)
                a = mp.sqrt((2 * L - 1) * (2 * L + 1) / ((L - m) * (L + m)))
                b = mp.sqrt((2 * L + 1) * ((L - 1) ** 2 - m * m) / ((2 * L - 3) * (L - m) * (L + m)))
                prev, cur = cur, a * x * cur - b * prev
                vals.append(cur)
            lmin = m
        else:
            M, Mp = -m, spin
            lmin = max(abs(M), abs(Mp))
            k0 = max(0, M - Mp)
            lf = mp.mpf(0.5) * (mp.loggamma(lmin + M + 1) + mp.loggamma(lmin - M + 1) + mp.loggamma(lmin + Mp + 1)
                                + mp.loggamma(lmin - Mp + 1)) - (mp.loggamma(k0 + 1) + mp.loggamma(lmin + M - k0 + 1)
                                + mp.loggamma(lmin - Mp - k0 + 1) + mp.loggamma(k0 - M + Mp + 1))
            cur = (-1) ** k0 * mp.e**lf * mp.cos(th / 2) ** (2 * lmin - 2 * k0 + M - Mp) * mp.sin(th / 2) ** (2 * k0 - M + Mp)
            prev = mp.mpf(0)
            ds = [cur]
            for ell in range(lmin, lmax):
                L = mp.mpf(ell)
                D = L * mp.sqrt(((L + 1) ** 2 - M * M) * ((L + 1) ** 2 - Mp * Mp))
                A = (2 * L + 1) * L * (L + 1) / D
                C = -(2 * L + 1) * M * Mp / D
                B = (L + 1) * mp.sqrt((L * L - M * M) * (L * L - Mp * Mp)) / D
                prev, cur = cur, (A * x + C) * cur - B * prev
                ds.append(cur)
            vals = [(-1) ** m * mp.sqrt((2 * (lmin + i) + 1) / (4 * mp.pi)) * d for i, d in enumerate(ds)]
        ref = np.array([float(v) for v in vals])
        amp = np.sqrt((2 * np.arange(lmin, lmax + 1) + 1) / (4 * np.pi))
        assert np.max(np.abs(ours[:, j] - ref) / amp) <= 1e-13


def test_lambda_bounded_and_finite_near_poles():
    x = np.array([1.0, 1.0 - 1e-12, np.cos(1e-6), -1.0])
    for m in (0, 1, 2, 64, 1000):
        assert np.all(np.isfinite(O.lambda_column(x, m, 1000)))
    assert O.lambda_column(np.array([1.0]), 5, 5)[0, 0] == 0.0
    theta = np.linspace(0.01, np.pi - 0.01, 29)
    lam = O.lambda_column(np.cos(theta), 17, 1000)
    ell = np.arange(17, 1001)[:, None]
    assert np.all(np.abs(lam) <= np.sqrt((2 * ell + 1) / (4 * np.pi)) * (1 + 1e-9))


# ------------------------------------------------------------------------------------
# structural identities
# ------------------------------------------------------------------------------------
@pytest.mark.parametrize("spin", [0, 2])
def test_oracle_inner_product_identity(spin):
    nside, lmax = 16, 24
    rng = np.random.default_rng(5 + spin)
    K = O.alm_size(lmax)
    npix = 12 * nside**2
    shape = (K,) if spin == 0 else (2, K)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    if spin == 2:
        ells, _ = O.lm_of_index(lmax)
        a[:, ells < 2] = 0
    v = rng.standard_normal(npix if spin == 0 else (2, npix))
    lhs = np.sum(O.synthesis(a, nside, lmax, spin) * v)
    b = O.adjoint_synthesis(v, nside, lmax, spin)
    rhs = np.sum(O.metric_weight(lmax) * np.real(np.conj(a) * b))
    assert abs(lhs - rhs) / abs(lhs) <= 1e-12


@pytest.mark.parametrize("nside", [2, 4, 8, 16, 32, 64])
def test_weight_moments(nside):
    geo = O.Rings(nside)
    ring_w = np.add.reduceat(O.pixel_weights(nside), geo.start)
    q = ring_w @ legvander(geo.z, 2 * nside)
    assert abs(q[0] - 4 * np.pi) < 1e-9 * 4 * np.pi
    assert np.max(np.abs(q[np.arange(2, 2 * nside + 1, 2)])) < 1e-9 * 4 * np.pi
    assert abs(O.pixel_weights(nside).sum() - 4 * np.pi) < 1e-11


def test_bandpower_formula():
    rng = np.random.default_rng(9)
    lmax = 10
    a = rng.standard_normal(O.alm_size(lmax)) + 1j * rng.standard_normal(O.alm_size(lmax))
    cl = O.bandpower(a, lmax)
    for ell in range(lmax + 1):
        tot = abs(a[O.alm_base(0, lmax) + ell]) ** 2
        for m in range(1, ell + 1):
            tot += 2 * abs(a[O.alm_base(m, lmax) + ell - m]) ** 2
        assert abs(cl[ell] - tot / (2 * ell + 1)) <= 1e-14 * max(tot, 1)


@pytest.mark.parametrize("spin", [0, 2])
def test_oracle_wiener_matches_golden(golden, spin):
    if spin == 0:
        out = O.wiener(golden["wiener/s0_data"], golden["wiener/s0_cl"], 8, 12, 0, mask=golden["wiener/s0_mask"], tol=1e-10)
        ref = golden["wiener/s0_alm"]
        assert np.all(out[:2] == 0)  # zero-power multipoles are pinned exactly
    else:
        cl = golden["wiener/s2_cl"]
        out = O.wiener(golden["wiener/s2_data"], (cl[0], cl[1]), 8, 12, 2, inv_noise=golden["wiener/s2_invn"], tol=1e-10)
        ref = golden["wiener/s2_alm"]
    assert relerr(out, ref) <= 1e-12


@pytest.mark.parametrize("spin", [0, 2])
def test_oracle_cg_matches_dense_solve(spin):
    """jht tests/test_masked.py's dense-operator gate: the CG solution of the masked normal
    equations equals the dense solve of the same system (real-DOF matrix assembled column by
    column from the oracle's S and S^T)."""
    nside, lmax, reg = 4, 6, 1e-6
    rng = np.random.default_rng(20 + spin)
    geo = O.Rings(nside)
    zpix = np.repeat(geo.z, geo.nring)
    mask = (np.abs(zpix) >= 0.3).astype(np.float64)
    w = mask * O.pixel_weights(nside)
    w = w if spin == 0 else w[None, :]
    n = O.n_dof(lmax, spin)

    def normal(x):
        a = O.real_to_alm(x, lmax, spin)
        return O.alm_to_real(O.adjoint_synthesis(w * O.synthesis(a, nside, lmax, spin), nside, lmax, spin), lmax, spin)

    A = np.stack([normal(e) for e in np.eye(n)], axis=1) + reg * np.eye(n)
    assert np.allclose(A, A.T, atol=1e-12)  # the normal operator is symmetric
    npix = 12 * nside * nside
    maps = rng.standard_normal(npix) if spin == 0 else rng.standard_normal((2, npix))
    b = O.alm_to_real(O.adjoint_synthesis(w * maps, nside, lmax, spin), lmax, spin)
    x_dense = np.linalg.solve(A, b)
    x_cg = O.alm_to_real(O.deconvolve(maps, mask, nside, lmax, spin, tol=1e-12, reg=reg, max_iter=5000), lmax, spin)
    assert np.max(np.abs(x_cg - x_dense)) <= 1e-6 * np.max(np.abs(x_dense))
    assert np.linalg.norm(A @ x_cg - b) <= 1e-10 * np.linalg.norm(b)


# ------------------------------------------------------------------------------------
# the extended-precision arbiter (oracle/legendre_ref.c in long double) against a
# 30-digit mpmath evaluation of the same sums: it must be far below FP64 rounding
# ------------------------------------------------------------------------------------
def _mp_column_sum(spin, m, lmax, x, coef):
    """sum_l coef[l - lmin] lambda^{s}_lm(x) (spin 0), or the +2 / -2 sums (spin 2), in mpmath."""
    import mpmath as mp

    mp.mp.dps = 30
    xm = mp.mpf(x)
    th = mp.acos(xm)
    if spin == 0:
        c = -mp.mpf(0.5) * mp.log(4 * mp.pi)
        for k in range(1, m + 1):
            c += mp.mpf(0.5) * mp.log(mp.mpf(2 * k + 1) / (2 * k))
        cur, prev = (-1) ** m * mp.e**c * mp.sin(th) ** m, mp.mpf(0)
        tot = mp.mpc(coef[0]) * cur
        for ell in range(m + 1, lmax + 1):
            L = mp.mpf(ell)
            a = mp.sqrt((2 * L - 1) * (2 * L + 1) / ((L - m) * (L + m)))
            b = mp.sqrt((2 * L + 1) * ((L - 1) ** 2 - m * m) / ((2 * L - 3) * (L - m) * (L + m)))
            prev, cur = cur, a * xm * cur - b * prev
            tot += mp.mpc(coef[ell - m]) * cur
        return [tot]
    out = []
    lmin = max(m, 2)
    for Mp in (2, -2):
        M = -m
        k0 = max(0, M - Mp)
        lf = mp.mpf(0.5) * (mp.loggamma(lmin + M + 1) + mp.loggamma(lmin - M + 1) + mp.loggamma(lmin + Mp + 1)
                            + mp.loggamma(lmin - Mp + 1)) - (mp.loggamma(k0 + 1) + mp.loggamma(lmin + M - k0 + 1)
                                                             + mp.loggamma(lmin - Mp - k0 + 1) + mp.loggamma(k0 - M + Mp + 1))
        cur = (-1) ** k0 * mp.e**lf * mp.cos(th / 2) ** (2 * lmin - 2 * k0 + M - Mp) * mp.sin(th / 2) ** (2 * k0 - M + Mp)
        prev = mp.mpf(0)
        tot = mp.mpc(coef[0]) * (-1) ** m * mp.sqrt((2 * lmin + 1) / (4 * mp.pi)) * cur
        for ell in range(lmin, lmax):
            L = mp.mpf(ell)
            D = L * mp.sqrt(((L + 1) ** 2 - M * M) * ((L + 1) ** 2 - Mp * Mp))
            A, C = (2 * L + 1) * L * (L + 1) / D, -(2 * L + 1) * M * Mp / D
            B = (L + 1) * mp.sqrt((L * L - M * M) * (L * L - Mp * Mp)) / D
            prev, cur = cur, (A * xm + C) * cur - B * prev
            tot += mp.mpc(coef[ell + 1 - lmin]) * (-1) ** m * mp.sqrt((2 * (ell + 1) + 1) / (4 * mp.pi)) * cur
        out.append(tot)
    return out


@pytest.mark.parametrize("spin", [0, 2])
def test_extended_arbiter_matches_mpmath(spin):
    from oracle import _cref

    ref = _cref.load()
    lmax = 1500
    geo = O.Rings(1024)
    x = geo.z[[0, 3, 700]]  # next to the pole, a polar cap ring, the belt
    rng = np.random.default_rng(31)
    K = O.alm_size(lmax)
    for m in (0, 3, 700):
        a = np.zeros((2, K), np.complex128)
        n = lmax + 1 - m
        b = O.alm_base(m, lmax)
        a[:, b : b + n] = (rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))) / (np.arange(m, lmax + 1) + 10)
        if spin == 2:
            a[:, b : b + max(0, 2 - m)] = 0
            cp = -(a[0] + 1j * a[1])
            lmin = max(m, 2)
            coef = cp[b + lmin - m : b + n]
            arb = ref.synth(2, lmax, x, a, m, m + 1, extended=True)[0][m]  # FpN: +2 channel
            f64 = ref.synth(2, lmax, x, a, m, m + 1)[0][m]
            exact = np.array([complex(_mp_column_sum(2, m, lmax, xx, coef)[0]) for xx in x])
        else:
            arb = ref.synth(0, lmax, x, a[:1], m, m + 1, extended=True)[0][m]
            f64 = ref.synth(0, lmax, x, a[:1], m, m + 1)[0][m]
            exact = np.array([complex(_mp_column_sum(0, m, lmax, xx, a[0, b : b + n])[0]) for xx in x])
        scale = np.max(np.abs(exact))
        # 80-bit evaluation: its rounding (mostly the running log-scale of the renormalised
        # form) stays a thousand times below the FP64 differences it has to decide
        e_arb, e_f64 = np.max(np.abs(arb - exact)) / scale, np.max(np.abs(f64 - exact)) / scale
        print(f"spin {spin} m {m}: arbiter {e_arb:.2e}, FP64 oracle {e_f64:.2e}")
        assert e_arb <= 5e-15, (m, e_arb)
        assert e_f64 <= 1e-11
