"""GPU parity of the layers above the transforms (needs a B200).

* ``analysis`` / ``bare_analysis`` vs the reference's own outputs (golden vectors);
* the real-DOF layer and the CG ``deconvolve`` vs the golden vectors and the oracle;
* torch gradients vs central finite differences (the reference checks its JAX
  gradients the same way, test_grad.py:175-191, at 1e-6).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from oracle import jht_oracle as O  # noqa: E402

TOL = 1e-12
FD_TOL = 1e-6


def _np(t):
    return t.detach().cpu().numpy()


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
def test_analysis_matches_golden(golden, tag, nside, lmax, spin, niter, use_w):
    out = jhtb.analysis(golden[f"{tag}/map"], nside, lmax, spin, niter=niter, use_weights=use_w)
    assert relerr(_np(out), golden[f"{tag}/alm"]) <= TOL
    assert relerr(_np(jhtb.map2alm(golden[f"{tag}/map"], nside, lmax, spin, niter, use_w)), golden[f"{tag}/alm"]) <= TOL
    if niter == 0:
        out0 = jhtb.bare_analysis(golden[f"{tag}/map"], nside, lmax, spin, use_weights=use_w)
        assert relerr(_np(out0), golden[f"{tag}/alm"]) <= TOL


@pytest.mark.parametrize("nside,lmax,spin,niter", [(64, 96, 0, 3), (64, 96, 2, 3), (128, 64, 2, 1)])
def test_analysis_matches_oracle(nside, lmax, spin, niter):
    rng = np.random.default_rng(nside + lmax + spin)
    npix = 12 * nside * nside
    m = rng.standard_normal(npix if spin == 0 else (2, npix))
    ref = O.analysis(m, nside, lmax, spin, niter=niter)
    assert relerr(_np(jhtb.analysis(m, nside, lmax, spin, niter=niter)), ref) <= TOL


def test_analysis_inverts_band_limited_maps():
    nside, lmax = 32, 40
    rng = np.random.default_rng(1)
    K = jhtb.alm_size(lmax)
    a = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / (np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)]) + 5.0)
    a[: lmax + 1] = a[: lmax + 1].real
    m = jhtb.synthesis(a, nside, lmax, 0)
    errs = [relerr(_np(jhtb.analysis(m, nside, lmax, 0, niter=n)), a) for n in (0, 1, 3, 6)]
    assert errs[-1] < errs[1] < errs[0]
    assert errs[-1] < 1e-12


def test_pseudo_alm_is_analysis_of_masked_map():
    nside, lmax = 16, 24
    rng = np.random.default_rng(4)
    m = rng.standard_normal((2, 12 * nside * nside))
    mask = (rng.uniform(size=12 * nside * nside) > 0.3).astype(np.float64)
    got = jhtb.pseudo_alm(m, mask, nside, lmax, 2)
    ref = O.analysis(mask[None, :] * m, nside, lmax, 2, niter=3)
    assert relerr(_np(got), ref) <= TOL


def test_real_dof_round_trip_on_gpu(golden):
    x0 = jhtb.alm_to_real(torch.as_tensor(golden["real/a0"], device="cuda"), 12, 0)
    np.testing.assert_array_equal(_np(x0), golden["real/x0"])
    x2 = jhtb.alm_to_real(torch.as_tensor(golden["real/a2"], device="cuda"), 12, 2)
    np.testing.assert_array_equal(_np(x2), golden["real/x2"])
    np.testing.assert_allclose(_np(jhtb.real_to_alm(x2, 12, 2)), golden["real/a2"], atol=1e-15)


def test_synthesis_real_and_analysis_real_match_oracle():
    nside, lmax = 16, 24
    rng = np.random.default_rng(9)
    for spin in (0, 2):
        x = rng.standard_normal(jhtb.n_dof(lmax, spin))
        ref = O.synthesis(O.real_to_alm(x, lmax, spin), nside, lmax, spin)
        got = jhtb.synthesis_real(torch.as_tensor(x, device="cuda"), nside, lmax, spin)
        assert relerr(_np(got), ref) <= TOL
        back = jhtb.analysis_real(got, nside, lmax, spin)
        assert relerr(_np(back), O.alm_to_real(O.analysis(ref, nside, lmax, spin), lmax, spin)) <= TOL


def _oracle_rel_residual(alm, maps, mask, nside, lmax, spin, reg):
    """||b - A x|| / ||b|| of the CG system, evaluated with the oracle's operators."""
    w = np.asarray(mask) * O.pixel_weights(nside)
    w = w if spin == 0 else w[None, :]
    b = O.alm_to_real(O.adjoint_synthesis(w * np.asarray(maps), nside, lmax, spin), lmax, spin)
    x = O.alm_to_real(np.asarray(alm), lmax, spin)
    Ax = O.alm_to_real(O.adjoint_synthesis(w * O.synthesis(O.real_to_alm(x, lmax, spin), nside, lmax, spin),
                                          nside, lmax, spin), lmax, spin) + reg * x
    return float(np.linalg.norm(b - Ax) / np.linalg.norm(b))


def test_deconvolve_matches_golden(golden):
    """Same system solved to the same stopping rule (|r| <= tol |b|).

    CG over ~130 iterations on this masked, weakly regularised system amplifies
    last-bit differences of the operator, so the solutions agree to the conditioning
    (1e-6 here) while both satisfy the residual bound of the reference's stopping rule.
    """
    out = _np(jhtb.deconvolve(golden["cg/data"], golden["cg/mask"], 8, 12, 0, tol=1e-8, reg=1e-6))
    assert relerr(out, golden["cg/alm"]) <= 1e-6
    assert _oracle_rel_residual(out, golden["cg/data"], golden["cg/mask"], 8, 12, 0, 1e-6) <= 2e-8


def test_deconvolve_batch_matches_per_column_and_oracle():
    nside, lmax, spin = 8, 12, 2
    rng = np.random.default_rng(21)
    npix = 12 * nside * nside
    mask = (rng.uniform(size=npix) > 0.2).astype(np.float64)
    maps = rng.standard_normal((3, 2, npix))
    maps[1] *= 1e3  # columns with very different scales converge independently
    batch, info = jhtb.deconvolve_batch(maps, mask, nside, lmax, spin, tol=1e-10, reg=1e-4, return_info=True)
    assert bool(torch.all(info["rel_residual"] <= 1e-10))
    for b in range(3):
        one = _np(jhtb.deconvolve(maps[b], mask, nside, lmax, spin, tol=1e-10, reg=1e-4))
        assert relerr(_np(batch[b]), one) <= 1e-8
        assert _oracle_rel_residual(_np(batch[b]), maps[b], mask, nside, lmax, spin, 1e-4) <= 2e-10
        ref = O.deconvolve(maps[b], mask, nside, lmax, spin, tol=1e-10, reg=1e-4)
        assert relerr(one, ref) <= 1e-8


def test_bandpower_on_gpu_matches_oracle():
    lmax = 30
    rng = np.random.default_rng(2)
    K = jhtb.alm_size(lmax)
    a = rng.standard_normal(K) + 1j * rng.standard_normal(K)
    got = jhtb.bandpower(torch.as_tensor(a, device="cuda"), lmax)
    assert relerr(_np(got), O.bandpower(a, lmax)) <= 1e-14


# ------------------------------------------------------------------------------------
# gradients vs central finite differences
# ------------------------------------------------------------------------------------
def _fd_check(f, x, ndir=6, h=1e-3, seed=0):
    """Compare autograd <grad f(x), u> with the central difference along random u."""
    xg = x.clone().requires_grad_(True)
    y = f(xg)
    (g,) = torch.autograd.grad(y, xg)
    gen = torch.Generator(device=x.device).manual_seed(seed)
    worst = 0.0
    with torch.no_grad():
        for _ in range(ndir):
            u = torch.randn(x.shape, dtype=x.dtype, device=x.device, generator=gen)
            fd = (f(x + h * u) - f(x - h * u)) / (2 * h)
            an = torch.sum(g * u) if not torch.is_complex(g) else torch.sum(torch.real(torch.conj(g) * u))
            worst = max(worst, abs(float(an - fd)) / max(abs(float(fd)), abs(float(an)), 1e-300))
    return worst


@pytest.mark.parametrize("spin", [0, 2])
def test_synthesis_real_gradient_matches_fd(spin):
    nside, lmax = 8, 12
    rng = np.random.default_rng(31 + spin)
    npix = 12 * nside * nside
    d = torch.as_tensor(rng.standard_normal(npix if spin == 0 else (2, npix)), device="cuda")
    x = torch.as_tensor(rng.standard_normal(jhtb.n_dof(lmax, spin)), device="cuda")

    def loss(v):
        return 0.5 * torch.sum((jhtb.synthesis_real(v, nside, lmax, spin) - d) ** 2)

    assert _fd_check(loss, x) <= FD_TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_analysis_real_gradient_matches_fd(spin):
    nside, lmax = 8, 12
    rng = np.random.default_rng(41 + spin)
    npix = 12 * nside * nside
    m = torch.as_tensor(rng.standard_normal(npix if spin == 0 else (2, npix)), device="cuda")
    w = torch.as_tensor(rng.standard_normal(jhtb.n_dof(lmax, spin)), device="cuda")

    def loss(v):
        x = jhtb.analysis_real(v, nside, lmax, spin, niter=2)
        return torch.sum(w * x) + 0.25 * torch.sum(x * x)

    assert _fd_check(loss, m) <= FD_TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_complex_alm_gradient_convention(spin):
    """torch's grad on complex a_lm is dL/dRe + i dL/dIm, including the m = 0 columns."""
    nside, lmax = 4, 6
    rng = np.random.default_rng(51 + spin)
    K = jhtb.alm_size(lmax)
    shape = (K,) if spin == 0 else (2, K)
    a = torch.as_tensor(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), device="cuda")
    g = torch.as_tensor(rng.standard_normal((12 * nside * nside,) if spin == 0 else (2, 12 * nside * nside)), device="cuda")

    def loss(v):
        return torch.sum(jhtb.synthesis(v, nside, lmax, spin) * g)

    ag = a.clone().requires_grad_(True)
    (grad,) = torch.autograd.grad(loss(ag), ag)
    h = 1e-3
    flat = a.reshape(-1)
    for k in range(flat.numel()):
        for unit, part in ((1.0, "re"), (1j, "im")):
            e = torch.zeros_like(flat)
            e[k] = unit * h
            fd = float((loss((flat + e).reshape(a.shape)) - loss((flat - e).reshape(a.shape))) / (2 * h))
            an = float(grad.reshape(-1)[k].real if part == "re" else grad.reshape(-1)[k].imag)
            assert abs(an - fd) <= FD_TOL * max(1.0, abs(fd)), (k, part, an, fd)


@pytest.mark.parametrize("spin", [0, 2])
def test_adjoint_gradient_matches_fd(spin):
    nside, lmax = 8, 12
    rng = np.random.default_rng(61 + spin)
    npix = 12 * nside * nside
    v = torch.as_tensor(rng.standard_normal(npix if spin == 0 else (2, npix)), device="cuda")
    K = jhtb.alm_size(lmax)
    c = torch.as_tensor(rng.standard_normal((K,) if spin == 0 else (2, K)) + 1j * rng.standard_normal((K,) if spin == 0 else (2, K)), device="cuda")

    def loss(t):
        b = jhtb.adjoint_synthesis(t, nside, lmax, spin)
        return torch.sum(torch.real(c * b)) + 0.5 * torch.sum(torch.abs(b) ** 2)

    assert _fd_check(loss, v) <= FD_TOL


# ------------------------------------------------------------------------------------
# Wiener filter and constrained realization (masked.py:320-439)
# ------------------------------------------------------------------------------------
@pytest.mark.parametrize("spin", [0, 2])
def test_wiener_matches_golden(golden, spin):
    """Spin 0 (mask weighting) converges well inside the iteration cap; spin 2 (stiff noise) does not."""
    if spin == 0:
        out = _np(jhtb.wiener(golden["wiener/s0_data"], golden["wiener/s0_cl"], 8, 12, 0,
                              mask=golden["wiener/s0_mask"], tol=1e-10))
        ref = golden["wiener/s0_alm"]
        assert np.all(out[:2] == 0)  # zero-power monopole and dipole pinned exactly
        assert relerr(out, ref) <= 1e-9
    else:
        # this noise level makes the whitened system stiff: both solvers stop at the
        # 200-iteration cap, where last-bit differences of the operator show at ~3e-8;
        # the two solutions must be equally converged on the oracle's operator
        cl = golden["wiener/s2_cl"]
        out = _np(jhtb.wiener(golden["wiener/s2_data"], (cl[0], cl[1]), 8, 12, 2,
                              inv_noise=golden["wiener/s2_invn"], tol=1e-10))
        ref = golden["wiener/s2_alm"]
        assert relerr(out, ref) <= 1e-6
        w = O.weight_pix(8, 2, inv_noise=golden["wiener/s2_invn"])
        pw = O.prior_sqrt((cl[0], cl[1]), 12, 2)
        b, op = O._whitened_system(golden["wiener/s2_data"], w, pw, 8, 12, 2)

        def resid(a):
            x = O.alm_to_real(a, 12, 2)
            y = np.where(pw > 0, x / np.where(pw > 0, pw, 1.0), 0.0)
            return np.linalg.norm(b - op(y)) / np.linalg.norm(b)

        assert resid(out) <= 2.0 * resid(ref)


def test_wiener_batch_matches_single():
    nside, lmax, spin = 16, 24, 2
    rng = np.random.default_rng(8)
    npix = 12 * nside * nside
    ell = np.arange(lmax + 1)
    cl = (1.0 / (ell + 10.0) ** 2, 0.1 / (ell + 10.0) ** 2)
    inv_noise = rng.uniform(0.5, 2.0, npix) * (rng.uniform(size=npix) > 0.1)
    maps = rng.standard_normal((3, 2, npix)) * 1e-2
    batch = _np(jhtb.wiener_batch(maps, cl, nside, lmax, spin, inv_noise=inv_noise, tol=1e-11))
    for b in range(3):
        one = _np(jhtb.wiener(maps[b], cl, nside, lmax, spin, inv_noise=inv_noise, tol=1e-11))
        assert relerr(batch[b], one) <= 1e-10
        ref = O.wiener(maps[b], cl, nside, lmax, spin, inv_noise=inv_noise, tol=1e-11)
        assert relerr(one, ref) <= 1e-9


@pytest.mark.parametrize("spin", [0, 2])
def test_constrained_realization_matches_oracle_with_the_same_sources(spin):
    nside, lmax = 8, 12
    rng = np.random.default_rng(30 + spin)
    npix = 12 * nside * nside
    ell = np.arange(lmax + 1)
    cl0 = 1.0 / (ell + 10.0) ** 2
    cl0[:2] = 0.0
    cl = cl0 if spin == 0 else (cl0, 0.1 * cl0)
    inv_noise = rng.uniform(10.0, 100.0, npix) * (rng.uniform(size=npix) > 0.2)
    ncomp = 1 if spin == 0 else 2
    maps = rng.standard_normal((ncomp, npix)).reshape((npix,) if spin == 0 else (2, npix)) * 1e-2
    draw = _np(jhtb.constrained_realization(maps, cl, nside, lmax, 1234, spin, inv_noise=inv_noise, tol=1e-11))
    # the same sources, drawn the documented way: omega (pixels) then xi (real DOF)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    omega = torch.randn((1, ncomp, npix), dtype=torch.float64, device="cuda", generator=gen)
    xi = torch.randn((1, jhtb.n_dof(lmax, spin)), dtype=torch.float64, device="cuda", generator=gen)
    om = _np(omega)[0] if spin else _np(omega)[0, 0]
    ref = O.constrained_realization(maps, cl, nside, lmax, om, _np(xi)[0], spin, inv_noise=inv_noise, tol=1e-11)
    assert relerr(draw, ref) <= 1e-9
    ells = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    assert np.all(draw[..., ells < 2] == 0)  # pinned modes are exactly zero in every draw
    mean = _np(jhtb.wiener(maps, cl, nside, lmax, spin, inv_noise=inv_noise, tol=1e-11))
    assert relerr(draw, mean) > 1e-3  # a draw, not the mean



@pytest.mark.slow
@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_masked_cg_16_rhs_at_nside512_converges(precision):
    """Batched masked CG at nside 512, lmax 1024: a |cos theta| < 0.34 cut plus 200 seeded
    1-degree discs, data S a + white noise (sigma 1e-2), 16 right-hand sides to relative
    residual 1e-8 with eps = 1e-6 of the largest diagonal entry of T S^T (M W) S T^-1.
    Every column reaches the tolerance and the returned a_lm satisfies the FP64 system.
    ``bf16x3``: CG on the tensor-core operator with the FP64 residual replacing the recursive one."""
    import time

    from jht_b200 import masked as MK

    nside, lmax, spin, B = 512, 1024, 0, 16
    npix = 12 * nside * nside
    rng = np.random.default_rng(16)
    geo = jhtb.healpix.RingInfo(nside)
    z = np.repeat(geo.z, geo.npix_ring)
    phi = np.concatenate([geo.phi0[r] + 2 * np.pi * np.arange(n) / n for r, n in enumerate(geo.npix_ring)])
    st = np.sqrt(1 - z * z)
    mask = (np.abs(z) >= 0.34).astype(np.float64)
    cz = rng.uniform(-1, 1, 200)
    cp = rng.uniform(0, 2 * np.pi, 200)
    cs = np.sqrt(1 - cz * cz)
    cos_r = np.cos(np.radians(1.0))
    for k in range(200):
        mask[z * cz[k] + st * cs[k] * np.cos(phi - cp[k]) > cos_r] = 0.0
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)
    cl = 1.0 / (ell + 10.0) ** 2
    a = np.sqrt(cl / 2) * (rng.standard_normal((B, K)) + 1j * rng.standard_normal((B, K)))
    a[:, : lmax + 1] = np.sqrt(cl[: lmax + 1]) * rng.standard_normal((B, lmax + 1))
    gen = torch.Generator("cuda").manual_seed(16)
    maps = jhtb.synthesis_batch(a, nside, lmax, spin)
    maps = maps + 1e-2 * torch.randn(maps.shape, dtype=torch.float64, device="cuda", generator=gen)
    w = MK._weight_pix(nside, npix, maps.device, mask=mask)
    # diagonal entries on 16 m = 0 columns: m = 0 functions keep the most weight near the
    # poles, outside the |cos theta| < 0.34 cut, so the largest of them bounds the diagonal
    probe = torch.zeros((16, MK.n_dof(lmax, spin)), dtype=torch.float64, device="cuda")
    cols = torch.as_tensor(np.linspace(0, lmax, 16).astype(np.int64), device="cuda")
    probe[torch.arange(16, device="cuda"), cols] = 1.0
    diag = MK._normal(probe, w, nside, lmax, spin, "fp64")[torch.arange(16, device="cuda"), cols]
    eps = 1e-6 * float(diag.max())
    assert 0.5 < float(diag.max()) <= 1.0 + 1e-6
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sol, info = jhtb.deconvolve_batch(maps, mask, nside, lmax, spin, tol=1e-8, reg=eps, max_iter=6000,
                                      return_info=True, precision=precision)
    torch.cuda.synchronize()
    print(f"masked CG {precision}: {time.perf_counter() - t0:.1f} s, {info['iterations']} iterations, "
          f"{info.get('outer', 0)} FP64 residuals")
    assert bool(torch.all(info["rel_residual"] <= 1e-8)), (info["iterations"], info["rel_residual"])
    x = MK._real_batch(sol.reshape(B, 1, K), lmax, spin)
    b = MK._real_batch(jhtb.healpix._adjoint_raw(w * maps.reshape(B, 1, npix), nside, lmax, spin, "fp64"), lmax, spin)
    Ax = MK._normal(x, w, nside, lmax, spin, "fp64") + eps * x
    rel = torch.linalg.norm(b - Ax, dim=1) / torch.linalg.norm(b, dim=1)
    assert float(rel.max()) <= 1e-7, float(rel.max())


@pytest.mark.slow
@pytest.mark.parametrize("sigma", [0.0, 1e-3])
def test_mixed_analysis_matches_fp64_at_nside1024(sigma):
    """Spin-0 analysis(niter=3) at nside 1024, lmax 2048 of a seeded synthesis (+ white
    noise): the tensor-core A0 applications with FP64 residuals stay within 1e-10 of the
    FP64 analysis (relative to the largest a_lm)."""
    nside, lmax = 1024, 2048
    rng = np.random.default_rng(11)
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)
    cl = 1.0 / (ell + 10.0) ** 2
    a = np.sqrt(cl / 2) * (rng.standard_normal(K) + 1j * rng.standard_normal(K))
    a[: lmax + 1] = np.sqrt(cl[: lmax + 1]) * rng.standard_normal(lmax + 1)
    m = jhtb.synthesis(a, nside, lmax, 0)
    if sigma:
        gen = torch.Generator("cuda").manual_seed(12)
        m = m + sigma * torch.randn(m.shape, dtype=torch.float64, device="cuda", generator=gen)
    ref = jhtb.analysis(m, nside, lmax, 0, niter=3)
    got = jhtb.analysis(m, nside, lmax, 0, niter=3, precision="bf16x3")
    err = float(torch.max(torch.abs(got - ref)) / torch.max(torch.abs(ref)))
    print(f"mixed analysis nside 1024 lmax 2048 sigma {sigma}: {err:.3e} vs FP64")
    assert err <= 1e-10, err


@pytest.mark.slow
@pytest.mark.parametrize("variant", ["clean", "noise"])
@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_analysis_matches_jht_at_nside1024(variant, precision):
    """Spin-0 analysis(niter=3, pixel weights) at nside 1024, lmax 2048 against jht's own
    output on the same map (tests/golden/make_analysis_golden.py: the FP64 oracle synthesis
    of seeded a_lm, plus seeded white noise of sigma 1e-3 for ``noise``), at the stored
    sample of 18398 a_lm (random entries, the m = 0 column, the l = m diagonal, the
    l = lmax row); relative to the largest stored |a_lm|."""
    import sys
    from pathlib import Path

    here = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(here))
    import make_analysis_golden as G

    gold = np.load(here / f"jht_golden_analysis_{variant}.npz")
    nside, lmax, niter = (int(v) for v in gold["meta"])
    m = torch.as_tensor(G.input_map(variant), device="cuda")
    got = jhtb.analysis(m, nside, lmax, 0, niter=niter, precision=precision).cpu().numpy()
    ref = gold["alm"]
    err = float(np.max(np.abs(got[gold["idx"]] - ref)) / np.max(np.abs(ref)))
    print(f"analysis nside {nside} lmax {lmax} {variant} {precision}: {err:.3e} vs jht")
    assert err <= 1e-10, err
