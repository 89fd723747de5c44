"""Generate the golden fixtures by running the reference jht code itself.

jht is pure Python over JAX; JAX is absent here, so ``jaxshim`` maps the JAX
calls jht makes onto NumPy and the reference source runs unchanged.  Every
fixture below is therefore the output of jht's own ``synthesis``,
``adjoint_synthesis``, ``analysis``, ``ring_weights``, ... (src/jht/healpix.py,
_analysis.py, weights.py, masked.py, _recursion.py) on seeded inputs.

Usage (needs the reference checkout; writes ``tests/golden/*.npz``)::

    python tests/golden/make_golden.py /path/to/jht/checkout

The fixtures are committed so the tests never need the reference at run time.
"""

from __future__ import annotations

import sys
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import jaxshim  # noqa: E402


def alm_size(lmax: int) -> int:
    return (lmax + 1) * (lmax + 2) // 2


def ell_of_index(lmax: int) -> np.ndarray:
    return np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])


def random_alm(rng, lmax: int, lmin: int = 0) -> np.ndarray:
    """Unit-variance complex alm, real m=0 column, l < lmin zeroed."""
    K = alm_size(lmax)
    a = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / np.sqrt(2.0)
    a[: lmax + 1] = a[: lmax + 1].real
    a[ell_of_index(lmax) < lmin] = 0.0
    return a.astype(np.complex128)


def spectrum_alm(rng, lmax: int, amp: float = 1.0, lmin: int = 0) -> np.ndarray:
    """alm with C_l = amp/(l+10)^2: a_l0 = sqrt(C) g, a_lm = sqrt(C/2)(g1 + i g2)."""
    ell = ell_of_index(lmax)
    cl = amp / (ell + 10.0) ** 2
    K = alm_size(lmax)
    g1 = rng.standard_normal(K)
    g2 = rng.standard_normal(K)
    a = np.sqrt(cl / 2.0) * (g1 + 1j * g2)
    a[: lmax + 1] = np.sqrt(cl[: lmax + 1]) * g1[: lmax + 1]
    a[ell < lmin] = 0.0
    return a.astype(np.complex128)


def main(ref_root: str) -> None:
    jht = jaxshim.import_reference(str(Path(ref_root) / "src"))
    hp = jht.healpix
    rec = jht._recursion
    warnings.simplefilter("ignore")

    out: dict[str, np.ndarray] = {}

    # ---- transforms: synthesis and adjoint_synthesis -----------------------------
    cases = [
        # (tag, nside, lmax, spin, alm kind)
        ("s0_n1_l3", 1, 3, 0, "rand"),
        ("s0_n4_l16", 4, 16, 0, "rand"),
        ("s0_n8_l12", 8, 12, 0, "rand"),
        ("s0_n16_l24", 16, 24, 0, "rand"),
        ("s0_n64_l128", 64, 128, 0, "spec"),  # the CPU-runnable headline case
        ("s2_n2_l5", 2, 5, 2, "rand"),
        ("s2_n4_l16", 4, 16, 2, "rand"),
        ("s2_n8_l12", 8, 12, 2, "rand"),
        ("s2_n16_l24", 16, 24, 2, "rand"),
        ("s2_n32_l64", 32, 64, 2, "spec"),
        ("s0_n12_l20", 12, 20, 0, "rand"),  # nside not a power of two
        ("s2_n12_l20", 12, 20, 2, "rand"),
    ]
    for k, (tag, nside, lmax, spin, kind) in enumerate(cases):
        rng = np.random.default_rng(1000 + k)
        npix = 12 * nside * nside
        lmin = 2 if spin == 2 else 0
        gen = random_alm if kind == "rand" else spectrum_alm
        if spin == 0:
            alm = gen(rng, lmax, lmin=lmin)
            vmap = rng.standard_normal(npix)
        else:
            if kind == "spec":
                alm = np.stack([spectrum_alm(rng, lmax, 1.0, 2), spectrum_alm(rng, lmax, 0.1, 2)])
            else:
                alm = np.stack([random_alm(rng, lmax, 2), random_alm(rng, lmax, 2)])
            vmap = rng.standard_normal((2, npix))
        out[f"{tag}/alm"] = alm
        out[f"{tag}/map"] = np.asarray(hp.synthesis(alm, nside, lmax, spin))
        out[f"{tag}/v"] = vmap
        out[f"{tag}/adj"] = np.asarray(hp.adjoint_synthesis(vmap, nside, lmax, spin))

    # complex a_l0 (imaginary parts are dropped by the real-part projection)
    rng = np.random.default_rng(77)
    a = (rng.standard_normal(alm_size(12)) + 1j * rng.standard_normal(alm_size(12))).astype(np.complex128)
    out["s0_n8_l12_cplx0/alm"] = a
    out["s0_n8_l12_cplx0/map"] = np.asarray(hp.synthesis(a, 8, 12, 0))

    # ---- analysis (weighted Jacobi and bare unweighted) ---------------------------
    ana = [
        ("ana_s0_n16_l24", 16, 24, 0, 3, True, 0.0),
        ("ana_s2_n16_l24", 16, 24, 2, 3, True, 0.0),
        ("ana_s0_n8_l12_bare", 8, 12, 0, 0, False, 0.0),
        ("ana_s0_n16_l32_noise", 16, 32, 0, 3, True, 1e-3),
        ("ana_s2_n8_l16_it2", 8, 16, 2, 2, True, 0.0),
    ]
    for k, (tag, nside, lmax, spin, niter, use_w, sigma) in enumerate(ana):
        rng = np.random.default_rng(2000 + k)
        npix = 12 * nside * nside
        if spin == 0:
            alm = spectrum_alm(rng, lmax)
        else:
            alm = np.stack([spectrum_alm(rng, lmax, 1.0, 2), spectrum_alm(rng, lmax, 0.1, 2)])
        m = np.asarray(hp.synthesis(alm, nside, lmax, spin))
        if sigma:
            m = m + sigma * rng.standard_normal(m.shape)
        out[f"{tag}/map"] = m
        out[f"{tag}/alm"] = np.asarray(
            jht._analysis.analysis(m, nside, lmax, spin=spin, niter=niter, use_weights=use_w)
        )

    # ---- ring / pixel weights -----------------------------------------------------
    for nside in (1, 2, 4, 8, 12, 16, 32, 64):
        out[f"weights/ring_n{nside}"] = np.asarray(jht.weights.ring_weights(nside))
    out["weights/pix_n8"] = np.asarray(jht.weights.pixel_weights(8, True))

    # ---- per-m recursion columns (lambda tables) ------------------------------------
    theta = np.array([1e-3, 0.05, 0.3, 0.9, np.pi / 2, 2.0, 3.0, np.pi - 1e-3])
    x = np.cos(theta)
    out["lambda/x"] = x
    for m in (0, 1, 5, 31, 64):
        out[f"lambda/s0_m{m}"] = np.asarray(rec.normalized_legendre(x, m, 64))
        for s in (2, -2):
            out[f"lambda/s{s}_m{m}"] = np.asarray(rec.spin_weighted_lambda(x, m, s, 64))

    # ---- real-DOF isometry ----------------------------------------------------------
    rng = np.random.default_rng(3000)
    a0 = random_alm(rng, 12)
    a2 = np.stack([random_alm(rng, 12, 2), random_alm(rng, 12, 2)])
    out["real/a0"] = a0
    out["real/x0"] = np.asarray(jht.masked.alm_to_real(a0, 12, 0))
    out["real/a2"] = a2
    out["real/x2"] = np.asarray(jht.masked.alm_to_real(a2, 12, 2))

    # ---- masked CG deconvolution (small) ----------------------------------------------
    nside, lmax = 8, 12
    rng = np.random.default_rng(4000)
    geo = hp.RingInfo(nside)
    zpix = np.repeat(geo.z, geo.npix_ring)
    mask = (np.abs(zpix) >= 0.34).astype(np.float64)
    a_true = spectrum_alm(rng, lmax)
    data = np.asarray(hp.synthesis(a_true, nside, lmax, 0)) + 1e-2 * rng.standard_normal(12 * nside**2)
    out["cg/mask"] = mask
    out["cg/data"] = data
    out["cg/alm"] = np.asarray(jht.masked.deconvolve(data, mask, nside, lmax, 0, tol=1e-8, reg=1e-6))

    # ---- Wiener filter (prior-whitened CG), spin 0 with the mask weighting and zero-power
    #      multipoles, spin 2 with a per-pixel inverse noise ------------------------------
    nside, lmax = 8, 12
    rng = np.random.default_rng(5000)
    ell = np.arange(lmax + 1)
    cl0 = 1.0 / (ell + 10.0) ** 2
    cl0[:2] = 0.0  # monopole and dipole pinned to zero
    a_true = spectrum_alm(rng, lmax)
    data = np.asarray(hp.synthesis(a_true, nside, lmax, 0)) + 1e-2 * rng.standard_normal(12 * nside**2)
    out["wiener/s0_mask"] = mask
    out["wiener/s0_data"] = data
    out["wiener/s0_cl"] = cl0
    out["wiener/s0_alm"] = np.asarray(jht.masked.wiener(data, cl0, nside, lmax, 0, mask=mask, tol=1e-10))
    cle = 1.0 / (ell + 10.0) ** 2
    clb = 0.1 / (ell + 10.0) ** 2
    a2_true = np.stack([spectrum_alm(rng, lmax, 1.0, 2), spectrum_alm(rng, lmax, 0.1, 2)])
    sigma = 1e-2 * (1.0 + 0.5 * np.abs(zpix))
    inv_noise = mask / sigma**2
    data2 = np.asarray(hp.synthesis(a2_true, nside, lmax, 2)) + sigma[None, :] * rng.standard_normal((2, 12 * nside**2))
    out["wiener/s2_invn"] = inv_noise
    out["wiener/s2_data"] = data2
    out["wiener/s2_cl"] = np.stack([cle, clb])
    out["wiener/s2_alm"] = np.asarray(
        jht.masked.wiener(data2, (cle, clb), nside, lmax, 2, inv_noise=inv_noise, tol=1e-10))

    np.savez_compressed(HERE / "jht_golden.npz", **out)
    print(f"wrote {len(out)} arrays to {HERE / 'jht_golden.npz'}")

    off = offgrid_fixtures(jht)
    np.savez_compressed(HERE / "jht_golden_offgrid.npz", **off)
    print(f"wrote {len(off)} arrays to {HERE / 'jht_golden_offgrid.npz'}")


def offgrid_fixtures(jht) -> dict[str, np.ndarray]:
    """jht's own off-grid ``synthesis_general`` / ``adjoint_synthesis_general`` (offgrid.py)
    and its NUFFT plan tables (_nufft.py) on seeded inputs."""
    og, nu = jht.offgrid, jht._nufft
    out: dict[str, np.ndarray] = {}
    cases = [
        # (tag, lmax, spin, npts, epsilon)
        ("og_s0_l16", 16, 0, 40, 1e-10),
        ("og_s0_l40", 40, 0, 60, 1e-10),
        ("og_s2_l16", 16, 2, 40, 1e-10),
        ("og_s2_l40", 40, 2, 60, 1e-10),
        ("og_s0_l24_e6", 24, 0, 30, 1e-6),
        ("og_s2_l24_e12", 24, 2, 30, 1e-12),
    ]
    for k, (tag, lmax, spin, npts, eps) in enumerate(cases):
        rng = np.random.default_rng(6000 + k)
        loc = np.stack([rng.uniform(0.02, np.pi - 0.02, npts), rng.uniform(0.0, 2.0 * np.pi, npts)], axis=1)
        # points on the grid's special lines: both poles, phi = 0, the equator
        loc[:4] = [[0.0, 0.3], [np.pi, 1.1], [0.7, 0.0], [np.pi / 2, 2.0 * np.pi - 1e-9]]
        if spin == 0:
            alm = spectrum_alm(rng, lmax)
            v = rng.standard_normal(npts)
        else:
            alm = np.stack([spectrum_alm(rng, lmax, 1.0, 2), spectrum_alm(rng, lmax, 0.1, 2)])
            v = rng.standard_normal((2, npts))
        out[f"{tag}/loc"] = loc
        out[f"{tag}/alm"] = alm
        out[f"{tag}/field"] = np.asarray(og.synthesis_general(alm, loc, spin=spin, lmax=lmax, epsilon=eps))
        out[f"{tag}/v"] = v
        out[f"{tag}/adj"] = np.asarray(og.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax, epsilon=eps))
    # NUFFT plan tables: oversampled sizes, kernel width and the deconvolution factors
    for tag, (Nk, Nm, eps) in {"nu_a": (36, 33, 1e-10), "nu_b": (64, 49, 1e-6)}.items():
        pl = nu.nufft_plan(Nk, Nm, eps)
        out[f"{tag}/sizes"] = np.array([pl.nk, pl.nm, pl.W], dtype=np.int64)
        out[f"{tag}/beta"] = np.array([pl.beta_k, pl.beta_m])
        out[f"{tag}/corr_k"] = np.asarray(pl.corr_k)
        out[f"{tag}/corr_m"] = np.asarray(pl.corr_m)
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py /path/to/jht/checkout")
    main(sys.argv[1])
