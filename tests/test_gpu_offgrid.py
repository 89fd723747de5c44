"""Off-grid transforms on a B200 against jht's own outputs, the oracle and the exact sum.

* forward / adjoint vs the golden vectors produced by jht's ``synthesis_general`` /
  ``adjoint_synthesis_general`` (poles, phi = 0 and the equator among the points);
* vs the NumPy restatement at larger sizes, and vs the exact point-by-point sum
  a_lm sY_lm at jht's accuracy tier (FWD_TOL = 1e-9 at epsilon = 1e-10, jht
  tests/test_offgrid.py:38);
* the adjoint identity <S_g a, v> = <a, S_g^T v>_G (jht's ADJ_TOL = 1e-12);
* torch gradients in a_lm (real DOFs) and in the pointing (theta, phi) vs central
  finite differences (jht's FD_TOL = 1e-6).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from oracle import offgrid_oracle as G  # noqa: E402

GOLD = np.load(ROOT / "tests" / "golden" / "jht_golden_offgrid.npz")


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.max(np.abs(a - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def _alm(rng, lmax, spin):
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)

    def one(amp):
        a = np.sqrt(amp / 2) * (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / (ell + 10.0)
        a[: lmax + 1] = a[: lmax + 1].real * np.sqrt(2)
        if spin == 2:
            a[ell < 2] = 0
        return a

    return one(1.0) if spin == 0 else np.stack([one(1.0), one(0.1)])


def _loc(rng, n):
    return np.stack([rng.uniform(0.0, np.pi, n), rng.uniform(0.0, 2.0 * np.pi, n)], axis=1)


@pytest.mark.parametrize("tag,lmax,spin,eps", [
    ("og_s0_l16", 16, 0, 1e-10), ("og_s0_l40", 40, 0, 1e-10), ("og_s2_l16", 16, 2, 1e-10),
    ("og_s2_l40", 40, 2, 1e-10), ("og_s0_l24_e6", 24, 0, 1e-6), ("og_s2_l24_e12", 24, 2, 1e-12)])
def test_offgrid_matches_reference_golden(tag, lmax, spin, eps):
    loc, alm, v = GOLD[f"{tag}/loc"], GOLD[f"{tag}/alm"], GOLD[f"{tag}/v"]
    f = jhtb.synthesis_general(alm, loc, spin=spin, lmax=lmax, epsilon=eps)
    assert _rel(f, GOLD[f"{tag}/field"]) <= 1e-12
    a = jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax, epsilon=eps)
    assert _rel(a, GOLD[f"{tag}/adj"]) <= 1e-12


@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("lmax,npts", [(1, 10), (127, 400), (200, 300)])
def test_offgrid_matches_oracle_and_direct_sum(spin, lmax, npts):
    rng = np.random.default_rng(lmax + spin)
    alm, loc = _alm(rng, lmax, spin), _loc(rng, npts)
    if spin == 2 and lmax < 2:
        pytest.skip("no spin-2 modes below l = 2")
    f = jhtb.synthesis_general(alm, loc, spin=spin, lmax=lmax)
    assert _rel(f, G.synthesis_general(alm, loc, lmax, spin)) <= 1e-12
    assert _rel(f, G.direct_field(alm, loc, lmax, spin)) <= 1e-9
    v = rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts))
    a = jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax)
    assert _rel(a, G.adjoint_synthesis_general(v, loc, lmax, spin)) <= 1e-12


@pytest.mark.parametrize("spin", [0, 2])
def test_offgrid_adjoint_identity(spin):
    lmax, npts = 300, 200_000  # enough points for the tile-sorted path
    rng = np.random.default_rng(31 + spin)
    alm, loc = _alm(rng, lmax, spin), _loc(rng, npts)
    v = rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts))
    lhs = float(torch.sum(jhtb.synthesis_general(alm, loc, spin=spin, lmax=lmax) * torch.as_tensor(v, device="cuda")))
    b = jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax).cpu().numpy()
    gm = jhtb.alm_metric_weight(lmax)
    rhs = float(np.sum(gm * np.real(np.conj(np.atleast_2d(alm)) * np.atleast_2d(b))))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("spin", [0, 2])
def test_offgrid_alm_gradient_matches_fd(spin):
    lmax, npts = 24, 50
    rng = np.random.default_rng(5 + spin)
    alm, loc = _alm(rng, lmax, spin), _loc(rng, npts)
    d = rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts))
    d_t = torch.as_tensor(d, device="cuda")

    def loss(a):
        f = jhtb.synthesis_general(a, loc, spin=spin, lmax=lmax)
        return 0.5 * torch.sum((f - d_t) ** 2)

    a = torch.as_tensor(alm, device="cuda").requires_grad_(True)
    loss(a).backward()
    gr = a.grad.detach().cpu().numpy()
    h = 1e-6
    flat = alm.reshape(-1)
    for idx in rng.choice(flat.size, 12, replace=False):
        for unit in (1.0, 1j):
            e = np.zeros_like(flat)
            e[idx] = unit * h
            lp = float(loss(torch.as_tensor((flat + e).reshape(alm.shape), device="cuda")))
            lm = float(loss(torch.as_tensor((flat - e).reshape(alm.shape), device="cuda")))
            fd = (lp - lm) / (2 * h)
            an = gr.reshape(-1)[idx].real if unit == 1.0 else gr.reshape(-1)[idx].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (idx, unit, fd, an)


@pytest.mark.parametrize("spin", [0, 2])
def test_offgrid_pointing_gradient_matches_fd(spin):
    lmax, npts = 40, 64
    rng = np.random.default_rng(17 + spin)
    alm = torch.as_tensor(_alm(rng, lmax, spin), device="cuda")
    loc0 = _loc(rng, npts)
    loc0[:, 0] = np.clip(loc0[:, 0], 0.05, np.pi - 0.05)
    w = torch.as_tensor(rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts)), device="cuda")

    def loss(lc):
        return torch.sum(w * jhtb.synthesis_general(alm, lc, spin=spin, lmax=lmax))

    lc = torch.as_tensor(loc0, device="cuda").requires_grad_(True)
    loss(lc).backward()
    gl = lc.grad.detach().cpu().numpy()
    h = 1e-6
    for j in rng.choice(npts, 10, replace=False):
        for ax in (0, 1):
            e = np.zeros_like(loc0)
            e[j, ax] = h
            fd = (float(loss(torch.as_tensor(loc0 + e, device="cuda"))) -
                  float(loss(torch.as_tensor(loc0 - e, device="cuda")))) / (2 * h)
            assert abs(fd - gl[j, ax]) <= 1e-6 * max(1.0, abs(fd)), (j, ax, fd, gl[j, ax])


def test_offgrid_adjoint_gradient_in_the_field():
    lmax, npts, spin = 16, 30, 2
    rng = np.random.default_rng(44)
    loc = _loc(rng, npts)
    v = torch.as_tensor(rng.standard_normal((2, npts)), device="cuda").requires_grad_(True)
    c = torch.as_tensor(_alm(rng, lmax, spin), device="cuda")
    gm = torch.as_tensor(jhtb.alm_metric_weight(lmax), device="cuda")
    out = jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax)
    L = torch.sum(gm * torch.real(torch.conj(c) * out))
    L.backward()
    # <c, S^T v>_G = <S c, v>: its gradient in v is S c
    ref = jhtb.synthesis_general(c, loc, spin=spin, lmax=lmax)
    assert _rel(v.grad, ref.detach().cpu().numpy()) <= 1e-10


def test_offgrid_rejects_bad_inputs():
    loc = np.zeros((4, 2))
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis_general(np.zeros(5, complex), loc, spin=0, lmax=4)
    with pytest.raises(TypeError):
        jhtb.adjoint_synthesis_general(np.zeros(4, complex), loc, spin=0, lmax=4)
    with pytest.raises(ValueError, match="field shape"):
        jhtb.adjoint_synthesis_general(np.zeros(5), loc, spin=0, lmax=4)


def test_tiled_spread_equals_plain_spread():
    """jhtb_nufft_spread_tiles (per-tile sums in on-chip memory) against jhtb_nufft_spread on
    the same points, including points whose coordinates lie outside [0, 2 pi) (their tile
    key names another tile, so they take the direct path)."""
    import ctypes

    from jht_b200 import _lib, offgrid

    g = offgrid._geometry(64, 0, 1e-10, torch.cuda.current_device())
    rng = np.random.default_rng(3)
    n = 100_000
    th = rng.uniform(0, np.pi, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    th[:50] = rng.uniform(-3.0, -0.1, 50)
    ph[50:100] = rng.uniform(6.5, 9.0, 50)
    theta = torch.as_tensor(th, device="cuda")
    phi = torch.as_tensor(ph, device="cuda")
    vals = torch.complex(torch.randn(n, dtype=torch.float64, device="cuda"), torch.randn(n, dtype=torch.float64, device="cuda"))
    ks, order = torch.sort(offgrid._tile_keys(g, theta, phi))
    theta, phi, vals = theta[order].contiguous(), phi[order].contiguous(), vals[order].contiguous()
    s0, c0, t0 = offgrid._segments(ks)
    lib = _lib.load_library()
    g1 = torch.zeros((g.nk, g.nm), dtype=torch.complex128, device="cuda")
    g2 = torch.zeros_like(g1)
    _lib.check(lib.jhtb_nufft_spread(vals.data_ptr(), theta.data_ptr(), phi.data_ptr(), n, g.nk, g.nm, g.W,
                                     ctypes.c_double(g.beta), g1.data_ptr(), _lib.stream_ptr()), "spread")
    _lib.check(lib.jhtb_nufft_spread_tiles(vals.data_ptr(), theta.data_ptr(), phi.data_ptr(), n, s0.numel(),
                                           s0.data_ptr(), c0.data_ptr(), t0.data_ptr(), g.tiles_m, g.nk, g.nm, g.W,
                                           ctypes.c_double(g.beta), g2.data_ptr(), _lib.stream_ptr()), "spread_tiles")
    assert float(torch.max(torch.abs(g1 - g2))) <= 1e-12 * float(torch.max(torch.abs(g1)))
