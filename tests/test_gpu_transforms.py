"""GPU parity of the CUDA transforms through the C ABI (needs a B200).

* vs golden vectors produced by the reference's own code (FP64, <= 1e-12 relative);
* vs the CPU oracle at sizes the golden set does not cover;
* the inner-product identity <S a, v> = <a, S^T v>_G (test_grad.py:105-128);
* shape / spin validation and the band-ceiling warning (test_healpix.py:295-313).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TRANSFORM_TAGS, parse_tag, relerr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU hosts
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from oracle import jht_oracle as O  # noqa: E402

TOL = 1e-12


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("tag", TRANSFORM_TAGS)
def test_synthesis_matches_golden(golden, tag):
    spin, nside, lmax = parse_tag(tag)
    out = jhtb.synthesis(golden[f"{tag}/alm"], nside, lmax, spin)
    assert relerr(_np(out), golden[f"{tag}/map"]) <= TOL


@pytest.mark.parametrize("tag", TRANSFORM_TAGS)
def test_adjoint_matches_golden(golden, tag):
    spin, nside, lmax = parse_tag(tag)
    out = jhtb.adjoint_synthesis(golden[f"{tag}/v"], nside, lmax, spin)
    assert relerr(_np(out), golden[f"{tag}/adj"]) <= TOL


def test_complex_m0_projection_matches_golden(golden):
    out = jhtb.synthesis(golden["s0_n8_l12_cplx0/alm"], 8, 12, 0)
    assert relerr(_np(out), golden["s0_n8_l12_cplx0/map"]) <= TOL


def _rand_alm(rng, lmax, spin):
    K = O.alm_size(lmax)
    ells, _ = O.lm_of_index(lmax)

    def one():
        a = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / np.sqrt(2)
        a[: lmax + 1] = a[: lmax + 1].real
        if spin == 2:
            a[ells < 2] = 0
        return a

    return one() if spin == 0 else np.stack([one(), one()])


@pytest.mark.parametrize(
    "nside,lmax",
    [(1, 0), (1, 4), (2, 1), (3, 7), (5, 9), (32, 48), (64, 200), (128, 256), (256, 300), (100, 150)],
)
@pytest.mark.parametrize("spin", [0, 2])
def test_transforms_match_oracle(nside, lmax, spin):
    rng = np.random.default_rng(nside * 1000 + lmax + spin)
    a = _rand_alm(rng, lmax, spin)
    npix = 12 * nside * nside
    v = rng.standard_normal(npix if spin == 0 else (2, npix))
    ref_s = O.synthesis(a, nside, lmax, spin)
    ref_a = O.adjoint_synthesis(v, nside, lmax, spin)
    out_s = _np(jhtb.synthesis(a, nside, lmax, spin))
    out_a = _np(jhtb.adjoint_synthesis(v, nside, lmax, spin))
    if np.max(np.abs(ref_s)) > 0:
        assert relerr(out_s, ref_s) <= TOL
    else:
        assert np.max(np.abs(out_s)) == 0.0
    if np.max(np.abs(ref_a)) > 0:
        assert relerr(out_a, ref_a) <= TOL
    else:
        assert np.max(np.abs(out_a)) == 0.0


@pytest.mark.parametrize("nside,lmax,spin", [(16, 24, 0), (16, 24, 2), (512, 1024, 0), (256, 512, 2)])
def test_inner_product_identity(nside, lmax, spin):
    rng = np.random.default_rng(7 + spin)
    a = torch.as_tensor(_rand_alm(rng, lmax, spin), device="cuda")
    npix = 12 * nside * nside
    v = torch.randn((npix,) if spin == 0 else (2, npix), dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(3))
    lhs = float(torch.sum(jhtb.synthesis(a, nside, lmax, spin) * v))
    b = jhtb.adjoint_synthesis(v, nside, lmax, spin)
    G = torch.as_tensor(jhtb.alm_metric_weight(lmax), device="cuda")
    rhs = float(torch.sum(G * torch.real(torch.conj(a) * b)))
    assert abs(lhs - rhs) / abs(lhs) <= TOL


def test_batch_matches_single():
    nside, lmax = 16, 32
    rng = np.random.default_rng(11)
    for spin in (0, 2):
        a = np.stack([_rand_alm(rng, lmax, spin) for _ in range(5)])
        out = _np(jhtb.synthesis_batch(a, nside, lmax, spin))
        for b in range(5):
            assert relerr(out[b], _np(jhtb.synthesis(a[b], nside, lmax, spin))) == 0.0
        back = _np(jhtb.adjoint_synthesis_batch(out, nside, lmax, spin))
        for b in range(5):
            assert relerr(back[b], _np(jhtb.adjoint_synthesis(out[b], nside, lmax, spin))) == 0.0


def test_deterministic():
    nside, lmax = 64, 128
    rng = np.random.default_rng(5)
    v = rng.standard_normal((2, 12 * nside**2))
    a1 = _np(jhtb.adjoint_synthesis(v, nside, lmax, 2))
    a2 = _np(jhtb.adjoint_synthesis(v, nside, lmax, 2))
    assert np.array_equal(a1, a2)


def test_input_validation():
    nside, lmax = 16, 24
    K = jhtb.alm_size(lmax)
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis(np.zeros(K - 1, dtype=np.complex128), nside, lmax, spin=0)
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis(np.zeros(K, dtype=np.complex128), nside, lmax, spin=2)
    with pytest.raises(ValueError, match="map shape"):
        jhtb.adjoint_synthesis(np.zeros(12 * nside**2 - 1), nside, lmax, spin=0)
    with pytest.raises(ValueError, match="map shape"):
        jhtb.adjoint_synthesis(np.zeros(12 * nside**2), nside, lmax, spin=2)
    with pytest.raises(NotImplementedError):
        jhtb.synthesis(np.zeros((2, K), dtype=np.complex128), nside, lmax, spin=1)


def test_band_ceiling_warning():
    a = np.zeros(jhtb.alm_size(7), dtype=np.complex128)
    with pytest.warns(UserWarning, match="ceiling"):
        jhtb.synthesis(a, 4, 7, spin=0)


@pytest.mark.parametrize("spin", [0, 2])
def test_transforms_replay_in_a_cuda_graph(spin):
    """S and S^T captured once in a CUDA graph (plan built before the capture) and replayed
    on new inputs give the eager results bit for bit: the C ABI calls are stream-ordered
    and allocate nothing inside a capture."""
    nside, lmax = 32, 48
    rng = np.random.default_rng(80 + spin)
    K = jhtb.alm_size(lmax)
    shape = (K,) if spin == 0 else (2, K)
    npix = 12 * nside * nside
    mshape = (npix,) if spin == 0 else (2, npix)

    def rand_alm():
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        a[..., : lmax + 1] = a[..., : lmax + 1].real
        return torch.as_tensor(a, device="cuda")

    a_in = rand_alm()
    v_in = torch.as_tensor(rng.standard_normal(mshape), device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up: builds the plan outside the capture
        jhtb.synthesis(a_in, nside, lmax, spin)
        jhtb.adjoint_synthesis(v_in, nside, lmax, spin)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        m_out = jhtb.synthesis(a_in, nside, lmax, spin)
        b_out = jhtb.adjoint_synthesis(v_in, nside, lmax, spin)
    for _ in range(2):
        a_new, v_new = rand_alm(), torch.as_tensor(rng.standard_normal(mshape), device="cuda")
        a_in.copy_(a_new)
        v_in.copy_(v_new)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(m_out, jhtb.synthesis(a_new, nside, lmax, spin))
        assert torch.equal(b_out, jhtb.adjoint_synthesis(v_new, nside, lmax, spin))
