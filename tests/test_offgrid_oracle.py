"""CPU checks of the off-grid restatement and of the product's host-side NUFFT tables.

* the oracle reproduces jht's own ``synthesis_general`` / ``adjoint_synthesis_general``
  (golden vectors from the reference source, tests/golden/make_golden.py) to rounding;
* the golden fields agree with the exact point-by-point sum a_lm sY_lm at the accuracy
  tier the kernel table promises (offgrid tests in jht: forward vs direct <= 1e-9);
* the product's kernel-table lookup, FFT sizes and deconvolution factors equal jht's
  plan tables (_nufft.py:97-147).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import ROOT
from oracle import offgrid_oracle as G

GOLD = np.load(ROOT / "tests" / "golden" / "jht_golden_offgrid.npz")
CASES = [
    ("og_s0_l16", 16, 0, 1e-10),
    ("og_s0_l40", 40, 0, 1e-10),
    ("og_s2_l16", 16, 2, 1e-10),
    ("og_s2_l40", 40, 2, 1e-10),
    ("og_s0_l24_e6", 24, 0, 1e-6),
    ("og_s2_l24_e12", 24, 2, 1e-12),
]


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


@pytest.mark.parametrize("tag,lmax,spin,eps", CASES)
def test_oracle_matches_reference_offgrid(tag, lmax, spin, eps):
    loc, alm, v = GOLD[f"{tag}/loc"], GOLD[f"{tag}/alm"], GOLD[f"{tag}/v"]
    assert _rel(G.synthesis_general(alm, loc, lmax, spin, eps), GOLD[f"{tag}/field"]) <= 1e-13
    assert _rel(G.adjoint_synthesis_general(v, loc, lmax, spin, eps), GOLD[f"{tag}/adj"]) <= 1e-13


@pytest.mark.parametrize("tag,lmax,spin,eps", CASES)
def test_reference_offgrid_meets_its_accuracy_tier(tag, lmax, spin, eps):
    loc, alm = GOLD[f"{tag}/loc"], GOLD[f"{tag}/alm"]
    tol = 1e-9 if eps <= 1e-10 else 1e-6
    assert _rel(G.direct_field(alm, loc, lmax, spin), GOLD[f"{tag}/field"]) <= tol


@pytest.mark.parametrize("spin", [0, 2])
def test_oracle_adjoint_identity(spin):
    lmax, npts = 20, 37
    rng = np.random.default_rng(9)
    loc = np.stack([rng.uniform(0, np.pi, npts), rng.uniform(0, 2 * np.pi, npts)], axis=1)
    K = G.O.alm_size(lmax)
    a = rng.standard_normal((2, K)) + 1j * rng.standard_normal((2, K))
    a[:, : lmax + 1] = a[:, : lmax + 1].real
    a = a[0] if spin == 0 else a
    v = rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts))
    lhs = float(np.sum(G.synthesis_general(a, loc, lmax, spin) * v))
    b = G.adjoint_synthesis_general(v, loc, lmax, spin)
    gm = G.O.metric_weight(lmax)
    rhs = float(np.sum(gm * np.real(np.conj(np.atleast_2d(a)) * np.atleast_2d(b))))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("tag,Nk,Nm,eps", [("nu_a", 36, 33, 1e-10), ("nu_b", 64, 49, 1e-6)])
def test_product_nufft_tables_match_reference(tag, Nk, Nm, eps):
    from jht_b200 import offgrid

    W, sigma = offgrid._kernel_for(eps)
    nk, nm = offgrid._fft_size(sigma * Nk), offgrid._fft_size(sigma * Nm)
    np.testing.assert_array_equal([nk, nm, W], GOLD[f"{tag}/sizes"])
    beta = float(np.pi * W * (1.0 - 0.5 / sigma))
    assert beta == GOLD[f"{tag}/beta"][0]
    np.testing.assert_allclose(offgrid._kernel_ft(Nk, nk, W, beta), GOLD[f"{tag}/corr_k"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(offgrid._kernel_ft(Nm, nm, W, beta), GOLD[f"{tag}/corr_m"], rtol=1e-14, atol=0)


def test_offgrid_validation_errors_without_gpu():
    import jht_b200 as jhtb

    with pytest.raises(NotImplementedError):
        jhtb.synthesis_general(np.zeros(jhtb.alm_size(4), complex), np.zeros((3, 2)), spin=1, lmax=4)
    with pytest.raises(ValueError, match="loc must have shape"):
        jhtb.synthesis_general(np.zeros(jhtb.alm_size(4), complex), np.zeros((3, 3)), spin=0, lmax=4)


def test_tile_segments_cover_every_sorted_point_once():
    """Host-side grouping of the points for the tiled spread: segments of one tile each,
    at most _SEG_POINTS long, covering the sorted points exactly once in order."""
    import types

    import torch

    from jht_b200 import offgrid

    g = types.SimpleNamespace(nk=8640, nm=8640, tiles_m=8640 // 32 + 2)
    rng = np.random.default_rng(7)
    n = 50_000
    th = np.concatenate([rng.uniform(0, np.pi, n - 3000), np.full(3000, 0.5)])  # one crowded tile
    ph = np.concatenate([rng.uniform(0, 2 * np.pi, n - 3000), np.full(3000, 1.0)])
    th[:5] = [-0.3, 7.0, np.nan, 0.0, np.pi]
    keys = offgrid._tile_keys(g, torch.as_tensor(th), torch.as_tensor(ph))
    assert int(keys.min()) >= 0
    ks, order = torch.sort(keys)
    start, count, tile = offgrid._segments(ks)
    assert int(count.max()) <= offgrid._SEG_POINTS
    assert int(count.min()) >= 1
    ends = start + count.to(torch.int64)
    assert int(start[0]) == 0 and int(ends[-1]) == n
    assert torch.equal(start[1:], ends[:-1])  # contiguous, in order, no overlap
    for i in rng.choice(start.numel(), 50, replace=False):
        seg = ks[int(start[i]) : int(ends[i])]
        assert bool(torch.all(seg == tile[i]))
    crowded = int(offgrid._tile_keys(g, torch.tensor([0.5]), torch.tensor([1.0]))[0])
    n_crowded = int((ks == crowded).sum())
    assert n_crowded >= 3000
    assert int((tile == crowded).sum()) == -(-n_crowded // offgrid._SEG_POINTS)
