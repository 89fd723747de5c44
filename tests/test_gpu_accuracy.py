"""Round-trip accuracy gates of jht's analysis, on the B200 (jht tests/test_accuracy.py,
tests/test_floor.py), plus the off-grid real-DOF transpose (diff.py:79-107).

* weighted + niter = 3 broadband round trip ``max|analysis(synthesis(a)) - a| <= 1e-4``
  over nside x lmax in {(32, 32), (64, 64), (128, 128), (256, 256), (64, 96)}, spin 0 / 2;
* ring weights beat the unweighted bare estimator;
* spin 2 iterates to the same deep floor as spin 0 (< 1e-9 at lmax = nside);
* single spin-2 modes at nside 8, l0 = 8: the bare inverse stays at the HEALPix floor
  (< 1e-2, no m < l defect), iteration drives it below 1e-4, and the spin-2 floor is
  within 5x of the spin-0 one.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from jht_b200.healpix import alm_column_base  # noqa: E402

GATE = 1e-4
DEEP_FLOOR = 1e-9


def _broadband(lmax, spin, seed=0):
    rng = np.random.default_rng(seed)
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)

    def one():
        a = rng.standard_normal(K) + 1j * rng.standard_normal(K)
        a[: lmax + 1] = a[: lmax + 1].real
        a[ell < abs(spin)] = 0.0
        return a

    return one() if spin == 0 else np.stack([one(), one()])


def _roundtrip(a, nside, lmax, spin, niter, use_weights):
    m = jhtb.synthesis(a, nside, lmax, spin)
    r = jhtb.analysis(m, nside, lmax, spin, niter=niter, use_weights=use_weights)
    return float(torch.max(torch.abs(r - torch.as_tensor(a, device=r.device))))


@pytest.mark.parametrize("nside,lmax", [(32, 32), (64, 64), (128, 128), (256, 256), (64, 96)])
@pytest.mark.parametrize("spin", [0, 2])
def test_weighted_iterated_round_trip_meets_gate(nside, lmax, spin):
    a = _broadband(lmax, spin)
    assert _roundtrip(a, nside, lmax, spin, 3, True) <= GATE


@pytest.mark.parametrize("nside,lmax", [(32, 32), (64, 64)])
@pytest.mark.parametrize("spin", [0, 2])
def test_ring_weights_beat_unweighted_bare(nside, lmax, spin):
    a = _broadband(lmax, spin)
    assert _roundtrip(a, nside, lmax, spin, 0, True) < _roundtrip(a, nside, lmax, spin, 0, False)


@pytest.mark.parametrize("nside,lmax", [(64, 64), (128, 128)])
def test_spin2_reaches_the_spin0_floor(nside, lmax):
    assert _roundtrip(_broadband(lmax, 0), nside, lmax, 0, 3, True) < DEEP_FLOOR
    assert _roundtrip(_broadband(lmax, 2), nside, lmax, 2, 3, True) < DEEP_FLOOR


NS, LM, L0 = 8, 12, 8


def _single_mode(m0, spin, niter, channel=0):
    K = jhtb.alm_size(LM)
    if spin == 0:
        a = np.zeros(K, complex)
        a[alm_column_base(m0, LM) + (L0 - m0)] = 1.0
    else:
        a = np.zeros((2, K), complex)
        a[channel, alm_column_base(m0, LM) + (L0 - m0)] = 1.0
    return _roundtrip(a, NS, LM, spin, niter, False)


def test_spin2_single_modes_sit_at_the_healpix_floor():
    errs = [_single_mode(m0, 2, 0) for m0 in (0, 4, 8)]
    assert max(errs) < 1e-2


def test_spin2_single_mode_iteration_converges():
    bare, it = _single_mode(4, 2, 0), _single_mode(4, 2, 3)
    assert it < bare
    assert it < 1e-4


def test_spin2_floor_matches_spin0_floor():
    assert _single_mode(4, 2, 0) < 5.0 * _single_mode(4, 0, 0)


@pytest.mark.parametrize("spin", [0, 2])
def test_offgrid_real_dof_transpose(spin):
    """<S_g T^-1 x, v> = <x, T S_g^T v> in plain real inner products (diff.py:95-107)."""
    lmax, npts = 20, 80
    rng = np.random.default_rng(12 + spin)
    x = torch.as_tensor(rng.standard_normal(jhtb.n_dof(lmax, spin)), device="cuda")
    loc = np.stack([rng.uniform(0, np.pi, npts), rng.uniform(0, 2 * np.pi, npts)], axis=1)
    v = torch.as_tensor(rng.standard_normal(npts) if spin == 0 else rng.standard_normal((2, npts)), device="cuda")
    lhs = float(torch.sum(jhtb.synthesis_general_real(x, loc, spin=spin, lmax=lmax) * v))
    rhs = float(torch.sum(x * jhtb.adjoint_synthesis_general_real(v, loc, spin=spin, lmax=lmax)))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
