"""Batched mixed-precision (BF16x3 tensor-core) synthesis vs the FP64 path (needs a B200).

The mixed form must stay within 1e-6 of FP64 (relative to each map's max), and the
device-side error flag of its bounded waits must stay clear.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from jht_b200 import _lib  # noqa: E402

MIXED_TOL = 1e-6


def _alms(rng, B, lmax, spin, amp_spread=False):
    K = jhtb.alm_size(lmax)
    ells = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    shape = (B, K) if spin == 0 else (B, 2, K)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    a = a / (ells + 10.0)
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    if spin == 2:
        a[..., ells < 2] = 0
    if amp_spread:  # per-map amplitude log-uniform in [1e-2, 1e2]
        amp = 10.0 ** rng.uniform(-2, 2, size=B)
        a = a * amp.reshape((B,) + (1,) * (a.ndim - 1))
    return a


@pytest.mark.parametrize("nside,lmax,B", [(8, 12, 2), (16, 40, 9), (64, 128, 3), (128, 256, 8), (32, 96, 17)])
@pytest.mark.parametrize("spin", [0, 2])
def test_bf16x3_synthesis_matches_fp64(nside, lmax, B, spin):
    rng = np.random.default_rng(nside + lmax + B + spin)
    a = _alms(rng, B, lmax, spin, amp_spread=True)
    ref = jhtb.synthesis_batch(a, nside, lmax, spin).cpu().numpy()
    out = jhtb.synthesis_batch(a, nside, lmax, spin, precision="bf16x3").cpu().numpy()
    plan = _lib.get_plan(nside, lmax, spin, "bf16x3", B)
    assert plan.status() == 0
    for b in range(B):
        err = np.max(np.abs(out[b] - ref[b])) / np.max(np.abs(ref[b]))
        assert err <= MIXED_TOL, (b, err)


@pytest.mark.slow
def test_bf16x3_batch64_at_nside512():
    """64 spin-0 maps at nside 512, lmax 1024, per-map amplitudes log-uniform in [1e-2, 1e2]:
    every map within 1e-6 of the FP64 synthesis (the batched configuration's error report)."""
    nside, lmax, B, spin = 512, 1024, 64, 0
    rng = np.random.default_rng(64)
    a = _alms(rng, B, lmax, spin, amp_spread=True)
    a_t = torch.as_tensor(a, device="cuda")
    out = jhtb.synthesis_batch(a_t, nside, lmax, spin, precision="bf16x3")
    assert _lib.get_plan(nside, lmax, spin, "bf16x3", B).status() == 0
    worst = 0.0
    for b0 in range(0, B, 16):
        ref = jhtb.synthesis_batch(a_t[b0 : b0 + 16], nside, lmax, spin)
        got = out[b0 : b0 + 16]
        err = torch.amax(torch.abs(got - ref), dim=1) / torch.amax(torch.abs(ref), dim=1)
        worst = max(worst, float(err.max()))
    assert worst <= MIXED_TOL


def _maps(rng, B, nside, spin, amp_spread=True):
    npix = 12 * nside * nside
    shape = (B, npix) if spin == 0 else (B, 2, npix)
    m = rng.standard_normal(shape)
    if amp_spread:
        amp = 10.0 ** rng.uniform(-2, 2, size=B)
        m = m * amp.reshape((B,) + (1,) * (m.ndim - 1))
    return m


# (nside, lmax, B): partial last map group (B not a multiple of 16), lmax below one 128-degree
# block, lmax far above nside (m mod N folds, many dead polar rings), several blocks per order
@pytest.mark.parametrize("nside,lmax,B", [(8, 12, 2), (16, 40, 9), (64, 128, 3), (128, 256, 16), (32, 300, 17)])
@pytest.mark.parametrize("spin", [0, 2])
def test_bf16x3_adjoint_matches_fp64(nside, lmax, B, spin):
    """The tensor-core adjoint (split-BF16 products, FP32 sums folded into FP64 every 256
    rings) within 1e-6 of the FP64 adjoint for every map, amplitudes spread over 1e-2..1e2."""
    rng = np.random.default_rng(1000 + nside + lmax + B + spin)
    v = _maps(rng, B, nside, spin)
    ref = jhtb.adjoint_synthesis_batch(v, nside, lmax, spin).cpu().numpy()
    out = jhtb.adjoint_synthesis_batch(v, nside, lmax, spin, precision="bf16x3").cpu().numpy()
    assert _lib.get_plan(nside, lmax, spin, "bf16x3", B).status() == 0
    for b in range(B):
        err = np.max(np.abs(out[b] - ref[b])) / np.max(np.abs(ref[b]))
        assert err <= MIXED_TOL, (b, err)


@pytest.mark.slow
@pytest.mark.parametrize("spin", [0, 2])
def test_bf16x3_adjoint_batch64_at_nside512(spin):
    """64 maps at nside 512, lmax 1024 (the batched configuration), per-map amplitudes
    log-uniform in [1e-2, 1e2]: every adjoint within 1e-6 of FP64."""
    nside, lmax, B = 512, 1024, 64
    rng = np.random.default_rng(640 + spin)
    v = torch.as_tensor(_maps(rng, B, nside, spin), device="cuda")
    out = jhtb.adjoint_synthesis_batch(v, nside, lmax, spin, precision="bf16x3")
    assert _lib.get_plan(nside, lmax, spin, "bf16x3", B).status() == 0
    worst = 0.0
    for b0 in range(0, B, 16):
        ref = jhtb.adjoint_synthesis_batch(v[b0 : b0 + 16], nside, lmax, spin)
        got = out[b0 : b0 + 16]
        err = torch.amax(torch.abs(got - ref).reshape(16, -1), dim=1) / torch.amax(torch.abs(ref).reshape(16, -1), dim=1)
        worst = max(worst, float(err.max()))
    print(f"tensor-core adjoint, nside 512, lmax 1024, spin {spin}: worst per-map error {worst:.3e}")
    assert worst <= MIXED_TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_tuning_knobs_keep_the_results(spin):
    """Every knob setting the autotuner may pick keeps the transforms: mixed precision within
    1e-6 of FP64, FP64 bit-identical to the default launch."""
    nside, lmax, B = 32, 96, 9
    rng = np.random.default_rng(77 + spin)
    a = torch.as_tensor(_alms(rng, B, lmax, spin, amp_spread=True), device="cuda").reshape(B, -1, jhtb.alm_size(lmax))
    v = torch.as_tensor(_maps(rng, B, nside, spin), device="cuda").reshape(B, a.shape[1], -1)

    def pair(plan):
        m = torch.empty(v.shape, dtype=torch.float64, device="cuda")
        b = torch.empty(a.shape, dtype=torch.complex128, device="cuda")
        s = _lib.stream_ptr()
        _lib.check(plan.lib.jhtb_synthesis(plan.handle, a.data_ptr(), m.data_ptr(), B, s), "synthesis")
        _lib.check(plan.lib.jhtb_adjoint_synthesis(plan.handle, v.data_ptr(), b.data_ptr(), B, s), "adjoint")
        torch.cuda.synchronize()
        return m, b

    p64 = _lib.Plan(nside, lmax, spin, "fp64", max_batch=B)
    m0, b0 = pair(p64)
    for c in (1, 2, 3):
        p64.set_tuning(leg_ctas=c)
        m1, b1 = pair(p64)
        assert torch.equal(m0, m1) and torch.equal(b0, b1)
    p64.close()
    pm = _lib.Plan(nside, lmax, spin, "bf16x3", max_batch=B)
    from jht_b200 import autotune as A

    for knobs in A.candidates("bf16x3", spin) + [{"tc_fold": 128, "tca_fold": 64}]:
        pm.set_tuning(**knobs)
        m1, b1 = pair(pm)
        assert pm.status() == 0
        em = torch.amax(torch.abs(m1 - m0).reshape(B, -1), 1) / torch.amax(torch.abs(m0).reshape(B, -1), 1)
        eb = torch.amax(torch.abs(b1 - b0).reshape(B, -1), 1) / torch.amax(torch.abs(b0).reshape(B, -1), 1)
        assert float(em.max()) <= MIXED_TOL and float(eb.max()) <= MIXED_TOL, (knobs, float(em.max()), float(eb.max()))
    pm.close()
