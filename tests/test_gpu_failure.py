"""Failure detection on the GPU without a GPU fault.

* The tensor-core kernels bound every wait between their warp roles (a poll count and a
  watchdog time limit).  The test shortens the limit, injects a stall (the operand
  builders publish nothing, so the waits on them run out), and checks that the kernel
  reports status 1, returns, releases its tensor memory (the next launches allocate it
  again on every SM) and that the next call on the same plan is correct.
* Non-finite inputs propagate to the outputs they touch and leave the plan usable.
* A device allocation that cannot be satisfied is reported as MemoryError, and the
  library keeps working.
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


def _alm(rng, B, lmax):
    K = jhtb.alm_size(lmax)
    a = rng.standard_normal((B, 2, K)) + 1j * rng.standard_normal((B, 2, K))
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    return torch.as_tensor(a, device="cuda")


def _synth(plan, a, B, npix):
    out = torch.empty((B, 2, npix), dtype=torch.float64, device="cuda")
    _lib.check(plan.lib.jhtb_synthesis(plan.handle, a.data_ptr(), out.data_ptr(), B, _lib.stream_ptr()),
               "jhtb_synthesis")
    return out


@pytest.mark.parametrize("nside,lmax,B", [(16, 24, 2), (64, 128, 16)])
def test_tensor_core_wait_runs_out_and_the_plan_recovers(nside, lmax, B):
    rng = np.random.default_rng(5)
    a = _alm(rng, B, lmax)
    npix = 12 * nside * nside
    ref = jhtb.synthesis_batch(a, nside, lmax, 2)  # FP64
    plan = _lib.Plan(nside, lmax, 2, "bf16x3", max_batch=B)
    try:
        plan.set_watchdog(20_000_000)  # 20 ms
        plan.inject_fault(1)
        _synth(plan, a, B, npix)
        assert plan.status() == 1
        # a second stalled call on the same plan: the kernel left nothing behind
        _synth(plan, a, B, npix)
        assert plan.status() == 1
        plan.inject_fault(0)
        plan.set_watchdog(2_000_000_000)
        for _ in range(2):
            got = _synth(plan, a, B, npix)
            assert plan.status() == 0
            err = float(torch.max(torch.abs(got - ref)) / torch.max(torch.abs(ref)))
            assert err <= 1e-6, err
    finally:
        plan.close()
    # a fresh plan (every SM allocates tensor memory again) is correct as well
    got = jhtb.synthesis_batch(a, nside, lmax, 2, precision="bf16x3")
    assert float(torch.max(torch.abs(got - ref)) / torch.max(torch.abs(ref))) <= 1e-6


def test_watchdog_and_injection_arguments_are_checked():
    plan = _lib.Plan(8, 12, 2, "bf16x3", max_batch=1)
    try:
        with pytest.raises(ValueError):
            plan.set_watchdog(10)
        with pytest.raises(ValueError):
            plan.inject_fault(7)
    finally:
        plan.close()


def test_non_finite_inputs_propagate_and_leave_the_plan_usable():
    nside, lmax = 16, 24
    rng = np.random.default_rng(9)
    K = jhtb.alm_size(lmax)
    a = rng.standard_normal(K) + 1j * rng.standard_normal(K)
    a[: lmax + 1] = a[: lmax + 1].real
    bad = a.copy()
    bad[jhtb.alm_size(lmax) - 1] = np.nan  # (l, m) = (lmax, lmax): every ring carries it
    m_bad = jhtb.synthesis(bad, nside, lmax, 0).cpu().numpy()
    assert np.isnan(m_bad).any()
    v = rng.standard_normal(12 * nside * nside)
    v[0] = np.inf
    b_bad = jhtb.adjoint_synthesis(v, nside, lmax, 0).cpu().numpy()
    assert not np.isfinite(b_bad).all()
    # the same plan still gives finite, correct results
    from oracle import jht_oracle as O

    got = jhtb.synthesis(a, nside, lmax, 0).cpu().numpy()
    ref = O.synthesis(a, nside, lmax, 0)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= 1e-12


def test_unsatisfiable_device_allocation_raises_memory_error():
    with pytest.raises(MemoryError):
        _lib.Plan(64, 128, 0, "fp64", max_batch=10_000_000)  # ~5 TB of ring spectra
    torch.cuda.synchronize()
    a = torch.zeros(jhtb.alm_size(12), dtype=torch.complex128, device="cuda")
    a[0] = 1.0
    m = jhtb.synthesis(a, 8, 12, 0)
    assert torch.allclose(m, torch.full_like(m, 1.0 / np.sqrt(4 * np.pi)), rtol=0, atol=1e-15)
