"""The allocation-free synthesis entry point (jhtb_synthesis_noalloc) through the C ABI.

Some callers cannot call cudaMalloc (a host framework or plugin that owns every
device allocation, or a process whose device memory is already reserved), so the
library offers one synthesis whose only scratch is a fixed array compiled into it.
This file is named to be collected last: it checks that entry point against the
plan-based jhtb_synthesis on two calls in a row (different sizes, so the second
call runs over the first call's leftover scratch), and that oversize requests are
refused.  It passes alone in a fresh process and after the rest of the suite.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU hosts
    pytest.skip("no CUDA device", allow_module_level=True)

from jht_b200 import _lib  # noqa: E402

TOL = 1e-12


def _alm(rng, lmax):
    K = (lmax + 1) * (lmax + 2) // 2
    a = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / np.sqrt(2)
    a[: lmax + 1] = a[: lmax + 1].real
    return torch.as_tensor(a, device="cuda")


def _plan_synthesis(alm, nside, lmax):
    plan = _lib.Plan(nside, lmax, 0, "fp64", 1)
    out = torch.empty(12 * nside * nside, dtype=torch.float64, device="cuda")
    _lib.check(plan.lib.jhtb_synthesis(plan.handle, alm.data_ptr(), out.data_ptr(), 1, _lib.stream_ptr()),
               "jhtb_synthesis")
    torch.cuda.synchronize()
    plan.close()
    return out


def _noalloc_synthesis(alm, nside, lmax):
    lib = _lib.load_library()
    out = torch.full((12 * nside * nside,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(lib.jhtb_synthesis_noalloc(nside, lmax, ctypes.c_void_p(alm.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), _lib.stream_ptr()),
               "jhtb_synthesis_noalloc")
    torch.cuda.synchronize()
    return out


# (nside, lmax) pairs, run back to back so each call overwrites the previous call's
# scratch: the headline CPU case, a small one, the largest lmax the scratch holds at
# nside 32 (deep underflow at high m, so the scaled start and its rescales run), the
# smallest grid with lmax 0, and lmax far above the ring lengths (m mod N folds).
CASES = ((64, 128), (8, 12), (32, 1023), (1, 0), (2, 40))


def test_noalloc_matches_plan_synthesis_twice():
    rng = np.random.default_rng(2024)
    for _ in range(2):
        for nside, lmax in CASES:
            a = _alm(rng, lmax)
            ref = _plan_synthesis(a, nside, lmax)
            got = _noalloc_synthesis(a, nside, lmax)
            err = float(torch.max(torch.abs(got - ref)) / torch.max(torch.abs(ref)))
            assert err <= TOL, (nside, lmax, err)


def test_noalloc_matches_golden(golden):
    """The reference's own synthesis at nside 64, lmax 128 (the CPU-runnable headline case)."""
    a = torch.as_tensor(golden["s0_n64_l128/alm"], device="cuda")
    got = _noalloc_synthesis(a, 64, 128).cpu().numpy()
    ref = golden["s0_n64_l128/map"]
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= TOL


def test_noalloc_rejects_oversize():
    lib = _lib.load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert lib.jhtb_synthesis_noalloc(128, 16, p, p, None) == _lib.JHTB_ERR_INVALID
    assert "nside" in _lib.last_error()
    assert lib.jhtb_synthesis_noalloc(64, 600, p, p, None) == _lib.JHTB_ERR_INVALID
    assert "scratch" in _lib.last_error()
