"""Ring-pair shards of the transforms on one B200 (needs a GPU).

Plans restricted to half-grid ring ranges (the per-device shares of a multi-GPU
run) are evaluated one after another on the same device: the shard maps cover
disjoint pixels and sum to the full synthesis, the shard adjoints sum to the full
adjoint, for the FP64 kernels and the tensor-core synthesis.
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
from jht_b200 import _lib  # noqa: E402
from jht_b200 import distributed as D  # noqa: E402


def _inputs(nside, lmax, spin, B, seed):
    rng = np.random.default_rng(seed)
    K = jhtb.alm_size(lmax)
    ells = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    nc = 1 if spin == 0 else 2
    a = (rng.standard_normal((B, nc, K)) + 1j * rng.standard_normal((B, nc, K))) / (ells + 10.0)
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    if spin == 2:
        a[..., ells < 2] = 0
    v = rng.standard_normal((B, nc, 12 * nside * nside))
    return torch.as_tensor(a, device="cuda"), torch.as_tensor(v, device="cuda")


@pytest.mark.parametrize("nside,lmax,cuts", [(256, 384, (0, 256, 512)), (512, 700, (0, 256, 768, 1024))])
@pytest.mark.parametrize("spin", [0, 2])
def test_fp64_shards_sum_to_full(nside, lmax, cuts, spin):
    a, v = _inputs(nside, lmax, spin, 2, nside + spin)
    full = D.ShardedTransform(nside, lmax, spin, max_batch=2)
    ref_s = full.synthesis(a)
    ref_a = full.adjoint_synthesis(v)
    s_sum = torch.zeros_like(ref_s)
    a_sum = torch.zeros_like(ref_a)
    for t0, t1 in zip(cuts, cuts[1:]):
        sh = D.ShardedTransform(nside, lmax, spin, max_batch=2, ring_range=(t0, t1))
        part = sh.synthesis(a, gather=False)
        blocks = D.ring_pixel_blocks(nside, t0, t1)
        inside = torch.zeros(12 * nside * nside, dtype=torch.bool, device="cuda")
        for p0, p1 in blocks:
            inside[p0:p1] = True
        assert float(torch.max(torch.abs(part[..., ~inside]))) == 0.0  # only its own rings
        s_sum += part
        a_sum += sh.adjoint_synthesis(v)
        sh.close()
    assert relerr(s_sum.cpu().numpy(), ref_s.cpu().numpy()) == 0.0
    assert relerr(a_sum.cpu().numpy(), ref_a.cpu().numpy()) <= 1e-13
    # the unsharded transform agrees with the public API
    assert relerr(ref_s[0].cpu().numpy(), jhtb.synthesis(a[0] if spin else a[0, 0], nside, lmax, spin).cpu().numpy().reshape(ref_s[0].shape)) == 0.0
    full.close()


@pytest.mark.parametrize("spin", [0, 2])
def test_tensor_core_shards_sum_to_full(spin):
    nside, lmax = 256, 384
    a, _ = _inputs(nside, lmax, spin, 8, 5 + spin)
    full = D.ShardedTransform(nside, lmax, spin, precision="bf16x3", max_batch=8)
    ref = full.synthesis(a)
    acc = torch.zeros_like(ref)
    for t0, t1 in ((0, 256), (256, 512)):
        sh = D.ShardedTransform(nside, lmax, spin, precision="bf16x3", max_batch=8, ring_range=(t0, t1))
        acc += sh.synthesis(a, gather=False)
        assert sh.plan.status() == 0
        sh.close()
    assert relerr(acc.cpu().numpy(), ref.cpu().numpy()) == 0.0
    full.close()


def test_balanced_ranges_from_plan_costs():
    plan = _lib.Plan(512, 1024, 2, "fp64", 1)
    costs = plan.ring_costs(D.GRANULE)
    assert costs.size == 4 and np.all(costs > 0)
    ranges = D.ring_ranges(512, costs, 2)
    assert ranges[0][0] == 0 and ranges[-1][1] == 1024 and ranges[0][1] == ranges[1][0]
    plan.close()


def test_invalid_ring_range_is_rejected():
    plan = _lib.Plan(256, 384, 0, "fp64", 1)
    with pytest.raises(ValueError, match="multiples of 256"):
        plan.set_ring_range(100, 512)
    with pytest.raises(ValueError):
        plan.set_ring_range(256, 256)
    plan.close()
