"""Host logic of the ring-pair sharding over devices (CPU, gloo, world size 2).

The GPU kernels cannot run here, so each gloo rank evaluates its share with the
oracle: the synthesis restricted to the rank's ring pixels, and the adjoint of the
map restricted to them (S^T is linear in the map, so the shares sum to S^T v).  The
partition, the pixel blocks and the all-reduce that combines the shares are the
product's own code (jht_b200.distributed).
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import relerr

from jht_b200 import distributed as D  # noqa: E402
from oracle import jht_oracle as O  # noqa: E402


def test_partition_is_contiguous_and_balanced():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        costs = rng.uniform(1, 10, size=37)
        parts = D.ring_partition(costs, world)
        assert parts[0][0] == 0 and parts[-1][1] == costs.size
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        loads = [costs[g0:g1].sum() for g0, g1 in parts]
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9


def test_partition_bound_on_skewed_costs():
    """The load bound (total/world + the largest granule) also for heavy-tailed and rising
    costs (the polar-to-equator ring profile), and with one granule outweighing the rest."""
    rng = np.random.default_rng(1)
    for it in range(3000):
        n, world = int(rng.integers(1, 60)), int(rng.integers(1, 12))
        costs = rng.pareto(1.5, n) + 0.01 if it % 2 else np.linspace(1.0, 3.0, n) ** 2
        parts = D.ring_partition(costs, world)
        assert parts[0][0] == 0 and parts[-1][1] == n
        assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(parts, parts[1:]))
        assert max(costs[g0:g1].sum() for g0, g1 in parts) <= (costs.sum() / world + costs.max()) * (1 + 1e-12)
    parts = D.ring_partition([1.0, 1.0, 1.0, 100.0], 4)
    assert max(sum([1.0, 1.0, 1.0, 100.0][g0:g1]) for g0, g1 in parts) == 100.0


def test_partition_of_few_granules_leaves_ranks_idle():
    parts = D.ring_partition([1.0, 1.0], 4)
    assert [p for p in parts if p[1] > p[0]] == [(0, 1), (1, 2)]


@pytest.mark.parametrize("nside", [1, 4, 13, 64])
def test_pixel_blocks_cover_the_map_once(nside):
    T = 2 * nside
    cover = np.zeros(12 * nside * nside, dtype=int)
    cuts = sorted({0, T, *np.linspace(0, T, 5).astype(int).tolist()})
    for t0, t1 in zip(cuts, cuts[1:]):
        for p0, p1 in D.ring_pixel_blocks(nside, t0, t1):
            cover[p0:p1] += 1
    assert np.all(cover == 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, nside, lmax, spin, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(11)
        K = O.alm_size(lmax)
        ells, _ = O.lm_of_index(lmax)
        shape = (K,) if spin == 0 else (2, K)
        a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / (ells + 3.0)
        a[..., : lmax + 1] = a[..., : lmax + 1].real
        if spin == 2:
            a[..., ells < 2] = 0
        npix = 12 * nside * nside
        v = rng.standard_normal((npix,) if spin == 0 else (2, npix))
        # equal per-ring costs at a granule of 2 rings (the plan supplies real costs on GPUs)
        T = 2 * nside
        t0, t1 = D.ring_ranges(nside, np.ones((T + 1) // 2), world, granule=2)[rank]
        mask = np.zeros(npix)
        for p0, p1 in D.ring_pixel_blocks(nside, t0, t1):
            mask[p0:p1] = 1.0
        ranges = D.ring_ranges(nside, np.ones((T + 1) // 2), world, granule=2)
        # this rank's rings, the other pixels filled with junk the gather must ignore
        mine = np.where(mask > 0, O.synthesis(a, nside, lmax, spin), 1e30)
        full_map = D.gather_pixel_blocks(torch.as_tensor(mine), nside, ranges, rank)
        part = O.adjoint_synthesis(v * (mask if spin == 0 else mask[None, :]), nside, lmax, spin)
        full_adj = D.all_reduce_sum(torch.as_tensor(part))
        if rank == 0:
            q.put((relerr(full_map.numpy(), O.synthesis(a, nside, lmax, spin)),
                   relerr(full_adj.numpy(), O.adjoint_synthesis(v, nside, lmax, spin)), (t0, t1)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spin", [0, 2])
def test_two_rank_shards_sum_to_the_full_transforms(spin):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, nside, lmax = 2, 8, 12
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nside, lmax, spin, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    err_map, err_adj, rng0 = q.get(timeout=10)
    assert rng0[0] == 0 and 0 < rng0[1] < 2 * nside  # both ranks own rings
    assert err_map <= 1e-14
    assert err_adj <= 1e-13

