"""On-grid transforms sharded over devices by ring pairs (torch.distributed).

jht runs on one device; this module is an extension.  Every half-grid ring t
(north cap and equator, t < 2 nside) and its southern mirror 4 nside - 2 - t are
independent in both directions of the transform, so the rings are split into
contiguous ranges, one per rank, balanced by the plan's own measure of Legendre
work (ring-recursion steps per group of 256 rings, which accounts for the
underflowed polar work the kernels skip):

* synthesis: each rank evaluates its rings from the full a_lm (no exchange); the
  map is assembled by one all-gather of every rank's own pixel blocks (each rank
  sends only its share of the map), or left sharded (``gather=False``);
* adjoint: each rank contracts its rings into a partial a_lm; one all-reduce (sum)
  gives S^T v.

Every rank holds the full inputs.  The collectives are torch.distributed
all-reduces on the default (or given) process group: NCCL over NVLink on B200
nodes, gloo on CPU for the host logic tested without a GPU.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .healpix import RingInfo, _check_spin, alm_size

__all__ = ["GRANULE", "ring_partition", "ring_ranges", "ring_pixel_blocks", "all_reduce_sum", "gather_pixel_blocks",
           "ShardedTransform"]

GRANULE = 256  # ring ranges are aligned to the tile widths of every kernel


def ring_partition(costs, world: int) -> list[tuple[int, int]]:
    """Split granules 0..len(costs)-1 into `world` contiguous ranges with near-equal total
    cost: boundary r sits at the prefix sum closest to r/world of the total, moved one
    granule past boundary r-1 if it would not advance (while granules remain).  No range
    costs more than total/world + the largest granule cost; a range can be empty (an idle
    rank) when one granule outweighs several shares.  Returns [(g0, g1), ...] in granule
    units."""
    c = np.asarray(costs, dtype=np.float64)
    n = c.size
    if world < 1:
        raise ValueError("world must be >= 1")
    pref = np.concatenate([[0.0], np.cumsum(np.maximum(c, 0.0) + 1e-9)])
    total = pref[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.argmin(np.abs(pref - target)))
        b = min(max(b, bounds[-1] + (1 if bounds[-1] < n else 0)), n)
        bounds.append(b)
    bounds.append(n)
    return [(bounds[r], max(bounds[r], bounds[r + 1])) for r in range(world)]


def ring_ranges(nside: int, costs, world: int, granule: int = GRANULE) -> list[tuple[int, int]]:
    """Half-grid ring ranges [t0, t1) per rank from per-granule costs."""
    T = 2 * nside
    out = []
    for g0, g1 in ring_partition(costs, world):
        out.append((min(g0 * granule, T), min(g1 * granule, T)))
    return out


def ring_pixel_blocks(nside: int, t0: int, t1: int) -> list[tuple[int, int]]:
    """RING-order pixel blocks [p0, p1) of half-grid rings [t0, t1) and their mirrors."""
    if t0 >= t1:
        return []
    geo = RingInfo(nside)
    T = 2 * nside
    start = np.concatenate([geo.startpix, [geo.npix]])
    blocks = [(int(start[t0]), int(start[t1]))]  # northern rings t0..t1-1 (equator included)
    tn = min(t1, T - 1)  # rings with a southern mirror
    if t0 < tn:
        r_lo, r_hi = 4 * nside - 1 - tn, 4 * nside - 1 - t0  # mirrors of t in [t0, tn)
        blocks.append((int(start[r_lo]), int(start[r_hi])))
    return blocks


def all_reduce_sum(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place sum over the ranks of `group` (no-op without an initialised process group)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        if t.is_complex():
            dist.all_reduce(torch.view_as_real(t), op=dist.ReduceOp.SUM, group=group)
        else:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def gather_pixel_blocks(local: torch.Tensor, nside: int, ranges, rank: int, group=None) -> torch.Tensor:
    """Assemble the full maps (..., npix) from every rank's own rings: rank r contributes the
    pixel blocks of its half-grid range ``ranges[r]`` (and their southern mirrors), packed
    into one buffer; one all-gather moves the packed buffers (padded to the largest share).
    ``local`` holds this rank's rings (other pixels are ignored).  Without an initialised
    process group (or with one rank) it returns ``local``."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1):
        return local
    world = dist.get_world_size(group)
    blocks = [ring_pixel_blocks(nside, t0, t1) for t0, t1 in ranges]
    sizes = [sum(p1 - p0 for p0, p1 in b) for b in blocks]
    nmax = max(max(sizes), 1)
    lead = local.shape[:-1]
    mine = [local[..., p0:p1] for p0, p1 in blocks[rank]]
    packed = torch.zeros(lead + (nmax,), dtype=local.dtype, device=local.device)
    if mine:
        cat = torch.cat(mine, dim=-1)
        packed[..., : cat.shape[-1]] = cat
    parts = [torch.empty_like(packed) for _ in range(world)]
    dist.all_gather(parts, packed.contiguous(), group=group)
    out = torch.zeros_like(local)
    for r in range(world):
        off = 0
        for p0, p1 in blocks[r]:
            out[..., p0:p1] = parts[r][..., off : off + (p1 - p0)]
            off += p1 - p0
    return out


class ShardedTransform:
    """S and S^T of one geometry with this rank's share of the rings.

    ``ring_range`` overrides the balanced split (half-grid rings [t0, t1), aligned
    to 256 rings); without a process group the whole grid is local.
    """

    def __init__(self, nside: int, lmax: int, spin: int = 0, precision: str = "fp64", max_batch: int = 1,
                 group=None, ring_range: tuple[int, int] | None = None):
        import torch.distributed as dist

        _check_spin(spin)
        self.nside, self.lmax, self.spin, self.precision = nside, lmax, spin, precision
        self.group = group
        dist_on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if dist_on else 0
        self.world = dist.get_world_size(group) if dist_on else 1
        self.plan = _lib.Plan(nside, lmax, spin, precision, max_batch)
        T = 2 * nside
        if ring_range is None:
            if self.world > 1:
                costs = self.plan.ring_costs(GRANULE)
                self.ranges = ring_ranges(nside, costs, self.world)
                ring_range = self.ranges[self.rank]
            else:
                ring_range = (0, T)
                self.ranges = [ring_range]
        else:
            # every rank's explicit range is needed to assemble the map: collect them
            self.ranges = [tuple(ring_range)] * self.world
            if self.world > 1:
                got = [None] * self.world
                dist.all_gather_object(got, tuple(ring_range), group=group)
                self.ranges = [tuple(r) for r in got]
        self.t0, self.t1 = ring_range
        if (self.t0, self.t1) != (0, T) and self.t0 < self.t1:
            self.plan.set_ring_range(self.t0, self.t1)
        self.ncomp = 1 if spin == 0 else 2
        self.npix = 12 * nside * nside
        self.K = alm_size(lmax)

    def _batched(self, x, last: int):
        t = x if x.dim() == 3 else x.reshape(1, self.ncomp, last)
        return t.contiguous()

    def synthesis(self, alm: torch.Tensor, gather: bool = True) -> torch.Tensor:
        """Map (B, ncomp, npix) of this rank's rings (zeros elsewhere), or with `gather` the whole
        map assembled from every rank's pixel blocks."""
        a = self._batched(alm.to(torch.complex128), self.K)
        B = a.shape[0]
        out = torch.zeros((B, self.ncomp, self.npix), dtype=torch.float64, device=a.device)
        if self.t0 < self.t1 and B:
            _lib.check(self.plan.lib.jhtb_synthesis(self.plan.handle, a.data_ptr(), out.data_ptr(), B, _lib.stream_ptr()),
                       "jhtb_synthesis")
        return gather_pixel_blocks(out, self.nside, self.ranges, self.rank, self.group) if gather else out

    def adjoint_synthesis(self, maps: torch.Tensor) -> torch.Tensor:
        """S^T maps (B, ncomp, K): this rank's rings contracted, summed over ranks."""
        m = self._batched(maps.to(torch.float64), self.npix)
        B = m.shape[0]
        out = torch.zeros((B, self.ncomp, self.K), dtype=torch.complex128, device=m.device)
        if self.t0 < self.t1 and B:
            _lib.check(self.plan.lib.jhtb_adjoint_synthesis(self.plan.handle, m.data_ptr(), out.data_ptr(), B,
                                                            _lib.stream_ptr()), "jhtb_adjoint_synthesis")
        return all_reduce_sum(out, self.group)

    def close(self) -> None:
        self.plan.close()
