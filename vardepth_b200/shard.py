"""Sharding a region batch over GPUs: one process per GPU, no data-path collective.

Regions are independent, so each rank scores a disjoint set of regions on its
own GPU with its own persistent queue, and the results land in disjoint
slices of the full output vector.  Regions go to ranks longest-processing-time
first by DP cells (sum of n*m over the region's pairs), which balances the
ranks' kernel time.  Only when one rank must hold every result does a single
gather run at the end (torch.distributed: NCCL between GPUs, gloo on CPUs).
"""
from __future__ import annotations

import heapq

import numpy as np

from . import native


def region_cells(packed: native.Packed) -> np.ndarray:
    """DP cells of every region of a region-form batch."""
    rl = np.diff(packed.read_off)
    hl = np.diff(packed.hap_off)
    rsum = np.concatenate([[0], np.cumsum(rl)])
    hsum = np.concatenate([[0], np.cumsum(hl)])
    rr, hh = packed.region_read_off, packed.region_hap_off
    return (rsum[rr[1:]] - rsum[rr[:-1]]) * (hsum[hh[1:]] - hsum[hh[:-1]])


def shard_regions(cells: np.ndarray, world: int) -> list[np.ndarray]:
    """Longest-processing-time assignment of regions to ranks; each rank's regions in input order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(-np.asarray(cells), kind="stable")
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(order), np.int64)
    for g in order:
        load, r = heapq.heappop(heap)
        owner[g] = r
        heapq.heappush(heap, (load + int(cells[g]), r))
    return [np.flatnonzero(owner == r) for r in range(world)]


def subset(packed: native.Packed, regions: np.ndarray):
    """The batch restricted to `regions` (in that order) and, for each of its outputs, the
    position of that output in the full batch's output vector."""
    regions = np.asarray(regions, np.int64)
    rr, hh = packed.region_read_off, packed.region_hap_off
    nout = np.diff(rr) * np.diff(hh)
    out0 = np.concatenate([[0], np.cumsum(nout)])
    rb, rq, hb, ro, ho, pos = [], [], [], [0], [0], []
    rro, rho = [0], [0]
    for g in regions:
        r0, r1, h0, h1 = rr[g], rr[g + 1], hh[g], hh[g + 1]
        a, b = packed.read_off[r0], packed.read_off[r1]
        rb.append(packed.read_bases[a:b])
        rq.append(packed.read_quals[a:b])
        ro.extend((packed.read_off[r0 + 1:r1 + 1] - a + ro[-1]).tolist())
        c, d = packed.hap_off[h0], packed.hap_off[h1]
        hb.append(packed.hap_bases[c:d])
        ho.extend((packed.hap_off[h0 + 1:h1 + 1] - c + ho[-1]).tolist())
        rro.append(rro[-1] + (r1 - r0))
        rho.append(rho[-1] + (h1 - h0))
        pos.append(np.arange(out0[g], out0[g + 1]))
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.empty(0, dt)
    sub = native.Packed(cat(rb, np.uint8), cat(rq, np.uint8), ro, cat(hb, np.uint8), ho,
                        region_read_off=rro, region_hap_off=rho)
    return sub, cat(pos, np.int64)


def score_sharded(packed: native.Packed, rank: int, world: int, scorer, gather: bool = True, group=None):
    """Score this rank's shard with ``scorer(sub_packed) -> ln L`` (normally
    ``lambda p: engine.forward(p, params)[0]`` on this rank's GPU).

    Returns (positions, values) of this rank's outputs; with gather=True rank 0
    instead receives the full output vector (other ranks get None) through one
    torch.distributed gather_object at the end.
    """
    shards = shard_regions(region_cells(packed), world)
    sub, pos = subset(packed, shards[rank])
    values = np.asarray(scorer(sub), np.float64) if len(pos) else np.empty(0)
    if not gather or world == 1:
        if world == 1 and gather:
            full = np.empty(packed.n_outputs())
            full[pos] = values
            return full
        return pos, values
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object((pos, values), parts, dst=0, group=group)
    if rank != 0:
        return None
    full = np.empty(packed.n_outputs())
    for p, v in parts:
        full[p] = v
    return full
