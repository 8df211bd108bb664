"""Sharding a region batch over GPUs: one process per GPU, no data-path collective.

Regions are independent, so each rank scores a disjoint set of regions on its
own GPU with its own persistent queue, and the results land in disjoint
slices of the full output vector.  Regions go to ranks longest-processing-time
first by DP cells (sum of n*m over the region's pairs), which balances the
ranks' kernel time.  On one node the full output vector is a shared-memory
array that every rank writes its slices of (``SharedOutput``), so rank 0 holds
every result after one barrier and no result crosses a collective; across
nodes a single gather at the end collects them (torch.distributed: NCCL
between GPUs, gloo on CPUs).
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


class SharedOutput:
    """The full output vector (float64) in POSIX shared memory, one per node: each rank
    writes the slices of its regions and rank 0 reads the whole vector after a barrier.
    Rank 0 creates the segment (``name``) before the others attach."""

    def __init__(self, name: str, n: int, create: bool):
        from multiprocessing import resource_tracker, shared_memory
        size = max(8, 8 * int(n))
        if create:
            try:  # a segment left by an earlier run under the same name
                old = shared_memory.SharedMemory(name=name)
                old.close()
                old.unlink()
            except FileNotFoundError:
                pass
            self.shm = shared_memory.SharedMemory(name=name, create=True, size=size)
        else:
            self.shm = shared_memory.SharedMemory(name=name)
            # the creator unlinks it; this rank's resource tracker must not
            resource_tracker.unregister(self.shm._name, "shared_memory")
        self.creator = create
        self.values = np.ndarray((int(n),), np.float64, buffer=self.shm.buf)

    def write(self, positions: np.ndarray, values: np.ndarray) -> None:
        self.values[positions] = values

    def close(self) -> None:
        self.values = None
        self.shm.close()
        if self.creator:
            self.shm.unlink()


def score_sharded(packed: native.Packed, rank: int, world: int, scorer, gather: bool = True, group=None,
                  shared_name: str | None = None):
    """Score this rank's shard with ``scorer(sub_packed) -> ln L`` (normally
    ``lambda p: engine.forward(p, params)[0]`` on this rank's GPU).

    Returns (positions, values) of this rank's outputs.  With gather=True rank 0 instead
    receives the full output vector (other ranks get None): through the node's shared-memory
    array when ``shared_name`` is given (every rank writes its slices, then one barrier), else
    through one torch.distributed gather_object at the end (ranks on several nodes).
    """
    shards = shard_regions(region_cells(packed), world)
    sub, pos = subset(packed, shards[rank])
    values = np.asarray(scorer(sub), np.float64) if len(pos) else np.empty(0)
    if not gather:
        return pos, values
    if world == 1:
        full = np.empty(packed.n_outputs())
        full[pos] = values
        return full
    import torch.distributed as dist
    if shared_name is not None:
        if rank == 0:
            out = SharedOutput(shared_name, packed.n_outputs(), create=True)
        dist.barrier(group=group)          # the segment exists
        if rank != 0:
            out = SharedOutput(shared_name, packed.n_outputs(), create=False)
        out.write(pos, values)
        dist.barrier(group=group)          # every slice is written
        full = out.values.copy() if rank == 0 else None
        dist.barrier(group=group)          # rank 0 has read it
        out.close()
        return full
    parts = [None] * world if rank == 0 else None
    dist.gather_object((pos, values), parts, dst=0, group=group)
    if rank != 0:
        return None
    full = np.empty(packed.n_outputs())
    for p, v in parts:
        full[p] = v
    return full
