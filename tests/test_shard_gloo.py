"""The multi-GPU path on the CPU: regions sharded over world_size 2 gloo ranks (127.0.0.1),
each rank scoring its own shard (here with the oracle as a stand-in scorer: no GPU), and the
full output vector reassembled on rank 0 in the batch's output order, through the node's
shared-memory array (each rank writes its slices) or through one gather."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from vardepth_b200 import native, shard
from vardepth_b200 import synthetic as S


def _workload():
    w = S.batched_regions(n_regions=30, seed=5)
    return w, native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                            region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)


def _oracle_scorer(gap, ext):
    def score(p):
        pr, ph = O.region_pairs(p.region_read_off, p.region_hap_off)
        return O.forward_pairs(p.read_bases, p.read_quals, p.read_off, p.hap_bases, p.hap_off, pr, ph, gap, ext,
                               threads=2)
    return score


def _rank(rank, world, port, result_path, shared_name):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, packed = _workload()
        full = shard.score_sharded(packed, rank, world, _oracle_scorer(w.gap, w.ext), shared_name=shared_name)
        if rank == 0:
            np.save(result_path, full)
        else:
            assert full is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_lpt_shards_are_disjoint_and_balanced():
    w, packed = _workload()
    cells = shard.region_cells(packed)
    assert cells.sum() == w.cells()
    shards = shard.shard_regions(cells, 4)
    assert sorted(np.concatenate(shards).tolist()) == list(range(w.n_regions))
    loads = [cells[s].sum() for s in shards]
    assert max(loads) - min(loads) <= cells.max()


def test_subset_positions_cover_the_outputs():
    w, packed = _workload()
    parts = [shard.subset(packed, s) for s in shard.shard_regions(shard.region_cells(packed), 3)]
    pos = np.concatenate([p for _, p in parts])
    assert sorted(pos.tolist()) == list(range(packed.n_outputs()))
    assert sum(sub.n_outputs() for sub, _ in parts) == packed.n_outputs()


@pytest.mark.parametrize("shared", [True, False])
def test_two_gloo_ranks_reassemble_the_batch(tmp_path, shared):
    w, packed = _workload()
    result = tmp_path / "full.npy"
    name = f"vd_test_{os.getpid()}" if shared else None
    mp.start_processes(_rank, args=(2, _free_port(), str(result), name), nprocs=2, join=True, start_method="spawn")
    full = np.load(result)
    want = _oracle_scorer(w.gap, w.ext)(packed)
    np.testing.assert_array_equal(full, want)
    if shared:
        assert not os.path.exists(f"/dev/shm/{name}")  # rank 0 removed the segment
