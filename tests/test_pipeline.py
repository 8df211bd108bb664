"""The actor pipeline (the message protocol of gpu_evidence_pipeline.py:74-122) with
asynchronous batch scoring, on the CPU: spawned actors, generator tasks, batching by mode and
max_pairs, results in task order, errors raised in the parent with no actor left behind.  The
oracle stands in for the GPU scorer."""
import multiprocessing as mp
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from vardepth_b200 import pipeline


def _pairs(seed, k):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        m = int(rng.integers(20, 60))
        hap = "".join(rng.choice(list("ACGT"), m))
        a = int(rng.integers(0, m - 15))
        read = hap[a:a + 15]
        out.append((read, [30] * len(read), hap))
    return out


def task(payload):
    """Two rounds of requests (semiglobal, then anchored), returning the sums of the likelihoods."""
    seed, k = payload
    first = yield False, _pairs(seed, k)
    second = yield True, _pairs(seed + 1000, k // 2 + 1)
    return seed, float(np.sum(first)), float(np.sum(second))


def failing(payload):
    yield False, _pairs(payload, 2)
    raise ValueError("boom")


def dying(payload):
    yield False, _pairs(payload, 1)
    os._exit(3)


def counting(n):
    """A task of integer 'pairs' whose value the counting scorer doubles (semiglobal) or
    triples (anchored): n requests of alternating mode with n+1 .. 1 pairs."""
    total = 0
    for i in range(n):
        values = yield bool(i % 2), [n] * (n - i + 1)
        total += int(np.sum(values))
    return n, total


def scorer(requests, anchored):
    return np.array([O.forward(s, np.asarray(q, np.uint8), h, 0.001, 0.1, anchored) for s, q, h in requests])


def test_results_follow_task_order_and_match_direct_scoring():
    tasks = [(s, 3 + s % 5) for s in range(12)]
    got = pipeline.run_tasks(tasks, task, workers=2, slots_per_worker=3, max_pairs=8, scorer=scorer)
    want = [(s, float(np.sum(scorer(_pairs(s, k), False))), float(np.sum(scorer(_pairs(s + 1000, k // 2 + 1), True))))
            for s, k in tasks]
    assert [g[0] for g in got] == [w[0] for w in want]
    np.testing.assert_allclose(np.array([g[1:] for g in got]), np.array([w[1:] for w in want]), rtol=1e-12)


def test_batches_respect_max_pairs_and_modes():
    batches = []

    def counting_scorer(jobs, anchored):
        batches.append((len(jobs), anchored))
        return np.asarray(jobs, np.float64) * (3 if anchored else 2)

    tasks = list(range(1, 9))
    got = pipeline.run_tasks(tasks, counting, workers=3, slots_per_worker=2, max_pairs=6, scorer=counting_scorer)
    want = [(n, sum(n * (n - i + 1) * (3 if i % 2 else 2) for i in range(n))) for n in tasks]
    assert got == want
    assert {a for _, a in batches} == {False, True}
    # a batch is whole requests up to max_pairs, or one larger request alone (at most 9 pairs here)
    assert all(n <= 9 for n, _ in batches)
    assert sum(n for n, _ in batches) == sum(sum(n - i + 1 for i in range(n)) for n in tasks)


def test_empty_task_list_and_bad_bounds():
    assert pipeline.run_tasks([], task, workers=1, scorer=scorer) == []
    for bad in (dict(workers=0), dict(slots_per_worker=0), dict(max_pairs=0)):
        with pytest.raises(ValueError):
            pipeline.run_tasks([], task, scorer=scorer, **bad)


def test_worker_errors_reach_the_parent_and_no_actor_survives():
    before = {p.pid for p in mp.active_children()}
    with pytest.raises(RuntimeError, match="boom"):
        pipeline.run_tasks([1, 2, 3, 4], failing, workers=2, slots_per_worker=2, scorer=scorer)
    assert {p.pid for p in mp.active_children()} == before


def test_an_actor_that_exits_is_detected():
    before = {p.pid for p in mp.active_children()}
    with pytest.raises(RuntimeError, match="exited"):
        pipeline.run_tasks([1, 2], dying, workers=1, scorer=scorer)
    assert {p.pid for p in mp.active_children()} == before


def test_scorer_shape_is_checked():
    before = {p.pid for p in mp.active_children()}
    with pytest.raises(ValueError, match="wrong shape"):
        pipeline.run_tasks([(1, 3)], task, workers=1, scorer=lambda r, a: np.zeros(len(r) + 1))
    assert {p.pid for p in mp.active_children()} == before


REFERENCE_CALLER = Path(os.environ.get("VARDEPTH_REFERENCE", "/root/reference")) / "caller" / "native" / "caller"


@pytest.mark.skipif(not (REFERENCE_CALLER / "gpu_evidence_pipeline.py").exists(),
                    reason="the reference sources are not present on this machine")
def test_the_reference_actor_runs_under_this_loop():
    """The reference's own actor function (gpu_evidence_pipeline._actor, with no BAM arguments)
    speaks the protocol this loop serves."""
    sys.path.insert(0, str(REFERENCE_CALLER))  # the spawned actors import it too
    try:
        import gpu_evidence_pipeline as ref
        tasks = [(s, 2 + s % 3) for s in range(6)]
        got = pipeline.run_tasks(tasks, task, workers=2, slots_per_worker=2, max_pairs=5, scorer=scorer,
                                 actor_target=ref._actor, actor_args=(None, None))
    finally:
        sys.path.remove(str(REFERENCE_CALLER))
    for (seed, a, b), (s, k) in zip(got, tasks):
        assert seed == s
        assert a == pytest.approx(float(np.sum(scorer(_pairs(s, k), False))), rel=1e-12)
        assert b == pytest.approx(float(np.sum(scorer(_pairs(s + 1000, k // 2 + 1), True))), rel=1e-12)


@pytest.mark.gpu
def test_pipeline_with_the_gpu_scorer():
    tasks = [(s, 4) for s in range(8)]
    got = pipeline.run_tasks(tasks, task, workers=2, slots_per_worker=2, max_pairs=16)
    for (seed, a, b), (s, k) in zip(got, tasks):
        assert seed == s
        assert abs(a - float(np.sum(scorer(_pairs(s, k), False)))) < 1e-3
        assert abs(b - float(np.sum(scorer(_pairs(s + 1000, k // 2 + 1), True)))) < 1e-3
