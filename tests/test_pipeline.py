"""The actor pipeline (gpu_evidence_pipeline.py:74-122 protocol) with asynchronous batch scoring,
on the CPU: spawned actors, generator tasks, batching by mode and max_pairs, results in task
order, and errors raised in the parent.  The oracle stands in for the GPU scorer."""
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


def scorer(requests, anchored):
    return np.array([O.forward(s, np.asarray(q, np.uint8), h, 0.001, 0.1, anchored) for s, q, h in requests])


def test_results_follow_task_order_and_match_direct_scoring():
    tasks = [(s, 3 + s % 5) for s in range(12)]
    got = pipeline.run_tasks(tasks, task, workers=2, slots_per_worker=3, max_pairs=8, scorer=scorer)
    want = [(s, float(np.sum(scorer(_pairs(s, k), False))), float(np.sum(scorer(_pairs(s + 1000, k // 2 + 1), True))))
            for s, k in tasks]
    assert [g[0] for g in got] == [w[0] for w in want]
    np.testing.assert_allclose(np.array([g[1:] for g in got]), np.array([w[1:] for w in want]), rtol=1e-12)


def test_empty_task_list_and_bad_bounds():
    assert pipeline.run_tasks([], task, workers=1, scorer=scorer) == []
    with pytest.raises(ValueError):
        pipeline.run_tasks([(1, 2)], task, workers=0, scorer=scorer)


def test_worker_errors_reach_the_parent():
    with pytest.raises(RuntimeError, match="boom"):
        pipeline.run_tasks([1, 2], failing, workers=1, scorer=scorer)


def test_scorer_shape_is_checked():
    with pytest.raises(ValueError, match="wrong shape"):
        pipeline.run_tasks([(1, 3)], task, workers=1, scorer=lambda r, a: np.zeros(len(r) + 1))


@pytest.mark.gpu
def test_pipeline_with_the_gpu_scorer():
    tasks = [(s, 4) for s in range(8)]
    got = pipeline.run_tasks(tasks, task, workers=2, slots_per_worker=2, max_pairs=16)
    for (seed, a, b), (s, k) in zip(got, tasks):
        assert seed == s
        assert abs(a - float(np.sum(scorer(_pairs(s, k), False)))) < 1e-3
        assert abs(b - float(np.sum(scorer(_pairs(s + 1000, k // 2 + 1), True)))) < 1e-3
