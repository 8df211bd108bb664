"""The autotuner's search and its whole-batch confirmation, on the CPU with a scripted engine
(kernel times from a cost model, no device)."""
import numpy as np

from vardepth_b200 import autotune


class _Batch:
    def __init__(self, regions):
        self.read_off = np.arange(0, 10 * regions + 1, 10, dtype=np.int64)
        self.hap_off = np.arange(0, 100 * regions + 1, 100, dtype=np.int64)
        self.region_read_off = np.arange(regions + 1, dtype=np.int64)
        self.region_hap_off = np.arange(regions + 1, dtype=np.int64)


class _Engine:
    """tuning()/set_tuning()/plan()/info() of native.Engine; a plan's kernel time is
    cost(batch, tuning)."""

    def __init__(self, cost):
        self.cost = cost
        self.t = dict(autotune.DEFAULT, pipeline_gcells=0)
        self.timed = []

    def info(self):
        return {"gpu": "scripted"}

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **kw):
        self.t = dict(kw)

    def plan(self, batch, params):
        eng, setting = self, dict(self.t)

        class _Plan:
            def run(self):
                eng.timed.append((batch, setting))
                return type("St", (), {"kernel_ms": eng.cost(batch, setting)})()

            def close(self):
                pass

        return _Plan()


class _Params:
    anchored = 0


def _run(monkeypatch, whole_prefers_default):
    sample, whole = _Batch(20), _Batch(1000)
    monkeypatch.setattr(autotune, "split_samples", lambda packed: (sample, None))

    def cost(batch, t):
        if batch is sample:   # on the sample, the single-read kernel looks faster
            return 6.0 if t["pair_mask"] == 0 else 8.0
        if whole_prefers_default:
            return 290.0 if t["pair_mask"] == 0 else 211.0
        return 190.0 if t["pair_mask"] == 0 else 211.0

    eng = _Engine(cost)
    best = autotune.autotune(eng, whole, _Params(), repeats=1, use_cache=False, stratify=True, confirm=True)
    return eng, best


def test_a_sample_choice_the_whole_batch_rejects_is_dropped(monkeypatch):
    eng, best = _run(monkeypatch, whole_prefers_default=True)
    assert best["whole_batch"] == {"batch_ms_default": 211.0, "batch_ms_chosen": 290.0, "kept": "default"}
    assert {k: best[k] for k in autotune.DEFAULT} == autotune.DEFAULT
    assert {k: eng.tuning()[k] for k in autotune.DEFAULT} == autotune.DEFAULT
    # the long-read knobs were not timed (no long-read sample); the whole batch was timed twice
    assert sum(1 for b, _ in eng.timed if b.region_read_off[-1] == 1000) == 4  # capture + one run, each setting


def test_a_sample_choice_the_whole_batch_confirms_is_kept(monkeypatch):
    eng, best = _run(monkeypatch, whole_prefers_default=False)
    assert best["whole_batch"]["kept"] == "chosen" and best["pair_mask"] == 0
    assert eng.tuning()["pair_mask"] == 0


def test_no_confirmation_when_the_default_wins(monkeypatch):
    sample, whole = _Batch(20), _Batch(1000)
    monkeypatch.setattr(autotune, "split_samples", lambda packed: (sample, None))
    eng = _Engine(lambda batch, t: 5.0)
    best = autotune.autotune(eng, whole, _Params(), repeats=1, use_cache=False, stratify=True, confirm=True)
    assert best["whole_batch"] is None
    assert all(b is sample for b, _ in eng.timed)
