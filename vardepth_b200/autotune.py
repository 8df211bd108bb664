"""Autotuner of the batched schedule's work-list choices (vd_tuning).

The persistent kernels are fixed; what depends on the workload is how the host
lays out the work list:

* ``long_read_rows``  strip height of reads longer than 256 bases (64, 128,
  256).  Each strip boundary is renormalised by an exact power of two, so
  shorter strips keep error-rich long reads inside the FP32 range (fewer
  pairs handed to the FP64 tiers) at the price of more passes over the
  haplotype;
* ``pair_mask``  which rows-per-lane classes run two reads per warp in the
  packed FP32 kernel (fewer issue slots per cell, more registers per warp);
* ``pair_split``  the tile of the packed kernels: from how many rows per lane
  a two-read item runs on the 12-warp-per-SM kernel (168 registers) rather
  than the 16-warp kernel (128 registers, where 6 rows per lane spill a
  little);
* ``max_item_columns``  how many haplotype columns one work item streams
  (shorter items balance the tail of the persistent queue, longer ones pay
  the 31-step wavefront ramp less often);
* ``long_mode``  how reads longer than one strip run: the warp-per-pair or
  block-per-pair split -- a read against two haplotypes per warp with
  per-lane power-of-two boosts (``VD_LONG_WARP``), the same items on a whole
  CTA whose warps split each strip (``VD_LONG_BLOCK``: more parallelism per
  pair, for batches of few long pairs), or one pair per warp in the
  single-read kernel with exact strip renormalisation and the drift tier
  behind it (``VD_LONG_SINGLE``).

``autotune`` times candidate settings with resident plans (CUDA events around
the captured tier graph) on a seeded region sample of the caller's batch,
coordinate by coordinate, and leaves the best setting on the engine.  Results
are cached per (device name, sample signature) in a JSON file.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

from . import native

DEFAULT = {"long_read_rows": 256, "pair_mask": 0x1FE, "max_item_columns": 0, "long_mode": native.VD_LONG_WARP,
           "pair_split": 6}
SPACE = {
    "pair_split": [6, 7],
    "long_mode": [native.VD_LONG_WARP, native.VD_LONG_BLOCK, native.VD_LONG_SINGLE],
    "long_read_rows": [256, 128, 64],
    "pair_mask": [0x1FE, 0x1F0, 0],
    "max_item_columns": [0, 16384, 4096],
}
CACHE = Path(os.environ.get("VARDEPTH_TUNING_CACHE", Path.home() / ".cache" / "vardepth_b200" / "tuning.json"))


def sample_regions(region_read_off, region_hap_off, fraction: float = 0.02, min_regions: int = 200,
                   seed: int = 2024) -> np.ndarray:
    """A seeded random subset of the regions (in input order)."""
    n = len(region_read_off) - 1
    k = min(n, max(min_regions, int(round(fraction * n))))
    return np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False))


def signature(read_off, hap_off) -> str:
    """Coarse description of a batch's shape: read and haplotype length classes."""
    n = np.diff(np.asarray(read_off))
    m = np.diff(np.asarray(hap_off))
    rb = np.histogram(n, bins=[0, 33, 65, 129, 257, 1025, 1 << 30])[0]
    hb = np.histogram(m, bins=[0, 257, 1025, 4097, 1 << 30])[0]
    f = lambda h: ",".join(f"{x / max(1, h.sum()):.2f}" for x in h)
    return f"reads[{f(rb)}] haps[{f(hb)}]"


def _apply(engine: native.Engine, setting: dict) -> None:
    """Set the tuned knobs, keeping the engine's other tuning fields."""
    engine.set_tuning(**dict(engine.tuning(), **{k: setting[k] for k in DEFAULT}))


def _time(engine: native.Engine, packed: native.Packed, params, setting: dict, repeats: int) -> float:
    _apply(engine, setting)
    plan = engine.plan(packed, params)
    try:
        plan.run()  # captures the graph
        ms = [plan.run().kernel_ms for _ in range(repeats)]
    finally:
        plan.close()
    return float(np.median(ms))


def autotune(engine: native.Engine, packed: native.Packed, params, repeats: int = 3, use_cache: bool = True,
             log: list | None = None) -> dict:
    """Choose vd_tuning for this batch shape by timing candidates on ``packed`` (normally a sample
    of the real batch); the best setting stays on the engine and is returned."""
    key = f"{engine.info()['gpu']}|{signature(packed.read_off, packed.hap_off)}|anch={params.anchored}"
    cache = {}
    if use_cache and CACHE.exists():
        try:
            cache = json.loads(CACHE.read_text())
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        best = cache[key]
        _apply(engine, best)
        return dict(best, cached=True)
    best = dict(DEFAULT)
    best_ms = _time(engine, packed, params, best, repeats)
    trials = [(dict(best), best_ms)]
    for knob, values in SPACE.items():
        for v in values:
            if v == best[knob]:
                continue
            cand = dict(best, **{knob: v})
            ms = _time(engine, packed, params, cand, repeats)
            trials.append((cand, ms))
            if ms < best_ms * 0.99:
                best, best_ms = cand, ms
    _apply(engine, best)
    if log is not None:
        log.extend({"setting": t, "ms": round(ms, 3)} for t, ms in trials)
    if use_cache:
        cache[key] = best
        try:
            CACHE.parent.mkdir(parents=True, exist_ok=True)
            CACHE.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return dict(best, sample_ms=round(best_ms, 3), default_ms=round(trials[0][1], 3), cached=False)
