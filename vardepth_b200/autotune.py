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
  behind it (``VD_LONG_SINGLE``);
* ``long_group``  haplotypes per warp item of a long read: the pairs after
  an item's first start each strip from the lane boosts the first pair
  measured, so larger items rerun fewer strips, smaller ones leave more items
  to balance the tail of a batch of few long reads.  It is not searched: the
  tail it trades against depends on how many long items the whole batch
  holds, which a sample does not show (on the mixed-length workload a 2%
  sample preferred 4 haplotypes per item, the 20,000-region batch runs 5%
  faster with 8).  The default (8) stays; a batch of few long reads is better
  served by the block or single-read path, which the search does cover.

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
           "pair_split": 6, "long_group": native.LONG_GROUP_MAX}
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


LONG_KNOBS = ("long_mode", "long_read_rows")     # act on reads longer than one strip only
SHORT_KNOBS = ("pair_split", "pair_mask", "max_item_columns")


def split_samples(packed: native.Packed, fraction: float = 0.02, min_regions: int = 200, long_items: int = 8192,
                  seed: int = 2024, short_items: int = 49152):
    """Two seeded region samples of a region-form batch: regions holding a read longer than one
    256-row strip ("long") and the others ("short").  The short sample is `fraction` of the short
    regions (at least `min_regions`), grown until it holds about `short_items` two-read items
    (half its reads); the long sample takes long regions until it holds about `long_items`
    read x haplotype-pair items.  Both fill every warp of the device many times over, because a
    persistent kernel's time on a few items per warp is its slowest warp's, not its throughput
    (on 200 of 10,000 batched regions, about 2.5 items per warp, the single-read kernel looked
    25% faster than the two-read kernels that run the whole batch 35% faster).  Either may be
    None."""
    from . import shard
    rr, hh = packed.region_read_off, packed.region_hap_off
    rl = np.diff(packed.read_off)
    longest = np.zeros(len(rr) - 1, np.int64)
    nz = np.diff(rr) > 0
    longest[nz] = np.maximum.reduceat(rl, rr[:-1][nz])
    is_long = longest > 256
    rng = np.random.default_rng(seed)
    out = []
    short = np.flatnonzero(~is_long)
    if len(short):
        order = rng.permutation(short)
        items = np.cumsum(np.diff(rr)[order] // 2 + 1)
        k = max(min_regions, int(round(fraction * len(short))), int(np.searchsorted(items, short_items)) + 1)
        out.append(np.sort(order[:min(len(short), k)]))
    else:
        out.append(None)
    long_ = np.flatnonzero(is_long)
    if len(long_):
        order = rng.permutation(long_)
        items = np.diff(rr)[order] * ((np.diff(hh)[order] + 1) // 2)
        k = min(len(order), int(np.searchsorted(np.cumsum(items), long_items)) + 1)
        out.append(np.sort(order[:k]))
    else:
        out.append(None)
    return [None if g is None else shard.subset(packed, g)[0] for g in out]


def autotune(engine: native.Engine, packed: native.Packed, params, repeats: int = 3, use_cache: bool = True,
             log: list | None = None, stratify: bool = False, confirm: bool = False) -> dict:
    """Choose vd_tuning for this batch shape by timing candidates and leave the best on the
    engine.  With stratify=False ``packed`` is already the sample every knob is timed on; with
    stratify=True it is the whole batch (region form) and the long-read knobs are timed on its
    long-read regions, the others on a sample of its short-read regions (split_samples).
    With confirm=True a choice other than the default is timed once more against the default
    on ``packed`` itself and kept only if faster there (``whole_batch`` in the result): a
    sample cannot show how a persistent kernel's tail behaves on the whole batch."""
    if stratify:
        short_s, long_s = split_samples(packed)
    else:
        short_s, long_s = packed, packed
    sig_src = packed
    key = f"{engine.info()['gpu']}|{signature(sig_src.read_off, sig_src.hap_off)}|anch={params.anchored}"
    cache = {}
    if use_cache and CACHE.exists():
        try:
            cache = json.loads(CACHE.read_text())
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        best = dict(DEFAULT, **cache[key])
        _apply(engine, best)
        return dict(best, cached=True)
    best = dict(DEFAULT)
    trials = []
    default_ms = {}
    sample_ms = {}
    for knobs, sample, name in ((LONG_KNOBS, long_s, "long"), (SHORT_KNOBS, short_s, "short")):
        if sample is None:
            continue
        best_ms = _time(engine, sample, params, best, repeats)
        default_ms[name] = round(best_ms, 3)
        trials.append((name, dict(best), best_ms))
        for knob in knobs:
            for v in SPACE[knob]:
                if v == best[knob]:
                    continue
                cand = dict(best, **{knob: v})
                ms = _time(engine, sample, params, cand, repeats)
                trials.append((name, cand, ms))
                if ms < best_ms * 0.99:
                    best, best_ms = cand, ms
        sample_ms[name] = round(best_ms, 3)
    whole = None
    if confirm and {k: best[k] for k in DEFAULT} != DEFAULT:
        ms_d = _time(engine, packed, params, DEFAULT, 1)
        ms_c = _time(engine, packed, params, best, 1)
        whole = {"batch_ms_default": round(ms_d, 3), "batch_ms_chosen": round(ms_c, 3),
                 "kept": "chosen" if ms_c < ms_d else "default"}
        if ms_c >= ms_d:
            best = dict(DEFAULT)
    _apply(engine, best)
    if log is not None:
        log.extend({"sample": nm, "setting": t, "ms": round(ms, 3)} for nm, t, ms in trials)
    if use_cache:
        cache[key] = best
        try:
            CACHE.parent.mkdir(parents=True, exist_ok=True)
            CACHE.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return dict(best, sample_ms=sample_ms, default_ms=default_ms, cached=False, whole_batch=whole,
                samples={k: (None if v is None else int(len(v.region_read_off) - 1))
                         for k, v in (("short", short_s), ("long", long_s))})
