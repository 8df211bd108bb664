#!/usr/bin/env python
"""PairHMM GCUPS on B200: the batched FP32-scaled forward against the reference CPU path.

Workload (batched regions): 10,000 synthetic regions, 2-16 haplotypes of
100-1,000 bp, lognormal(median 60) reads of 100-250 bp, gap-open Q45 /
gap-continuation Q10 (vardepth_b200/synthetic.py, seed 1).  A step scores every
read against every haplotype of its region.

  value    GCUPS of the device-resident plan: the captured CUDA graph of the kernel
           tiers (FP32 wavefront, FP32 drift rescue of long reads, FP64 rescue, FP64
           32-row strips) on inputs already in HBM, timed with CUDA events on the
           engine stream, max over ranks.
  e2e      GCUPS through the C-ABI call vd_forward with pinned host buffers: work-list
           build, host->device copies, kernels and the device->host copy of the
           results inside the timed region.
  roofline FP32-pipe roofline of the primary kernel: 12 algorithmic flops per cell
           (wide.cpp:19-21) times the cells it computes (value also counts the columns
           a haplotype shares with the previous one of its region, which are not
           streamed again) / its event-timed duration, against the FP32 FMA peak
           measured on the same device by vd_measure_fp32_peak.
  cpu_baseline  the reference's own C++ (oracle/_ref/libwide.so, compiled from
           caller/native/caller/wide.cpp) read_haplotype_batch_mode on every host
           core, on a deterministic region subsample of the same workload.

  parity   GPU results against the reference's own outputs on the whole CPU sample
           (vs_reference) and against the FP64 oracle on at least 1e10 cells of it
           (vs_oracle), with the genotype argmax of every checked region; for the
           mixed-length workload also a long_read block of 20 regions of 1-10 kb reads.
  e2e_pairs  GCUPS of score_pairs(list of (read, qualities, haplotype)) -- the
           reference's Python drop-in signature -- on a region sample of >= 1e6 pairs.

--impl reference times only that CPU implementation (rank 0), one subsample pass
per step.  Multi-GPU: one process per GPU under torchrun; every rank builds the
same workload, regions go to ranks longest-processing-time first by DP cells
(vardepth_b200/shard.py) and each rank scores its shard (strong scaling, no
data-path collective); the e2e results land in a node-wide shared-memory array,
each rank writing its own slices.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PairHMM GCUPS on 1 B200, batched vs plain, at ≤1e-4 log10L err vs FP64"
FLOPS_PER_CELL = 12          # M: 2 mul + 2 add + 1 emission; I: 3 mul + 1 add; D: 2 mul + 1 add (wide.cpp:19-21)
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--regions", type=int, default=0, help="regions of the workload (0: its full size)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--autotune", choices=["auto", "on", "off"], default="auto",
                    help="run vardepth_b200.autotune on a 2%% region sample first (auto: every forward workload)")
    ap.add_argument("--long-mode", choices=["warp", "block", "single"], default=None,
                    help="fix the long-read path (vd_tuning.long_mode) instead of autotuning it")
    ap.add_argument("--long-group", type=int, default=None,
                    help="with --long-mode: haplotypes per long-read warp item (vd_tuning.long_group, 1..8)")
    ap.add_argument("--workload", default="batched_regions",
                    choices=["batched_regions", "long_haplotype_stress", "planted_error_model", "mixed_length_regions"],
                    help="batched_regions (default) is the metric's workload; the others print their own line")
    return ap.parse_args()


WORKLOADS = {
    "batched_regions": "10000 regions, 2-16 haps of 100-1000 bp, lognormal(60) reads of 100-250 bp, "
                       "gap-open Q45, gap-cont Q10",
    "long_haplotype_stress": "2000 regions x 4 haps of 1000-5000 bp, 50 reads of 150-300 bp, 20% at 5% "
                             "error and Q2-Q15, gap-open Q45, gap-cont Q10",
    "planted_error_model": "1000 batched-regions-shaped regions simulated under gap-open Q40, gap-cont Q8, "
                           "bin offsets (+2,-1,0,+3); forward + reverse-wavefront gradient",
    "mixed_length_regions": "200000 regions, 2-32 haps of lognormal(400) 80-8000 bp, lognormal(40) reads of "
                            "150 bp, 2% of regions with 1-10 kb reads at 8% error, gap-open Q45, gap-cont Q10",
}
DEFAULT_REGIONS = {"batched_regions": 10_000, "long_haplotype_stress": 2_000, "planted_error_model": 1_000,
                   "mixed_length_regions": 200_000}


def make_workload(name, regions):
    from vardepth_b200 import synthetic
    if name == "batched_regions":
        return synthetic.batched_regions(n_regions=regions)
    if name == "long_haplotype_stress":
        return synthetic.long_haplotype_stress(n_regions=regions)
    if name == "planted_error_model":
        return synthetic.planted_error_model(n_regions=regions)
    return synthetic.mixed_length_regions(n_regions=regions, workers=0)


# ---- CPU reference (oracle/_ref, the reference's own wide.cpp) -----------------------

def _cpu_jobs(w, regions):
    """Pre-encoded ctypes arguments of read_haplotype_batch_mode, one job per read."""
    import ctypes
    jobs = []
    cells = 0
    for g in regions:
        h0, h1 = w.region_hap_off[g], w.region_hap_off[g + 1]
        haps = [bytes(w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]) for h in range(h0, h1)]
        hp = (ctypes.c_char_p * len(haps))(*haps)
        hl = (ctypes.c_int * len(haps))(*map(len, haps))
        msum = sum(map(len, haps))
        for r in range(w.region_read_off[g], w.region_read_off[g + 1]):
            a, b = w.read_off[r], w.read_off[r + 1]
            seq = bytes(w.read_bases[a:b])
            q = (ctypes.c_ubyte * (b - a)).from_buffer_copy(w.read_quals[a:b].tobytes())
            out = np.empty(len(haps))
            jobs.append((seq, q, b - a, hp, hl, len(haps), out, haps))
            cells += (b - a) * msum
    return jobs, cells


def _run_cpu(jobs, gap, ext, threads):
    import ctypes
    from oracle import oracle as O
    lib = O.ref_lib("wide")
    dp = ctypes.POINTER(ctypes.c_double)

    def one(j):
        seq, q, n, hp, hl, k, out, _ = j
        lib.read_haplotype_batch_mode(seq, q, n, hp, hl, k, gap, ext, out.ctypes.data_as(dp), 0)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as pool:
        list(pool.map(one, jobs, chunksize=4))
    return time.perf_counter() - t0


def cpu_reference(w, seconds, repeats=1, per_step=False):
    """Rate of the reference CPU path on a deterministic region subsample sized to ~`seconds`."""
    from oracle import oracle as O
    if not O.ref_available():
        O.build()
    threads = O.host_cores()
    order = np.random.default_rng(12345).permutation(w.n_regions)
    # calibrate on a small prefix of the order
    k = 1
    while True:
        jobs, cells = _cpu_jobs(w, order[:k])
        if cells >= 2e8 or k >= len(order):
            break
        k = min(len(order), k * 2)
    t = _run_cpu(jobs, w.gap, w.ext, threads)
    rate = cells / t
    need = rate * seconds
    k2 = max(k, int(np.ceil(0.01 * w.n_regions)))
    cum = 0
    sizes = np.array([(w.read_off[w.region_read_off[g + 1]] - w.read_off[w.region_read_off[g]]) *
                      (w.hap_off[w.region_hap_off[g + 1]] - w.hap_off[w.region_hap_off[g]]) for g in order])
    cum = np.cumsum(sizes)
    k2 = max(k2, int(np.searchsorted(cum, need)) + 1)
    k2 = min(k2, len(order))
    jobs, cells = _cpu_jobs(w, order[:k2])
    times = [_run_cpu(jobs, w.gap, w.ext, threads) for _ in range(repeats)]
    import platform
    model = ""
    try:
        model = next(l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name"))
    except (OSError, StopIteration):
        model = platform.processor()
    sample = (f"{k2} of {w.n_regions} regions (seeded order), {cells:.3e} cells, "
              f"read_haplotype_batch_mode (AVX-512 8-lane) on {threads} threads, {model}")
    return dict(cells=cells, times=times, threads=threads, sample=sample, jobs=jobs, regions=order[:k2])


def _diploid_gl(ll):
    """Unordered-genotype log-likelihoods of one region from its reads x haplotypes ln L."""
    v = np.exp(ll - ll.max(axis=1, keepdims=True))
    H = v.shape[1]
    a, b = np.array([(a, b) for b in range(H) for a in range(b + 1)]).T
    return np.log(np.maximum(1e-300, (v[:, a] + v[:, b]) / 2)).sum(axis=0)


# ---- clocks ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i] == "Active"})
        pw = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "power_w_median": statistics.median(pw) if pw else None}


# ---- main -------------------------------------------------------------------------------

def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = make_workload(args.workload, args.regions)
    per_step = max(2.0, args.cpu_seconds)
    res = cpu_reference(w, per_step, repeats=0)
    jobs, cells, threads = res["jobs"], res["cells"], res["threads"]
    for _ in range(args.warmup):
        _run_cpu(jobs, w.gap, w.ext, threads)
    times = [_run_cpu(jobs, w.gap, w.ext, threads) for _ in range(args.steps)]
    total = sum(times)
    value = cells * args.steps / total / 1e9
    line = {"metric": METRIC, "value": round(value, 4), "unit": "GCUPS", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "regions": args.regions,
                       "pairs": w.pairs(), "cells": w.cells(), "step": "one pass over the CPU sample"},
            "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
                             "sample": res["sample"]},
            "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def gradient_arm(args, local):
    """forward + reverse-wavefront gradient, checkpoint modes, accuracy and the fit."""
    import torch
    from vardepth_b200 import autograd as AG
    from vardepth_b200 import native
    w = make_workload("planted_error_model", args.regions)
    packed = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                           region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    engine = native.Engine(local, 65536)
    theta0 = np.array([45.0, 10.0, 0.0, 0.0, 0.0, 0.0])
    params, _keep = AG.params_from_theta(theta0)
    cells = w.cells()
    modes = {}
    launches = 0
    for name, ck in (("sqrt", native.VD_CHECKPOINT_SQRT), ("all", native.VD_CHECKPOINT_ALL)):
        for _ in range(max(1, args.warmup)):
            engine.forward_backward(packed, params, ck)
        torch.cuda.synchronize()
        ms = wall = 0.0
        for _ in range(args.steps):
            ln, jac, st = engine.forward_backward(packed, params, ck)
            ms += st.kernel_ms
            wall += st.total_ms
            launches += st.kernel_launches
        modes[name] = {"gcups": round(cells / (ms / args.steps) / 1e6, 3), "kernel_ms": round(ms / args.steps, 3),
                       "call_ms": round(wall / args.steps, 3), "scratch_bytes": int(st.scratch_bytes),
                       "fp64_pairs": int(st.fp64_pairs), "failed_pairs": int(st.failed_pairs)}
        if name == "sqrt":
            ref_ln, ref_jac = ln, jac
        elif not (np.array_equal(ln, ref_ln) and np.array_equal(jac, ref_jac)):
            raise SystemExit("checkpoint modes disagree")
    fw_ms = 0.0
    for _ in range(args.steps):
        _, fst = engine.forward(packed, params)
        fw_ms += fst.kernel_ms
    # gradient accuracy on a region subsample against the long-double expected-count oracle
    from oracle import oracle as O
    sub = np.random.default_rng(7).choice(w.n_regions, size=min(8, w.n_regions), replace=False)
    offs = np.concatenate([[0], np.cumsum(np.diff(w.region_read_off) * np.diff(w.region_hap_off))])
    idx = np.concatenate([np.arange(offs[g], offs[g + 1]) for g in sub])
    sw = w.subset(sub)
    pr, ph = sw.explicit_pairs()
    lo, jo = O.grad_pairs(sw.read_bases, sw.read_quals, sw.read_off, sw.hap_bases, sw.hap_off, pr, ph,
                          O.phred_to_prob(theta0[0]), O.phred_to_prob(theta0[1]), False, theta0[2:])
    tot, want = ref_jac[idx].sum(0), jo.sum(0)

    def per_pair(jac):
        """Relative error of every pair's Jacobian entries against the oracle (entries of
        magnitude >= 1e-3; smaller ones by their absolute error), and the pairs above 1e-6."""
        d = np.abs(jac - jo)
        rel = d / np.maximum(np.abs(jo), 1e-3)
        worst = rel.max(axis=1)
        over = np.flatnonzero(worst > 1e-6)
        return {"max_rel": float(worst.max()), "p99_rel": float(np.quantile(worst, 0.99)),
                "median_rel": float(np.median(worst)), "pairs_over_1e-6": int(len(over)),
                "fraction_over_1e-6": round(len(over) / len(worst), 5),
                "over_1e-6_read_lengths": sorted({int(sw.read_off[pr[i] + 1] - sw.read_off[pr[i]]) for i in over})[:20]}

    # the same pairs with every pair in the FP64 pass
    p64, _k64 = AG.params_from_theta(theta0, precision=native.VD_PRECISION_FLOAT64)
    sub_packed = native.Packed(sw.read_bases, sw.read_quals, sw.read_off, sw.hap_bases, sw.hap_off,
                               region_read_off=sw.region_read_off, region_hap_off=sw.region_hap_off)
    _, jac64, _ = engine.forward_backward(sub_packed, p64, native.VD_CHECKPOINT_SQRT)
    check = {"pairs": int(len(idx)), "oracle": "long-double expected-count gradient (oracle/)",
             "summed_gradient_rel_err": [float(v) for v in np.abs(tot - want) / np.abs(want)],
             "per_pair_mixed": per_pair(ref_jac[idx]), "per_pair_fp64": per_pair(jac64),
             "max_abs_dlog10": float(np.max(np.abs(ref_ln[idx] - lo)) / np.log(10.0))}
    # the fit on every region, from Q45 / Q10 / zero offsets
    batch = AG.Batch(engine, packed)
    hist = []
    t0 = time.perf_counter()
    theta = AG.fit_error_model(batch, w.region_read_off, w.region_hap_off, theta0, history=hist)
    fit_s = time.perf_counter() - t0
    planted = np.array(w.meta["planted"])
    line = {"metric": "PairHMM forward+gradient GCUPS on 1 B200 (planted-error-model workload)",
            "value": modes["sqrt"]["gcups"],
            "unit": "GCUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": modes["sqrt"]["kernel_ms"], "higher_is_better": True, "dtype": "fp32",
            "data": "synthetic", "config": {"workload": WORKLOADS["planted_error_model"], "regions": args.regions,
                                            "pairs": w.pairs(), "cells": cells, "seed": w.meta.get("seed")},
            "checkpointing": modes, "forward_gcups": round(cells / (fw_ms / args.steps) / 1e6, 3),
            "gradient_check": check,
            "fit": {"theta": [round(float(v), 4) for v in theta], "planted": planted.tolist(),
                    "max_abs_err_phred": float(np.max(np.abs(theta.numpy() - planted))),
                    "evaluations": len(hist), "seconds": round(fit_s, 2), "optimizer": "L-BFGS, FP32 theta",
                    "objective": "sum over reads of ln mean_h L (region mixture)"},
            "gpu_launches": launches}
    print(json.dumps(line), flush=True)
    engine.close()


def _region_offsets(w):
    return np.concatenate([[0], np.cumsum(np.diff(w.region_read_off) * np.diff(w.region_hap_off))])


def _compare(w, got, regions, want, region_cells):
    """|dlog10 L| of the GPU outputs of `regions` (in that order) against `want`, and the
    genotype argmax of each region (sum over reads of ln((L_a + L_b) / 2))."""
    offs = _region_offsets(w)
    idx = np.concatenate([np.arange(offs[g], offs[g + 1]) for g in regions])
    a, b = got[idx], want
    fin = np.isfinite(b)
    if not np.array_equal(np.isneginf(a), np.isneginf(b)) or not np.all(np.isfinite(a[fin])):
        raise SystemExit("-inf / non-finite results differ from the checker's")
    err = np.abs(a[fin] - b[fin]) / np.log(10.0)
    agree, o = 0, 0
    for g in regions:
        nr = int(w.region_read_off[g + 1] - w.region_read_off[g])
        nh = int(w.region_hap_off[g + 1] - w.region_hap_off[g])
        if nr and nh:
            x, y = a[o:o + nr * nh].reshape(nr, nh), b[o:o + nr * nh].reshape(nr, nh)
            agree += int(np.argmax(_diploid_gl(x)) == np.argmax(_diploid_gl(y)))
        else:
            agree += 1
        o += nr * nh
    return {"regions": int(len(regions)), "pairs": int(len(idx)), "cells": int(region_cells[regions].sum()),
            "max_abs_dlog10": float(err.max()) if err.size else 0.0,
            "p99_abs_dlog10": float(np.quantile(err, 0.99)) if err.size else 0.0,
            "genotype_argmax_agree": int(agree)}


def _oracle(w, regions):
    from oracle import oracle as O
    sw = w.subset(regions)
    pr, ph = sw.explicit_pairs()
    return O.forward_pairs(sw.read_bases, sw.read_quals, sw.read_off, sw.hap_bases, sw.hap_off, pr, ph, w.gap,
                           w.ext, threads=0)


def _pair_list(w, regions):
    """The regions as the reference's callers hand them over: a list of (read str, quality
    bytes, haplotype str), every read against every haplotype of its region."""
    out = []
    for g in regions:
        haps = [bytes(w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]).decode()
                for h in range(w.region_hap_off[g], w.region_hap_off[g + 1])]
        for r in range(w.region_read_off[g], w.region_read_off[g + 1]):
            a, b = w.read_off[r], w.read_off[r + 1]
            seq, q = bytes(w.read_bases[a:b]).decode(), bytes(w.read_quals[a:b])
            out.extend((seq, q, h) for h in haps)
    return out


def main():
    args = parse()
    if args.regions <= 0:
        args.regions = DEFAULT_REGIONS[args.workload]
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from vardepth_b200 import native, shard
    if args.workload == "planted_error_model":
        gradient_arm(args, local)
        return
    w = make_workload(args.workload, args.regions)
    cells, pairs = w.cells(), w.pairs()
    full = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                         region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    # this rank's regions: all of them on one GPU, its LPT shard on several
    if world > 1:
        shards = shard.shard_regions(shard.region_cells(full), world)
        mine, positions = shard.subset(full, shards[rank])
    else:
        shards, mine, positions = None, full, None
    my_cells = int(shard.region_cells(mine).sum()) if mine.n_outputs() else 0

    def pinned(a):
        t = torch.empty(max(1, a.nbytes), dtype=torch.uint8).pin_memory()
        v = t.numpy()[:a.nbytes].view(a.dtype)
        v[:] = a.reshape(-1)
        return t, v

    keep = []
    arrays = {}
    for name in ("read_bases", "read_quals", "read_off", "hap_bases", "hap_off", "region_read_off", "region_hap_off"):
        t, v = pinned(getattr(mine, name))
        keep.append(t)
        arrays[name] = v
    packed = native.Packed(arrays["read_bases"], arrays["read_quals"], arrays["read_off"], arrays["hap_bases"],
                           arrays["hap_off"], region_read_off=arrays["region_read_off"],
                           region_hap_off=arrays["region_hap_off"])
    engine = native.Engine(local, 65536)
    info = engine.info()
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    peak = __import__("ctypes").c_double()
    native.check(native.library().vd_measure_fp32_peak(local, __import__("ctypes").byref(peak)), "fp32 peak")
    warm = max(3, args.warmup)

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def gather_all(x):
        if dist is None:
            return [x]
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        parts = torch.empty(world, dtype=torch.float64, device="cuda")
        dist.all_gather_into_tensor(parts, t)
        return parts.tolist()

    # ---- autotuner: work-list choices timed on region samples, kept on the engine ----
    tuned = None
    if args.long_mode is not None:
        engine.set_tuning(**dict(engine.tuning(), long_mode={"warp": native.VD_LONG_WARP, "block": native.VD_LONG_BLOCK,
                                                             "single": native.VD_LONG_SINGLE}[args.long_mode],
                                 long_group=args.long_group or 0))
    elif args.autotune == "on" or args.autotune == "auto":
        from vardepth_b200 import autotune
        tlog = []
        t0 = time.perf_counter()
        best = autotune.autotune(engine, mine, params, use_cache=False, log=tlog, stratify=True, confirm=True)
        chosen = {k: best[k] for k in autotune.DEFAULT}
        confirm = best.get("whole_batch")
        tuned = {"chosen": chosen, "default": autotune.DEFAULT,
                 "samples_regions": best.get("samples"), "sample_ms_default": best.get("default_ms"),
                 "sample_ms_chosen": best.get("sample_ms"), "trials": tlog, "whole_batch": confirm,
                 "seconds": round(time.perf_counter() - t0, 2),
                 "method": "long-read knobs timed on long-read regions (about 8192 items), the others on "
                           "short-read regions holding about 49,152 two-read items (at least 2%); coordinate "
                           "descent, 1% threshold; a choice other than the default is kept only if one "
                           "captured run of the whole batch confirms it"}

    # ---- the warp-per-pair / block-per-pair split on a batch of few long pairs ----
    split = None
    if args.workload == "mixed_length_regions" and world == 1:
        rl = np.diff(w.read_off)
        longest = np.maximum.reduceat(rl, w.region_read_off[:-1])
        long_regions = np.flatnonzero(longest > 256)
        if len(long_regions):
            g = int(np.random.default_rng(5).choice(long_regions))
            one = w.subset([g])
            op = native.Packed(one.read_bases, one.read_quals, one.read_off, one.hap_bases, one.hap_off,
                               region_read_off=one.region_read_off, region_hap_off=one.region_hap_off)
            saved = engine.tuning()
            split = {"batch": f"one region with {len(one.read_off) - 1} reads of up to {int(longest[g])} bases",
                     "pairs": one.pairs(), "cells": one.cells(),
                     "kernel_ms": {}}
            for name, mode in (("warp", native.VD_LONG_WARP), ("block", native.VD_LONG_BLOCK),
                               ("single", native.VD_LONG_SINGLE)):
                engine.set_tuning(**dict(saved, long_mode=mode))
                p1 = engine.plan(op, params)
                p1.run()
                split["kernel_ms"][name] = round(float(np.median([p1.run().kernel_ms for _ in range(3)])), 3)
                p1.close()
            engine.set_tuning(**saved)

    # ---- device-resident batches (value) ----
    plan = engine.plan(packed, params)
    for _ in range(warm):
        plan.run()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        uuid = None
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    kernel_ms = primary_ms = 0.0
    rescued = drift_rescued = launches = shared = 0
    long_strips = long_runs = 0
    for _ in range(args.steps):
        st = plan.run()
        kernel_ms += st.kernel_ms
        primary_ms += st.primary_ms
        rescued = st.rescued_fp64 + st.rescued_robust
        drift_rescued = st.rescued_fp32
        long_strips, long_runs = st.long_strips, st.long_strip_runs
        shared = st.shared_cells
        launches += st.kernel_launches
    torch.cuda.synchronize()
    barrier()
    sampler.stop()
    rank_ms = gather_all(kernel_ms / args.steps)
    step_ms = max(rank_ms)
    value = cells / (step_ms / 1e3) / 1e9
    got = plan.fetch()
    plan.close()
    sharding = None
    if world > 1:
        rank_cells = gather_all(float(my_cells))
        sharding = {"policy": "LPT by DP cells (vardepth_b200/shard.py)", "ranks": world,
                    "rank_cells": [int(c) for c in rank_cells], "rank_kernel_ms": [round(x, 3) for x in rank_ms],
                    "imbalance_ms_max_over_mean": round(max(rank_ms) / (sum(rank_ms) / world), 4),
                    "imbalance_cells_max_over_mean": round(max(rank_cells) / (sum(rank_cells) / world), 4)}

    # ---- plain schedule on the same resident inputs (the batched-vs-plain comparison) ----
    plain = None
    if not args.no_plain:
        plain_params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED,
                                             schedule=native.VD_SCHEDULE_PLAIN)
        pplan = engine.plan(packed, plain_params)
        for _ in range(warm):
            pplan.run()
        barrier()
        torch.cuda.synchronize()
        plain_ms = 0.0
        plain_steps = max(1, min(args.steps, 3))
        plain_launches = 0
        for _ in range(plain_steps):
            st = pplan.run()
            plain_ms += st.kernel_ms
            plain_launches += st.kernel_launches
        torch.cuda.synchronize()
        barrier()
        plain_ms = allmax(plain_ms) / plain_steps
        plain_got = pplan.fetch()
        pplan.close()
        if not np.array_equal(plain_got, got, equal_nan=True):
            raise SystemExit("plain and batched schedules disagree")
        plain_value = cells / (plain_ms / 1e3) / 1e9
        plain = {"value": round(plain_value, 3), "unit": "GCUPS", "ms_per_step": round(plain_ms, 3),
                 "steps": plain_steps, "gpu_launches": plain_launches,
                 "batched_over_plain": round(value / plain_value, 3),
                 "schedule": "VD_SCHEDULE_PLAIN: one pair per warp item (a read longer than a strip: "
                             "the batched schedule's items of up to long_group haplotypes), fixed 8 rows "
                             "per lane, input order, static round-robin over a fixed grid; same tiers and "
                             "arithmetic, results bit-identical to the batched schedule"}

    # ---- end to end through vd_forward with pinned host buffers (e2e) ----
    e2e = None
    if not args.no_e2e:
        out_t = torch.empty(max(1, mine.n_outputs()) * 8, dtype=torch.uint8).pin_memory()
        out = out_t.numpy().view(np.float64)[:mine.n_outputs()]
        shared_out = None
        if world > 1:
            name = f"vd_bench_{os.environ.get('MASTER_PORT', '0')}_{os.getppid()}"
            if rank == 0:
                shared_out = shard.SharedOutput(name, pairs, create=True)
            barrier()
            if rank != 0:
                shared_out = shard.SharedOutput(name, pairs, create=False)
        for _ in range(warm):
            engine.forward(packed, params, out)
        barrier()
        torch.cuda.synchronize()
        wall = 0.0
        st = None
        for _ in range(args.steps):
            t0 = time.perf_counter()
            _, st = engine.forward(packed, params, out)
            if shared_out is not None:
                shared_out.write(positions, out)   # this rank's slices of the full output vector
            wall += time.perf_counter() - t0
        torch.cuda.synchronize()
        barrier()
        wall = allmax(wall)
        e2e = {"value": round(cells / (wall / args.steps) / 1e9, 3), "unit": "GCUPS",
               "h2d_bytes_per_step": int(st.h2d_bytes), "d2h_bytes_per_step": int(st.d2h_bytes),
               "ms_per_step": round(1e3 * wall / args.steps, 3), "host_ms_per_step": round(st.host_ms, 3),
               "api": "vd_forward (C ABI), pinned host inputs and outputs" +
                      ("; each rank writes its slices of a node-wide shared-memory output array" if world > 1 else "")}
        if not np.array_equal(out, got):
            raise SystemExit("vd_forward and the resident plan disagree")
        if shared_out is not None:
            if rank == 0:
                full_got = shared_out.values.copy()
                o = _region_offsets(w)
                for r in range(world):  # every rank's slices arrived, in input order
                    if not np.all(np.isfinite(full_got[np.concatenate([np.arange(o[g], o[g + 1])
                                                                       for g in shards[r]])]) |
                                  np.isneginf(full_got[np.concatenate([np.arange(o[g], o[g + 1])
                                                                       for g in shards[r]])])):
                        raise SystemExit(f"rank {r}'s slices of the shared output are missing")
            barrier()
            shared_out.close()

    # ---- the Python pair-list drop-in (score_pairs signature) on a >= 1e6-pair sample ----
    e2e_pairs = None
    if rank == 0 and world == 1 and not args.no_e2e:
        from vardepth_b200.accelerator import CudaPairHMM
        order = np.random.default_rng(99).permutation(w.n_regions)
        npairs = np.diff(w.region_read_off) * np.diff(w.region_hap_off)
        k = min(w.n_regions, int(np.searchsorted(np.cumsum(npairs[order]), 1_000_000)) + 1)
        sample = np.sort(order[:k])
        plist = _pair_list(w, sample)
        scorer = CudaPairHMM(device=local, memory_mb=65536, gap=w.gap, ext=w.ext)
        scorer.engine.set_tuning(**engine.tuning())  # the autotuned work-list choices, if any
        pl_cells = native.PairList(plist).cells()
        for _ in range(warm):
            res = scorer.score(plist)
        ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            res = scorer.score(plist)
            ms.append(1e3 * (time.perf_counter() - t0))
        o = _region_offsets(w)
        if not np.array_equal(res, got[np.concatenate([np.arange(o[g], o[g + 1]) for g in sample])]):
            raise SystemExit("score_pairs and the region batch disagree")
        last = scorer.last
        e2e_pairs = {"value": round(pl_cells / (np.mean(ms) / 1e3) / 1e9, 3), "unit": "GCUPS",
                     "pairs": len(plist), "cells": int(pl_cells), "regions": int(k),
                     "ms_per_step": round(float(np.mean(ms)), 3),
                     "host_ms_per_step": round(1e3 * last["host_packing_seconds"], 3),
                     "kernel_ms_per_step": round(1e3 * last["kernel_seconds"], 3),
                     "h2d_bytes_per_step": int(last["h2d_bytes"]), "d2h_bytes_per_step": int(last["d2h_bytes"]),
                     "api": "CudaPairHMM.score(list of (read str, quality bytes, haplotype str)): the list walked "
                            "in C, validated, deduplicated and regrouped into regions by vd_score_pair_list"}
        scorer.engine.close()

    # ---- CPU baseline (reference code, rank 0 at N=1) and parity against it and the oracle ----
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        res = None
        if not args.no_cpu:
            res = cpu_reference(w, args.cpu_seconds)
            cpu = {"value": round(res["cells"] / res["times"][0] / 1e9, 4), "unit": "GCUPS", "cores": res["threads"],
                   "kind": "reference", "sample": res["sample"]}
        parity = {}
        region_cells = shard.region_cells(full)
        if res is not None:
            ref_out = np.concatenate([j[6] for j in res["jobs"]])
            parity["vs_reference"] = dict(_compare(w, got, res["regions"], ref_out, region_cells),
                                          checker="the reference's read_haplotype_batch_mode (oracle/_ref, "
                                                  "compiled from wide.cpp), the CPU-baseline sample")
            base_order = res["regions"]
        else:
            base_order = np.random.default_rng(12345).permutation(w.n_regions)
        # the FP64 oracle on a prefix of the same seeded region order holding >= 1e10 cells
        cum = np.cumsum(region_cells[base_order])
        k = min(len(base_order), int(np.searchsorted(cum, 1e10)) + 1)
        t0 = time.perf_counter()
        parity["vs_oracle"] = dict(_compare(w, got, base_order[:k], _oracle(w, base_order[:k]), region_cells),
                                   checker="FP64 restatement (oracle/)",
                                   seconds=round(time.perf_counter() - t0, 1))
        if args.workload == "mixed_length_regions":
            # 20 regions of 1-10 kb reads (the drift and FP64 tiers' pairs), from the smaller half of them
            rl = np.diff(w.read_off)
            longest = np.maximum.reduceat(rl, w.region_read_off[:-1]) if len(rl) else rl
            long_regions = np.flatnonzero(longest > 256)
            small = long_regions[np.argsort(region_cells[long_regions])][:max(20, len(long_regions) // 2)]
            pick = np.sort(np.random.default_rng(11).choice(small, size=min(20, len(small)), replace=False))
            t0 = time.perf_counter()
            parity["long_read"] = dict(_compare(w, got, pick, _oracle(w, pick), region_cells),
                                       checker="FP64 restatement (oracle/)",
                                       selection="20 seeded regions with 1-10 kb reads at 8% error, from the half "
                                                 "with fewer cells", seconds=round(time.perf_counter() - t0, 1))

    primary_ms = allmax(primary_ms) / args.steps
    # batched regions: the primary tier holds all but ~0.5% of the work; elsewhere
    # the rescue tiers can hold a real share, so the whole step is the denominator
    roof_ms = primary_ms if args.workload == "batched_regions" else step_ms
    # the FMA pipe only sees the cells it computes: columns a haplotype shares
    # with the previous one of its region are counted in value, not here
    computed = my_cells - shared
    achieved = computed * FLOPS_PER_CELL / (roof_ms / 1e3) / 1e12
    traffic, traffic_source = None, None
    tf = ROOT / "profiles" / "pairhmm_f32_traffic.json"
    if tf.exists() and args.workload == "batched_regions" and world == 1:
        try:
            t = json.loads(tf.read_text())
            traffic = t.get("bytes_per_launch_full_batched_regions")
            traffic_source = t.get("source")
        except (OSError, ValueError):
            traffic = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": round(step_ms, 3), "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "regions": args.regions, "pairs": pairs, "cells": cells,
                       "shared_prefix_cells": int(shared) if world == 1 else None, "seed": w.meta.get("seed"),
                       "inputs_bytes": w.input_bytes(), "l2": "inputs (%.2f GB) exceed the 126 MB L2; "
                       "the recurrence state lives in registers" % (w.input_bytes() / 1e9),
                       "parallelism": f"{world} GPUs, LPT region shards" if world > 1 else "1 GPU",
                       "precision": "FP32 scaled, FP32 drift and FP64 rescue", "gpu": info["gpu"]},
            "roofline": {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak.value, 3),
                         "unit": "TFLOP/s", "frac": round(achieved / peak.value, 4), "traffic": traffic,
                         "traffic_source": traffic_source,
                         "flops_per_cell": FLOPS_PER_CELL, "cells_computed": int(computed),
                         "kernel": "FP32 tier: pairhmm_pair_kernel x2 + pairhmm_kernel<float>"
                         if args.workload == "batched_regions" else "every tier (whole step)",
                         "primary_ms": round(primary_ms, 3),
                         "peak_source": "vd_measure_fp32_peak (FMA loop, this device, this run)",
                         "nominal_peak": round(NOMINAL_FP32_TFLOPS, 1)},
            "plain": plain, "autotune": tuned, "long_split_few_pairs": split, "sharding": sharding,
            "cpu_baseline": cpu, "e2e": e2e, "e2e_pairs": e2e_pairs, "gpu_launches": launches,
            "rescued_pairs": int(rescued), "rescued_fraction": round(rescued / max(1, mine.n_outputs()), 6),
            "rescued_fp32_drift_pairs": int(drift_rescued), "parity": parity, "clocks": sampler.summary(),
        }
        if long_strips:
            # the long-read warp kernel: strips (per pair of an item) and their runs
            line["long_read_strips"] = {"strips": int(long_strips), "runs": int(long_runs),
                                        "runs_per_strip": round(long_runs / long_strips, 4)}
        print(json.dumps(line), flush=True)
    engine.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
