"""Drop-in PairHMM dispatch for VarDepth on B200 (sm_100a).

Mirrors the Python surface of caller/native/caller/accelerator.py:
``validate_pairs``, ``CudaPairHMM`` (``.score``, ``.last``, ``.metadata``),
``backend``, ``score_pairs`` and ``score_many``, with the same argument
meaning, result order, ``-inf`` for empty inputs and exception types.
``score_regions`` adds the batched form (many regions in one call) that the
reference builds by concatenating pairs.

Differences a caller can observe, all deliberate:

* There is no CPU path here: the CPU backend stays the reference's own code,
  so ``selection='cpu'`` raises RuntimeError, ``'auto'`` means CUDA, and the
  default backend is ``cuda``.
* ``precision`` defaults to ``'mixed'``: FP32 arithmetic with per-pair
  power-of-two scaling, the final row sums in FP64, and every pair whose
  scaled FP32 mass falls under the underflow floor recomputed in FP64 on the
  GPU.  ``'float64'`` runs every pair in the FP64 wavefront.
* ``strategy`` ('pair' or 'warp') is accepted and recorded; every pair runs
  in the anti-diagonal wavefront kernel.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from pathlib import Path

import numpy as np

from . import native

HERE = Path(__file__).resolve().parent
_ENGINE = None
_ENGINE_KEY = None

DEFAULT_GAP = 0.001   # every production call site (accelerator.py:52, base/caller.py:140)
DEFAULT_EXT = 0.1


def validate_pairs(pairs):
    """Check (read, qualities, haplotype) triples; return them with uint8 qualities.

    Same rules and messages as accelerator.py:25-40 (read and quality lengths
    agree, sequences are uppercase ACGTN strings, qualities are integer Phred
    scores in [0, 255]), checked in native code: the pair list is walked once
    by ``_pairlist.gather`` and the bases by ``vd_pair_list_plan``.
    """
    pairs = list(pairs)
    gathered = native.PairList(pairs)      # types, Phred range, lengths
    native.pair_list_plan(gathered)        # ACGTN of every distinct read and haplotype
    # one uint8 array per distinct quality object (``pairs`` keeps the objects, and so their
    # ids, alive while the table is used)
    arrays = {}
    for _, q, _ in pairs:
        if id(q) not in arrays:
            arrays[id(q)] = np.frombuffer(q, np.uint8) if isinstance(q, bytes) else np.asarray(q).astype(np.uint8)
    return [(s, arrays[id(q)], h) for s, q, h in pairs]


def pack_pairs(pairs) -> native.Packed:
    """Pack validated pairs into the pair form of vd_batch.

    Identical reads (same bases and qualities) and identical haplotypes are
    stored once; out[p] belongs to pairs[p].  (CudaPairHMM.score does this in
    native code through vd_score_pair_list; this form is for callers that
    want the packed batch itself.)
    """
    reads: dict = {}
    haps: dict = {}
    rb, rq, hb = [], [], []
    roff, hoff = [0], [0]
    pr = np.empty(len(pairs), np.int32)
    ph = np.empty(len(pairs), np.int32)
    for p, (s, q, h) in enumerate(pairs):
        key = (s, np.asarray(q, np.uint8).tobytes())
        r = reads.get(key)
        if r is None:
            r = len(reads)
            reads[key] = r
            rb.append(s.encode("ascii"))
            rq.append(key[1])
            roff.append(roff[-1] + len(s))
        g = haps.get(h)
        if g is None:
            g = len(haps)
            haps[h] = g
            hb.append(h.encode("ascii"))
            hoff.append(hoff[-1] + len(h))
        pr[p] = r
        ph[p] = g
    return native.Packed(np.frombuffer(b"".join(rb), np.uint8), np.frombuffer(b"".join(rq), np.uint8),
                         np.asarray(roff, np.int64), np.frombuffer(b"".join(hb), np.uint8),
                         np.asarray(hoff, np.int64), pair_read=pr, pair_hap=ph)


def _sources_sha256() -> str:
    h = hashlib.sha256()
    for p in sorted((HERE / "csrc").glob("*")):
        h.update(p.read_bytes())
    return h.hexdigest()


class CudaPairHMM:
    """GPU PairHMM engine with the constructor and attributes of accelerator.py:80-159."""

    def __init__(self, device=0, memory_mb=256, precision=None, strategy=None, gap=DEFAULT_GAP, ext=DEFAULT_EXT):
        strategy = strategy or os.environ.get("VARDEPTH_CUDA_KERNEL", "pair")
        if strategy not in ("pair", "warp"):
            raise ValueError("CUDA kernel must be pair or warp")
        self.strategy = strategy
        self.hap_bucket = int(os.environ.get("VARDEPTH_WARP_HAP_BUCKET", "128"))
        if self.hap_bucket < 32:
            raise ValueError("Warp haplotype bucket must be >=32")
        precision = precision or os.environ.get("VARDEPTH_CUDA_PRECISION", "mixed")
        if precision not in ("float64", "mixed"):
            raise ValueError("CUDA precision must be float64 or mixed")
        self.precision = precision
        if memory_mb < 8:
            raise ValueError("CUDA workspace budget must be at least 8 MiB")
        self.gap = float(gap)
        self.ext = float(ext)
        self.device = device
        self.memory_bytes = int(memory_mb) * 1024 ** 2
        self.engine = native.Engine(device, int(memory_mb))   # RuntimeError without a GPU
        info = self.engine.info()
        self.metadata = dict(backend="cuda", strategy=strategy, kernel="wavefront", hap_bucket=self.hap_bucket,
                             device=device, gpu=info["gpu"], compute_capability=info["compute_capability"],
                             sm_count=info["sm_count"], library=native.library().vd_version().decode(),
                             precision=precision, fmad=True, gap=self.gap, ext=self.ext,
                             kernel_sha256=_sources_sha256(), memory_budget_bytes=self.memory_bytes)
        self.last = None

    def _params(self, anchored, quality_offsets=None):
        mode = native.VD_PRECISION_FLOAT64 if self.precision == "float64" else native.VD_PRECISION_MIXED
        return native.make_params(self.gap, self.ext, anchored, mode, quality_offsets)

    def score(self, pairs, anchored=False):
        """ln L of (read, qualities, haplotype) triples in input order.  The list is walked
        once in C (pointers into the Python objects, no copies) and validated, deduplicated
        and regrouped into regions in the library (vd_score_pair_list)."""
        start = time.perf_counter()
        gathered = native.PairList(pairs)
        packing = time.perf_counter() - start
        params, _keep = self._params(anchored)
        out, st = self.engine.score_pair_list(gathered, params)
        self._record(st, anchored, start, packing)
        return out

    def score_packed(self, packed: native.Packed, anchored=False, quality_offsets=None):
        """Score a native.Packed batch (region or pair form) without Python packing."""
        start = time.perf_counter()
        params, _keep = self._params(anchored, quality_offsets)
        out, st = self.engine.forward(packed, params)
        self._record(st, anchored, start, 0.0)
        return out

    def _record(self, st, anchored, start, packing):
        s = st.as_dict()
        rescued = s["rescued_fp64"] + s["rescued_robust"]
        self.last = dict(**self.metadata,
                         float64_fallback_backend=("cuda_float64" if rescued else None),
                         float64_fallback_pairs=int(rescued),
                         float64_robust_pairs=int(s["rescued_robust"]),
                         float32_drift_pairs=int(s["rescued_fp32"]),
                         pairs=int(s["pairs"]), dp_cells=int(s["dp_cells"]), batches=int(s["batches"]),
                         work_items=int(s["work_items"]), live_array_bytes_upper_bound=int(s["live_bytes"]),
                         seconds=time.perf_counter() - start, includes_packing_transfers_and_synchronization=True,
                         anchored=bool(anchored), kernel_seconds=s["kernel_ms"] / 1000.0,
                         host_packing_seconds=packing + s["host_ms"] / 1000.0,
                         kernel_launches=int(s["kernel_launches"]), h2d_bytes=int(s["h2d_bytes"]),
                         d2h_bytes=int(s["d2h_bytes"]))


def backend():
    value = os.environ.get("VARDEPTH_PAIRHMM_BACKEND", "cuda")
    if value not in ("cpu", "cuda", "auto"):
        raise ValueError("Invalid PairHMM backend")
    return value


def _engine():
    global _ENGINE, _ENGINE_KEY
    key = (int(os.environ.get("VARDEPTH_CUDA_DEVICE", "0")), int(os.environ.get("VARDEPTH_CUDA_MEMORY_MB", "256")),
           os.environ.get("VARDEPTH_CUDA_PRECISION", "mixed"), os.environ.get("VARDEPTH_CUDA_KERNEL", "pair"),
           int(os.environ.get("VARDEPTH_WARP_HAP_BUCKET", "128")))
    if _ENGINE is None or _ENGINE_KEY != key:
        _ENGINE = CudaPairHMM(*key[:4])
        _ENGINE_KEY = key
    return _ENGINE


def _log(last):
    telemetry = os.environ.get("VARDEPTH_ACCELERATOR_LOG")
    if telemetry:
        import fcntl
        with open(telemetry, "a") as stream:
            fcntl.flock(stream.fileno(), fcntl.LOCK_EX)
            stream.write(json.dumps(last) + "\n")


def _choose(selection):
    choice = selection or backend()
    if choice not in ("cpu", "cuda", "auto"):
        raise ValueError("Invalid PairHMM backend")
    if choice == "cpu":
        raise RuntimeError("the CPU PairHMM backend is the reference caller's own code; "
                           "vardepth_b200 provides the CUDA backend only")
    return choice


def score_pairs(pairs, anchored=False, selection=None):
    """ln-likelihoods of (read, qualities, haplotype) pairs, in input order (accelerator.py:166-186)."""
    _choose(selection)
    pairs = list(pairs)
    if not pairs:
        return np.empty(0, np.float64)
    engine = _engine()
    result = engine.score(pairs, anchored)
    _log(engine.last)
    return result


def score_many(sequences, qualities, haplotypes, selection=None):
    """(reads x haplotypes) ln-likelihood matrix of one region (accelerator.py:188-190)."""
    if len(sequences) != len(qualities):
        raise ValueError("Sequence/quality batch lengths differ")
    _choose(selection)
    if not len(sequences) or not len(haplotypes):
        return np.empty((len(sequences), len(haplotypes)), np.float64)
    pairs = validate_pairs([(s, q, h) for s, q in zip(sequences, qualities) for h in haplotypes[:1]] +
                           [("", b"", h) for h in haplotypes])[:len(sequences)]
    rb = b"".join(s.encode("ascii") for s, _, _ in pairs)
    rq = b"".join(q.tobytes() for _, q, _ in pairs)
    roff = np.concatenate([[0], np.cumsum([len(s) for s, _, _ in pairs])]).astype(np.int64)
    hb = b"".join(h.encode("ascii") for h in haplotypes)
    hoff = np.concatenate([[0], np.cumsum([len(h) for h in haplotypes])]).astype(np.int64)
    packed = native.Packed(np.frombuffer(rb, np.uint8), np.frombuffer(rq, np.uint8), roff,
                           np.frombuffer(hb, np.uint8), hoff,
                           region_read_off=np.array([0, len(pairs)], np.int64),
                           region_hap_off=np.array([0, len(haplotypes)], np.int64))
    engine = _engine()
    out = engine.score_packed(packed)
    _log(engine.last)
    return out.reshape(len(sequences), len(haplotypes))


def score_regions(read_bases, read_quals, read_off, hap_bases, hap_off, region_read_off, region_hap_off,
                  anchored=False, engine: CudaPairHMM | None = None, quality_offsets=None):
    """Batched form: every region's reads x haplotypes, concatenated in region order.

    Inputs are packed numpy arrays (see include/vardepth_pairhmm.h vd_batch).
    """
    packed = native.Packed(read_bases, read_quals, read_off, hap_bases, hap_off,
                           region_read_off=region_read_off, region_hap_off=region_hap_off)
    engine = engine or _engine()
    out = engine.score_packed(packed, anchored, quality_offsets)
    _log(engine.last)
    return out
