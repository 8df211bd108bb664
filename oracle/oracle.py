"""ORACLE — test infrastructure only.

Only tests/, the smoke check of __graft_entry__ and bench.py's CPU legs load
this module; the vardepth_b200 product never imports it.

Two checkers:
  * ``liboracle.so``: the plain-C FP64 / long double restatement in
    pairhmm_oracle.c (wide.cpp:9-33, anchored.cpp:5-25);
  * ``_ref/lib*.so``: VarDepth's own PairHMM C++ compiled from the reference
    sources by oracle/Makefile, called with the reference's ctypes
    conventions (whole_pairhmm.py:176-185, trie_vector.py:8-13,
    cpu_batch.py:11-16, indel_refine.py:54-57, base/caller.py:30-40).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
SEMIGLOBAL_ROW_DIVIDE, SEMIGLOBAL_POW2 = 0, 2

c_u8p = ctypes.POINTER(ctypes.c_ubyte)
c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_i32p = ctypes.POINTER(ctypes.c_int32)


def build() -> None:
    """Compile liboracle.so and, where the reference tree is present, _ref/."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    path = HERE / "liboracle.so"
    if not path.exists():
        build()
    L = ctypes.CDLL(str(path))
    L.vdo_forward.restype = ctypes.c_double
    L.vdo_forward.argtypes = [c_u8p, c_u8p, ctypes.c_int, c_u8p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int, ctypes.c_int]
    L.vdo_forward_ex.restype = ctypes.c_double
    L.vdo_forward_ex.argtypes = L.vdo_forward.argtypes + [c_dp]
    L.vdo_forward_ld.restype = ctypes.c_double
    L.vdo_forward_ld.argtypes = [c_u8p, c_u8p, ctypes.c_int, c_u8p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int]
    L.vdo_forward_pairs.restype = ctypes.c_int
    L.vdo_forward_pairs.argtypes = [c_u8p, c_u8p, c_i64p, c_u8p, c_i64p, c_i32p, c_i32p, ctypes.c_int64,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, c_dp]
    L.vdo_grad_ex.restype = ctypes.c_int
    L.vdo_grad_ex.argtypes = [c_u8p, c_u8p, ctypes.c_int, c_u8p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int, c_dp, c_dp, c_dp]
    L.vdo_grad_pairs.restype = ctypes.c_int
    L.vdo_grad_pairs.argtypes = [c_u8p, c_u8p, c_i64p, c_u8p, c_i64p, c_i32p, c_i32p, ctypes.c_int64,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int, c_dp, ctypes.c_int, c_dp, c_dp]
    return L


def _bytes(x) -> np.ndarray:
    if isinstance(x, str):
        return np.frombuffer(x.encode("ascii"), np.uint8)
    if isinstance(x, (bytes, bytearray)):
        return np.frombuffer(bytes(x), np.uint8)
    return np.ascontiguousarray(x, dtype=np.uint8)


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_u8p)


def forward(read, qual, hap, gap=0.001, ext=0.1, anchored=False, scaling=SEMIGLOBAL_POW2, offsets=None) -> float:
    """FP64 restatement for one pair (ln L)."""
    r, q, h = _bytes(read), _bytes(qual), _bytes(hap)
    if offsets is None:
        return lib().vdo_forward(_p(r), _p(q), len(r), _p(h), len(h), gap, ext, int(anchored), scaling)
    off = np.ascontiguousarray(offsets, np.float64)
    return lib().vdo_forward_ex(_p(r), _p(q), len(r), _p(h), len(h), gap, ext, int(anchored), scaling,
                                off.ctypes.data_as(c_dp))


def forward_ld(read, qual, hap, gap=0.001, ext=0.1, anchored=False) -> float:
    """Extended-precision restatement for one pair (ln L)."""
    r, q, h = _bytes(read), _bytes(qual), _bytes(hap)
    return lib().vdo_forward_ld(_p(r), _p(q), len(r), _p(h), len(h), gap, ext, int(anchored))


def forward_pairs(read_bases, read_quals, read_off, hap_bases, hap_off, pair_read, pair_hap, gap=0.001, ext=0.1,
                  anchored=False, scaling=SEMIGLOBAL_POW2, extended=False, threads=0) -> np.ndarray:
    """Restatement over packed buffers and explicit pairs, on `threads` host threads."""
    rb, rq, hb = _bytes(read_bases), _bytes(read_quals), _bytes(hap_bases)
    ro = np.ascontiguousarray(read_off, np.int64)
    ho = np.ascontiguousarray(hap_off, np.int64)
    pr = np.ascontiguousarray(pair_read, np.int32)
    ph = np.ascontiguousarray(pair_hap, np.int32)
    out = np.empty(len(pr), np.float64)
    rc = lib().vdo_forward_pairs(_p(rb), _p(rq), ro.ctypes.data_as(c_i64p), _p(hb), ho.ctypes.data_as(c_i64p),
                                 pr.ctypes.data_as(c_i32p), ph.ctypes.data_as(c_i32p), len(pr), gap, ext,
                                 int(anchored), scaling, int(extended), int(threads), out.ctypes.data_as(c_dp))
    if rc:
        raise RuntimeError("oracle batch failed")
    return out


# ---- gradient checkers (theta = gap-open Phred, gap-continuation Phred, 4 bin offsets) ---------

def phred_to_prob(q: float) -> float:
    return float(10.0 ** (-q / 10.0))


def prob_to_phred(p: float) -> float:
    return float(-10.0 * np.log10(p))


def grad(read, qual, hap, gap, ext, anchored=False, offsets=None):
    """Expected-count (forward-backward) gradient of ln L for one pair, long double: (ln L, jac[6])."""
    r, q, h = _bytes(read), _bytes(qual), _bytes(hap)
    ln = ctypes.c_double()
    jac = np.zeros(6, np.float64)
    off = None if offsets is None else np.ascontiguousarray(offsets, np.float64)
    rc = lib().vdo_grad_ex(_p(r), _p(q), len(r), _p(h), len(h), gap, ext, int(anchored),
                           None if off is None else off.ctypes.data_as(c_dp), ctypes.byref(ln),
                           jac.ctypes.data_as(c_dp))
    if rc:
        raise MemoryError("oracle gradient: allocation failed")
    return ln.value, jac


def grad_pairs(read_bases, read_quals, read_off, hap_bases, hap_off, pair_read, pair_hap, gap, ext,
               anchored=False, offsets=None, threads=0):
    """grad() over explicit pairs of packed buffers, on host threads: (ln[P], jac[P, 6])."""
    rb, rq, hb = _bytes(read_bases), _bytes(read_quals), _bytes(hap_bases)
    ro = np.ascontiguousarray(read_off, np.int64)
    ho = np.ascontiguousarray(hap_off, np.int64)
    pr = np.ascontiguousarray(pair_read, np.int32)
    ph = np.ascontiguousarray(pair_hap, np.int32)
    ln = np.empty(len(pr), np.float64)
    jac = np.empty((len(pr), 6), np.float64)
    off = None if offsets is None else np.ascontiguousarray(offsets, np.float64)
    rc = lib().vdo_grad_pairs(_p(rb), _p(rq), ro.ctypes.data_as(c_i64p), _p(hb), ho.ctypes.data_as(c_i64p),
                              pr.ctypes.data_as(c_i32p), ph.ctypes.data_as(c_i32p), len(pr), gap, ext,
                              int(anchored), None if off is None else off.ctypes.data_as(c_dp), int(threads),
                              ln.ctypes.data_as(c_dp), jac.ctypes.data_as(c_dp))
    if rc:
        raise MemoryError("oracle gradient batch failed")
    return ln, jac


def fd_grad(read, qual, hap, theta, h=1e-3, anchored=False):
    """Central finite differences (step h on every Phred-scale parameter) of the FP64 forward."""
    theta = np.asarray(theta, np.float64)

    def f(t):
        return forward(read, qual, hap, phred_to_prob(t[0]), phred_to_prob(t[1]), anchored,
                       SEMIGLOBAL_ROW_DIVIDE, offsets=t[2:6])

    jac = np.empty(6)
    for k in range(6):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        jac[k] = (f(tp) - f(tm)) / (2 * h)
    return jac


# ---- region post-processing (checker of vd_region_genotypes) ----------------------------

def normalized_rows(ll, mapping_quality):
    """caller/native/caller/molecule_rows.py:6-14: rows exp(ll - row max) mixed with the
    mapping-quality error toward their mean; certainty = range of ln(max(1e-300, v))."""
    ll = np.asarray(ll, np.float64)
    err = 10.0 ** (-np.minimum(np.asarray(mapping_quality, np.int64), 60) / 10.0)
    with np.errstate(invalid="ignore"):
        v = np.exp(ll - ll.max(axis=1, keepdims=True))
        v = (1 - err[:, None]) * v + err[:, None] * v.mean(axis=1, keepdims=True)
        lv = np.log(np.maximum(1e-300, v))
    return v, lv.max(axis=1) - lv.min(axis=1)


_BALANCE = np.array([.2, .3, .4, .5, .6, .7, .8])
_BALANCE_W = np.array([.025, .1, .225, .3, .225, .1, .025])
_THETA = np.array([.02, .1, .2, .3])
_THETA_W = np.array([.4, .35, .2, .05])


def diploid_gl(v, artifact_prior=None):
    """Unordered diploid genotype log-likelihoods in VCF order (b = 0..H-1, a = 0..b):
    without a prior sum_rows ln max(1e-300, (v_a + v_b)/2) (triangular.py:13-16); with one the
    allele-balance mixture over _BALANCE and, for a prior > 0, the contamination mixture over
    _THETA x haplotypes, combined by log-sum-exp (mixture_general.cpp:9-37)."""
    v = np.asarray(v, np.float64)
    H = v.shape[1]
    a, b = np.array([(a, b) for b in range(H) for a in range(b + 1)]).T
    va, vb = v[:, a], v[:, b]
    if artifact_prior is None:
        # numpy's maximum keeps NaN (rows of an empty read)
        return np.log(np.maximum(1e-300, (va + vb) / 2)).sum(axis=0)
    # the C++ mixture's std::max(1e-300, x) turns NaN into 1e-300, as np.fmax does
    clean = np.array([np.log(np.fmax(1e-300, w * va + (1 - w) * vb)).sum(axis=0) + np.log(q)
                      for w, q in zip(_BALANCE, _BALANCE_W)])
    clean = np.logaddexp.reduce(clean, axis=0)
    if artifact_prior <= 0:
        return clean
    art = [np.log(np.fmax(1e-300, (1 - t) * (va + vb) / 2 + t * v[:, c, None])).sum(axis=0) + np.log(q / H)
           for t, q in zip(_THETA, _THETA_W) for c in range(H)]
    art = np.logaddexp.reduce(np.array(art), axis=0)
    return np.logaddexp(np.log1p(-artifact_prior) + clean, np.log(artifact_prior) + art)


def region_pairs(region_read_off, region_hap_off):
    """Explicit (read, hap) pairs of a region batch in the library's output order."""
    rr = np.asarray(region_read_off, np.int64)
    hh = np.asarray(region_hap_off, np.int64)
    pr, ph = [], []
    for g in range(len(rr) - 1):
        reads = np.arange(rr[g], rr[g + 1])
        haps = np.arange(hh[g], hh[g + 1])
        pr.append(np.repeat(reads, len(haps)))
        ph.append(np.tile(haps, len(reads)))
    if not pr:
        return np.empty(0, np.int32), np.empty(0, np.int32)
    return np.concatenate(pr).astype(np.int32), np.concatenate(ph).astype(np.int32)


# ---- the reference's own C++ (compiled from its sources into _ref/) ---------------------

def ref_available() -> bool:
    return all((REF / f).exists() for f in ("libwide.so", "libbatch_hmm.so", "libtrie_vector.so",
                                           "libanchored.so", "libcaller.so"))


@lru_cache(maxsize=None)
def ref_lib(name: str) -> ctypes.CDLL:
    path = REF / f"lib{name}.so"
    if not path.exists():
        raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference tree is present")
    L = ctypes.CDLL(str(path))
    if name in ("wide", "caller"):
        L.read_haplotype.restype = ctypes.c_double
        L.read_haplotype.argtypes = [ctypes.c_char_p, c_u8p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double]
        args = [ctypes.c_char_p, c_u8p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_double, c_dp]
        L.read_haplotype_batch.restype = None
        L.read_haplotype_batch.argtypes = args
        if name == "wide":
            L.read_haplotype_batch_mode.restype = None
            L.read_haplotype_batch_mode.argtypes = args + [ctypes.c_int]
            L.wide_capability.restype = ctypes.c_int
    elif name == "anchored":
        L.anchored_pairhmm.restype = ctypes.c_double
        L.anchored_pairhmm.argtypes = [ctypes.c_char_p, c_u8p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double]
    elif name == "batch_hmm":
        L.pairhmm_pairs.restype = ctypes.c_int
        L.pairhmm_pairs.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(c_u8p),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_char_p),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp]
    elif name == "trie_vector":
        L.trie_many.restype = ctypes.c_int
        L.trie_many.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(c_u8p), ctypes.POINTER(ctypes.c_int),
                                ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int),
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, ctypes.POINTER(ctypes.c_uint64)]
    return L


def _q(q) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(q, np.uint8) if isinstance(q, (bytes, bytearray)) else q, np.uint8)


def ref_read_haplotype(s: str, q, h: str, gap=0.001, ext=0.1, lib_name="wide") -> float:
    """wide.cpp:9 (2^512 rescaling) or core.cpp:9 (row division, lib_name='caller')."""
    qa = _q(q)
    return ref_lib(lib_name).read_haplotype(s.encode(), qa.ctypes.data_as(c_u8p), len(s), h.encode(), len(h), gap, ext)


def ref_anchored(s: str, q, h: str, gap=0.001, ext=0.1) -> float:
    """anchored.cpp:5."""
    qa = _q(q)
    return ref_lib("anchored").anchored_pairhmm(s.encode(), qa.ctypes.data_as(c_u8p), len(s), h.encode(), len(h),
                                                gap, ext)


def ref_batch_mode(s: str, q, haps, gap=0.001, ext=0.1, mode=0) -> np.ndarray:
    """wide.cpp:349 read_haplotype_batch_mode: one read against many haplotypes."""
    qa = _q(q)
    enc = [h.encode() for h in haps]
    hp = (ctypes.c_char_p * len(enc))(*enc)
    ln = (ctypes.c_int * len(enc))(*(len(h) for h in enc))
    out = np.empty(len(enc), np.float64)
    ref_lib("wide").read_haplotype_batch_mode(s.encode(), qa.ctypes.data_as(c_u8p), len(s), hp, ln, len(enc), gap,
                                              ext, out.ctypes.data_as(c_dp), mode)
    return out


def ref_core_pair_scores(s: str, q, haps) -> np.ndarray:
    """base/caller.py:142-149 pair_scores over core.cpp read_haplotype_batch (0.001/0.1)."""
    qa = _q(q)
    enc = [h.encode() for h in haps]
    hp = (ctypes.c_char_p * len(enc))(*enc)
    ln = (ctypes.c_int * len(enc))(*(len(h) for h in enc))
    out = np.empty(len(enc), np.float64)
    ref_lib("caller").read_haplotype_batch(s.encode(), qa.ctypes.data_as(c_u8p), len(s), hp, ln, len(enc), 0.001,
                                           0.1, out.ctypes.data_as(c_dp))
    return out


def ref_pairhmm_pairs(jobs, mode=0, lanes=0) -> np.ndarray:
    """batch_hmm.cpp:192 with the argument layout of cpu_batch._uncached_pairs (cpu_batch.py:44-62)."""
    count = len(jobs)
    enc = [(s.encode(), _q(q).tobytes(), h.encode()) for s, q, h in jobs]
    reads = (ctypes.c_char_p * count)(*(e[0] for e in enc))
    haps = (ctypes.c_char_p * count)(*(e[2] for e in enc))
    qp = (ctypes.c_char_p * count)(*(e[1] for e in enc))
    rn = (ctypes.c_int * count)(*(len(e[0]) for e in enc))
    hn = (ctypes.c_int * count)(*(len(e[2]) for e in enc))
    out = np.empty(count, np.float64)
    rc = ref_lib("batch_hmm").pairhmm_pairs(reads, ctypes.cast(qp, ctypes.POINTER(c_u8p)), rn, haps, hn, count,
                                            mode, lanes, out.ctypes.data_as(c_dp))
    if rc:
        raise RuntimeError("pairhmm_pairs failed")
    return out


def ref_trie_many(seqs, quals, haps, mode=0, lanes=0) -> np.ndarray:
    """trie_vector.cpp:284 for nr reads x nh haplotypes (row-major by read); NaN marks values <= 1e-200."""
    nr, nh = len(seqs), len(haps)
    renc = [s.encode() for s in seqs]
    qenc = [_q(q).tobytes() for q in quals]
    henc = [h.encode() for h in haps]
    rp = (ctypes.c_char_p * nr)(*renc)
    qp = (ctypes.c_char_p * nr)(*qenc)
    hp = (ctypes.c_char_p * nh)(*henc)
    rn = (ctypes.c_int * nr)(*(len(s) for s in renc))
    hn = (ctypes.c_int * nh)(*(len(h) for h in henc))
    out = np.empty(nr * nh, np.float64)
    cells = ctypes.c_uint64()
    rc = ref_lib("trie_vector").trie_many(rp, ctypes.cast(qp, ctypes.POINTER(c_u8p)), rn, nr, hp, hn, nh, mode,
                                          lanes, out.ctypes.data_as(c_dp), ctypes.byref(cells))
    if rc:
        raise RuntimeError("trie_many failed")
    return out.reshape(nr, nh)


def host_cores() -> int:
    """Usable host cores (affinity and cgroup quota), as caller/native/caller/cpu_schedule.py:5-18 counts them."""
    import math
    count = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        entry = next(line.split(":", 2)[2] for line in Path("/proc/self/cgroup").read_text().splitlines()
                     if line.startswith("0::"))
        root = Path("/sys/fs/cgroup")
        path = root / entry.lstrip("/")
        for directory in [path, *path.parents]:
            if directory == root.parent:
                break
            if not directory.is_relative_to(root):
                continue
            f = directory / "cpu.max"
            if f.exists():
                quota, period = f.read_text().split()
                if quota != "max":
                    count = min(count, max(1, math.floor(int(quota) / int(period))))
    except (OSError, ValueError, StopIteration):
        pass
    return max(1, count)
