"""Generates the golden PairHMM fixtures in tests/golden/ from the reference itself.

Runs only where the VarDepth reference tree is present (the build container):
the reference's own Python (caller/native/caller/accelerator.py,
whole_pairhmm.py, cpu_batch.py, trie_vector.py) is loaded from its source
files, read-only, and its native kernels are the reference C++ compiled from
source by oracle/Makefile into oracle/_ref/ (the shipped binaries are never
used).  Shapes and seeds are those of the reference's tests:

  accel_seed31.npz     tests/test_accelerator.py:41-53  (FP64 parity, both modes)
  accel_seed17391.npz  tests/test_accelerator.py:55-68  (mixed-precision set, both modes)
  base_seed712.npz     tests/test_base_acceleration.py:17-24 (core.cpp pair_scores)
  catalog_seed7713.npz tests/test_cpu_catalog.py:22-31  (anchored_pairhmm values)
  edge_cases.npz       tests/test_accelerator.py:21-40 shapes plus N bases, Q0/Q1/Q255,
                       1x1 and empty pairs
  single_region_q45.npz      the single-region workload (seed 0) at gap 10^-4.5 / ext 0.1 through
                       wide.cpp read_haplotype_batch_mode
  single_region_q30.npz      the same reads at the production 0.001 / 0.1 through
                       cpu_batch.pairs (trie_many, the production CPU path)
  genotypes_seed4242.npz  12 batched-regions-shaped regions: ln L from wide.cpp
                       read_haplotype_batch_mode, then per region molecule_rows.normalized_rows
                       with seeded mapping qualities, triangular._diploid_likelihood_numpy (no
                       prior) and mixture_cpu.general (mixture_general.cpp) at priors 0 and 0.001

Usage:  python tests/golden/make_golden.py [REFERENCE_CHECKOUT]
"""
from __future__ import annotations

import ctypes
import importlib.machinery
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

sys.dont_write_bytecode = True
HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
# the reference checkout: first command-line argument, else $VARDEPTH_REFERENCE, else the build
# container's read-only copy
REFERENCE = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VARDEPTH_REFERENCE", "/root/reference")) \
    / "caller" / "native" / "caller"
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from vardepth_b200 import synthetic  # noqa: E402


def load_source(name: str, path: Path):
    """Import a module from its .py source even where a compiled twin sits beside it."""
    loader = importlib.machinery.SourceFileLoader(name, str(path))
    spec = importlib.util.spec_from_loader(name, loader)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    loader.exec_module(mod)
    return mod


def reference_modules():
    O.build()
    # native_build.build_library compiles into the (read-only) reference tree;
    # point it at the libraries oracle/Makefile built from the same sources.
    nb = types.ModuleType("native_build")
    nb.build_library = lambda source: O.REF / f"lib{Path(source).stem}.so"
    sys.modules["native_build"] = nb
    # indel_refine.kernel (indel_refine.py:54-57) needs pysam to import; restate it.
    ir = types.ModuleType("indel_refine")

    def kernel():
        lib = ctypes.CDLL(str(O.REF / "libanchored.so"))
        lib.anchored_pairhmm.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int,
                                         ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.anchored_pairhmm.restype = ctypes.c_double
        return lib
    ir.kernel = kernel
    sys.modules["indel_refine"] = ir
    whole = load_source("whole_pairhmm", REFERENCE / "whole_pairhmm.py")
    lib = ctypes.CDLL(str(O.REF / "libwide.so"))
    arguments = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                 ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_double,
                 ctypes.POINTER(ctypes.c_double)]
    lib.read_haplotype_batch_mode.argtypes = arguments + [ctypes.c_int]
    lib.read_haplotype_batch_mode.restype = None
    lib.read_haplotype_batch.argtypes = arguments
    lib.read_haplotype_batch.restype = None
    lib.wide_capability.argtypes = []
    lib.wide_capability.restype = ctypes.c_int
    whole._LIB = lib
    accel = load_source("accelerator", REFERENCE / "accelerator.py")
    load_source("trie_vector", REFERENCE / "trie_vector.py")
    cpu_batch = load_source("cpu_batch", REFERENCE / "cpu_batch.py")
    return accel, whole, cpu_batch


def pack(pairs):
    """Pairs -> packed arrays (one read / haplotype slot per pair)."""
    rb, rq, hb = [], [], []
    roff, hoff = [0], [0]
    for s, q, h in pairs:
        qa = np.asarray(np.frombuffer(q, np.uint8) if isinstance(q, bytes) else q, np.uint8)
        rb.append(np.frombuffer(s.encode(), np.uint8))
        rq.append(qa)
        roff.append(roff[-1] + len(s))
        hb.append(np.frombuffer(h.encode(), np.uint8))
        hoff.append(hoff[-1] + len(h))
    cat = lambda xs: np.concatenate(xs).astype(np.uint8) if xs else np.empty(0, np.uint8)
    n = len(pairs)
    return dict(read_bases=cat(rb), read_quals=cat(rq), read_off=np.asarray(roff, np.int64), hap_bases=cat(hb),
                hap_off=np.asarray(hoff, np.int64), pair_read=np.arange(n, dtype=np.int32),
                pair_hap=np.arange(n, dtype=np.int32))


def main():
    accel, whole, cpu_batch = reference_modules()
    out = {}

    # test_accelerator.py:41-53
    rng = np.random.default_rng(31)
    pairs = []
    for n, m in [(1, 1), (7, 9), (30, 35), (151, 201), (300, 450), (700, 750)]:
        for _ in range(6):
            s = "".join(rng.choice(list("ACGT"), n))
            h = "".join(rng.choice(list("ACGT"), m))
            q = rng.integers(0, 61, n)
            pairs.append((s, q, h))
    out["accel_seed31"] = dict(pack(pairs), semiglobal=accel.cpu_pairs(pairs, False),
                               anchored=accel.cpu_pairs(pairs, True), gap=0.001, ext=0.1)

    # test_accelerator.py:55-68
    rng = np.random.default_rng(17391)
    pairs = []
    for n, m in [(1, 1), (7, 9), (30, 35), (151, 201), (300, 450), (512, 1000), (700, 750)]:
        for _ in range(12):
            seq = "".join(rng.choice(list("ACGT"), n))
            hap = "".join(rng.choice(list("ACGT"), m))
            pairs.append((seq, rng.integers(1, 61, n), hap))
    pairs.extend([("A" * 100, [60] * 100, "A" * 100), ("A" * 200, [35] * 200, "A" * 450),
                  ("ACGT" * 100, [60] * 400, "TGCA" * 160)])
    out["accel_seed17391"] = dict(pack(pairs), semiglobal=accel.cpu_pairs(pairs, False),
                                  anchored=accel.cpu_pairs(pairs, True), gap=0.001, ext=0.1)

    # test_base_acceleration.py:17-24 (core.cpp pair_scores, row division)
    rng = np.random.default_rng(712)
    seq = ["".join(rng.choice(list("ACGT"), n)) for n in [12, 151, 700]]
    qs = [rng.integers(2, 61, len(s)).tolist() for s in seq]
    haps = ["".join(rng.choice(list("ACGT"), n)) for n in [17, 197, 850]]
    expected = np.stack([O.ref_core_pair_scores(s, q, haps) for s, q in zip(seq, qs)])
    pairs = [(s, q, h) for s, q in zip(seq, qs) for h in haps]
    out["base_seed712"] = dict(pack(pairs), semiglobal=expected.ravel(), gap=0.001, ext=0.1)

    # test_cpu_catalog.py:22-31 (anchored, canonical FP64)
    rng = np.random.default_rng(7713)
    pairs = []
    for _ in range(31):
        n = int(rng.integers(12, 140))
        s = "".join(rng.choice(list("ACGT"), n))
        h = s[:n // 2] + "TA" + s[n // 2:]
        q = rng.integers(0, 61, n).tolist()
        pairs.append((s, q, h))
    canonical = cpu_batch.pairs(pairs, mode=1, canonical=True)
    out["catalog_seed7713"] = dict(pack(pairs), anchored=accel.cpu_pairs(pairs, True), canonical=canonical,
                                   gap=0.001, ext=0.1)

    # edge cases: test_accelerator.py:21-40 shapes, N bases, extreme qualities, empty
    reads = ["ACGT" * 8, "A" * 30, "GATTACA"]
    quals = [[30] * len(x) for x in reads]
    haps = ["TT" + r + "GG" for r in reads] + ["ACGT" * 10]
    pairs = [(r, q, h) for r, q in zip(reads, quals) for h in haps]
    pairs += [("ACGT" * 8, [30] * 32, "ACGT" * 9), ("ACGT" * 8, [3] * 32, "ACGT" * 9),
              ("GATTACA", [20] * 7, "GGGATTACAT"), ("ACGT" * 8, [30] * 32, "TCGT" * 9)]
    pairs += [("ACNT", [0, 20, 60, 255], "GATTACA"), ("G", [3], "G"), ("TGA", [10, 20, 30], "ACTG"),
              ("NNNN", [0, 1, 2, 3], "NANA"), ("ACGTN" * 20, [1] * 100, "ACGTN" * 25),
              ("A", [255], "A"), ("C", [0], "A"), ("A", [30], "ACGTACGT"), ("ACGTACGT", [30] * 8, "A")]
    prepared = np.concatenate([whole.Prepared(haps, mode=0)(r, q) for r, q in zip(reads, quals)])
    sg = accel.cpu_pairs(pairs, False)
    an = accel.cpu_pairs(pairs, True)
    empty = accel.cpu_pairs([("", [], "A"), ("A", [30], "")])
    assert np.isneginf(empty).all()
    out["edge_cases"] = dict(pack(pairs), semiglobal=sg, anchored=an, prepared=prepared,
                             n_prepared=np.int64(len(prepared)), gap=0.001, ext=0.1)

    # the single-region workload at the benchmark's Q45/Q10 and at the production 0.001/0.1
    w = synthetic.single_region()
    seqs, qls = [], []
    for r in range(len(w.read_off) - 1):
        a, b = w.read_off[r], w.read_off[r + 1]
        seqs.append(bytes(w.read_bases[a:b]).decode())
        qls.append(w.read_quals[a:b].copy())
    haps = [bytes(w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]).decode() for h in range(len(w.hap_off) - 1)]
    # Prepared.__call__ (whole_pairhmm.py:209-220) with the config's gap/ext in
    # place of its fixed 0.001/0.1: read_haplotype_batch_mode, automatic lanes
    q45 = np.stack([O.ref_batch_mode(s, q, haps, gap=w.gap, ext=w.ext) for s, q in zip(seqs, qls)])
    base = dict(read_bases=w.read_bases, read_quals=w.read_quals, read_off=w.read_off, hap_bases=w.hap_bases,
                hap_off=w.hap_off, region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    out["single_region_q45"] = dict(base, semiglobal=q45.ravel(), gap=w.gap, ext=w.ext)
    prod = cpu_batch.many(seqs, qls, haps, mode=0)
    out["single_region_q30"] = dict(base, semiglobal=np.asarray(prod).ravel(), gap=0.001, ext=0.1)

    # region post-processing (molecule_rows.py, triangular.py, mixture_general.cpp)
    blocks = types.ModuleType("blocks")
    blocks.blocks_for = None
    sys.modules["blocks"] = blocks
    load_source("artifact", REFERENCE / "base" / "artifact.py")
    rows = load_source("molecule_rows", REFERENCE / "molecule_rows.py")
    tri = load_source("triangular", REFERENCE / "triangular.py")
    mix = load_source("mixture_cpu", REFERENCE / "mixture_cpu.py")
    w = synthetic.batched_regions(seed=4242, n_regions=12)
    mq = np.random.default_rng(4242).choice([0, 3, 20, 37, 60, 255], size=len(w.read_off) - 1).astype(np.uint8)
    lns, vals, cert, gl_none, gl_p0, gl_p001 = [], [], [], [], [], []
    for g in range(w.n_regions):
        r0, r1 = w.region_read_off[g], w.region_read_off[g + 1]
        h0, h1 = w.region_hap_off[g], w.region_hap_off[g + 1]
        haps = [bytes(w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]).decode() for h in range(h0, h1)]
        ll = np.stack([O.ref_batch_mode(bytes(w.read_bases[w.read_off[r]:w.read_off[r + 1]]).decode(),
                                        w.read_quals[w.read_off[r]:w.read_off[r + 1]], haps, gap=w.gap, ext=w.ext)
                       for r in range(r0, r1)])
        v, c = rows.normalized_rows(ll, mq[r0:r1])
        lns.append(ll.ravel())
        vals.append(v.ravel())
        cert.append(c)
        gl_none.append(tri._diploid_likelihood_numpy(v, None))
        gl_p0.append(mix.general(v, 0.0, triangular=True))
        gl_p001.append(mix.general(v, 0.001, triangular=True))
    out["genotypes_seed4242"] = dict(
        read_bases=w.read_bases, read_quals=w.read_quals, read_off=w.read_off, hap_bases=w.hap_bases,
        hap_off=w.hap_off, region_read_off=w.region_read_off, region_hap_off=w.region_hap_off, mapping_quality=mq,
        semiglobal=np.concatenate(lns), values=np.concatenate(vals), certainty=np.concatenate(cert),
        gl_none=np.concatenate(gl_none), gl_prior0=np.concatenate(gl_p0), gl_prior001=np.concatenate(gl_p001),
        gap=w.gap, ext=w.ext)

    for name, arrays in out.items():
        np.savez_compressed(HERE / f"{name}.npz", **{k: np.asarray(v) for k, v in arrays.items()})
        print(name, {k: np.asarray(v).shape for k, v in arrays.items() if k in ("semiglobal", "anchored")})


if __name__ == "__main__":
    main()
