"""Parity of the CUDA PairHMM with the reference's own results and the FP64 oracle.

Tolerances:
  * precision='float64': 2e-9 in ln, the reference's FP64 CUDA-vs-CPU bound
    (caller/native/caller/tests/test_accelerator.py:50);
  * precision='mixed' (FP32 scaled + FP64 rescue): |delta log10 L| <= 1e-4 per
    pair, i.e. 2.303e-4 in ln, and identical genotype-likelihood argmax.
"""
import ctypes

import numpy as np
import pytest

from conftest import FP64_ATOL_LN, LN10, MIXED_ATOL_LN, golden, golden_pairs
from oracle import oracle as O
from vardepth_b200 import native
from vardepth_b200 import synthetic as S
from vardepth_b200.accelerator import CudaPairHMM, score_many, score_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed():
    return CudaPairHMM(memory_mb=4096, precision="mixed")


@pytest.fixture(scope="module")
def fp64():
    return CudaPairHMM(memory_mb=4096, precision="float64")


def _with(engine, gap, ext):
    engine.gap, engine.ext = float(gap), float(ext)
    return engine


def diploid_gl(ll_rows: np.ndarray) -> np.ndarray:
    """Unordered-genotype log-likelihoods of one region (caller/native/caller/triangular.py:27-30
    over molecule_rows.py:10 normalised rows): sum_reads ln((L_a + L_b)/2)."""
    v = np.exp(ll_rows - ll_rows.max(axis=1, keepdims=True))
    H = v.shape[1]
    a, b = np.array([(a, b) for b in range(H) for a in range(b + 1)]).T
    return np.log(np.maximum(1e-300, (v[:, a] + v[:, b]) / 2)).sum(axis=0)


def assert_mixed_close(got, want):
    finite = np.isfinite(want)
    assert np.array_equal(np.isneginf(got), np.isneginf(want))
    err = np.abs(got[finite] - want[finite]) / LN10
    assert err.size == 0 or err.max() <= 1e-4, f"max |dlog10| {err.max():.3e}"
    return err


@pytest.mark.parametrize("anchored", [False, True])
def test_fp64_matches_reference_cpu_pairs(fp64, anchored):
    d = golden("accel_seed31")
    got = _with(fp64, 0.001, 0.1).score(golden_pairs(d), anchored)
    np.testing.assert_allclose(got, d["anchored" if anchored else "semiglobal"], atol=FP64_ATOL_LN, rtol=0)


@pytest.mark.parametrize("anchored", [False, True])
@pytest.mark.parametrize("name", ["accel_seed31", "accel_seed17391"])
def test_mixed_matches_reference_cpu_pairs(mixed, name, anchored):
    d = golden(name)
    got = _with(mixed, 0.001, 0.1).score(golden_pairs(d), anchored)
    assert_mixed_close(got, d["anchored" if anchored else "semiglobal"])
    if name == "accel_seed17391":
        # random reads against random haplotypes underflow FP32: they must be rescued
        assert mixed.last["float64_fallback_pairs"] >= 12
        assert mixed.last["precision"] == "mixed"


def test_base_model_pair_scores(mixed, fp64):
    d = golden("base_seed712")
    pairs = golden_pairs(d)
    np.testing.assert_allclose(_with(fp64, 0.001, 0.1).score(pairs), d["semiglobal"], atol=FP64_ATOL_LN, rtol=0)
    assert_mixed_close(_with(mixed, 0.001, 0.1).score(pairs), d["semiglobal"])


def test_anchored_catalog(mixed, fp64):
    d = golden("catalog_seed7713")
    pairs = golden_pairs(d)
    np.testing.assert_allclose(_with(fp64, 0.001, 0.1).score(pairs, True), d["anchored"], atol=1e-11, rtol=0)
    assert_mixed_close(_with(mixed, 0.001, 0.1).score(pairs, True), d["anchored"])


@pytest.mark.parametrize("anchored", [False, True])
def test_edge_cases(mixed, fp64, anchored):
    d = golden("edge_cases")
    pairs = golden_pairs(d)
    want = d["anchored" if anchored else "semiglobal"]
    np.testing.assert_allclose(_with(fp64, 0.001, 0.1).score(pairs, anchored), want, atol=FP64_ATOL_LN, rtol=0)
    assert_mixed_close(_with(mixed, 0.001, 0.1).score(pairs, anchored), want)
    empty = _with(mixed, 0.001, 0.1).score([("", [], "A"), ("A", [30], ""), ("", [], "")], anchored)
    assert np.isneginf(empty).all()


@pytest.mark.parametrize("name", ["single_region_q45", "single_region_q30"])
def test_single_region_against_reference(mixed, name):
    d = golden(name)
    packed = native.Packed(d["read_bases"], d["read_quals"], d["read_off"], d["hap_bases"], d["hap_off"],
                           region_read_off=d["region_read_off"], region_hap_off=d["region_hap_off"])
    got = _with(mixed, d["gap"], d["ext"]).score_packed(packed)
    want = d["semiglobal"]
    assert_mixed_close(got, want)
    H = int(d["region_hap_off"][1])
    assert np.argmax(diploid_gl(got.reshape(-1, H))) == np.argmax(diploid_gl(want.reshape(-1, H)))


def _oracle_workload(w, anchored=False):
    pr, ph = w.explicit_pairs()
    return O.forward_pairs(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off, pr, ph, w.gap, w.ext,
                           anchored, O.SEMIGLOBAL_POW2, threads=0)


def _packed(w):
    return native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                         region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)


def _argmax_agree(w, got, want):
    o = 0
    agree = total = 0
    for g in range(w.n_regions):
        nr = int(w.region_read_off[g + 1] - w.region_read_off[g])
        nh = int(w.region_hap_off[g + 1] - w.region_hap_off[g])
        k = nr * nh
        if k:
            total += 1
            agree += int(np.argmax(diploid_gl(got[o:o + k].reshape(nr, nh))) ==
                         np.argmax(diploid_gl(want[o:o + k].reshape(nr, nh))))
        o += k
    return agree, total


def test_batched_regions_sample_against_oracle(mixed):
    w = S.batched_regions(n_regions=24)
    got = _with(mixed, w.gap, w.ext).score_packed(_packed(w))
    want = _oracle_workload(w)
    err = assert_mixed_close(got, want)
    agree, total = _argmax_agree(w, got, want)
    assert agree == total
    print(f"batched_regions sample: pairs {len(got)} max|dlog10| {err.max():.2e} "
          f"p99 {np.quantile(err, .99):.2e} rescued {mixed.last['float64_fallback_pairs']}")


def anchored_windows(seed, n_sites=40, reads_per_site=24):
    """Anchored refinement jobs as indel_refine.py builds them (caller/native/caller/indel_refine.py:143-151):
    a read span against left + allele + right haplotype windows of about the same length."""
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(n_sites):
        ref = "".join(rng.choice(list("ACGT"), 400))
        p = int(rng.integers(150, 250))
        k = int(rng.integers(1, 11))
        alt = ref[:p] + ref[p + k:] if rng.random() < 0.5 else ref[:p] + "".join(rng.choice(list("ACGT"), k)) + ref[p:]
        for _ in range(reads_per_site):
            src = alt if rng.random() < 0.5 else ref
            a = int(rng.integers(20, 120))
            b = int(rng.integers(p + 20, min(len(src), p + 140)))
            read = list(src[a:b])
            for i in np.flatnonzero(rng.random(len(read)) < 0.01):
                read[i] = "ACGT"[("ACGT".index(read[i]) + int(rng.integers(1, 4))) % 4]
            q = rng.choice([10, 20, 30, 40], len(read), p=[.05, .15, .5, .3])
            for hap in (ref, alt):
                w0 = a
                w1 = b + (len(hap) - len(src))
                pairs.append(("".join(read), q, hap[w0:w1]))
    return pairs


def test_anchored_refinement_windows(mixed, fp64):
    pairs = anchored_windows(5)
    want = np.array([O.forward(s, q.astype(np.uint8), h, 0.001, 0.1, True, 0) for s, q, h in pairs])
    np.testing.assert_allclose(_with(fp64, 0.001, 0.1).score(pairs, True), want, atol=FP64_ATOL_LN, rtol=0)
    err = assert_mixed_close(_with(mixed, 0.001, 0.1).score(pairs, True), want)
    print(f"anchored windows: pairs {len(pairs)} max|dlog10| {err.max():.2e} "
          f"rescued {mixed.last['float64_fallback_pairs']}")


def test_long_haplotype_stress_precision(mixed):
    w = S.long_haplotype_stress(n_regions=6)
    got = _with(mixed, w.gap, w.ext).score_packed(_packed(w))
    want = _oracle_workload(w)
    err = assert_mixed_close(got, want)
    agree, total = _argmax_agree(w, got, want)
    assert agree == total
    print(f"long_haplotype_stress sample: pairs {len(got)} max|dlog10| {err.max():.2e} rescued "
          f"{mixed.last['float64_fallback_pairs']}/{len(got)}")


@pytest.mark.parametrize("anchored", [False, True])
def test_long_reads_strip_mined(mixed, fp64, anchored):
    # reads longer than one 256-row strip, and reads just around the strip size
    rng = np.random.default_rng(99)
    pairs = []
    for n, m in [(255, 300), (256, 300), (257, 300), (513, 700), (1500, 1800), (3000, 3100)]:
        hap = "".join(rng.choice(list("ACGT"), m))
        start = int(rng.integers(0, m - n + 1))
        read = list(hap[start:start + n])
        for i in np.flatnonzero(rng.random(n) < 0.03):
            read[i] = "ACGT"[(("ACGT".index(read[i])) + 1) % 4]
        q = rng.choice([10, 20, 30, 40], n)
        pairs.append(("".join(read), q, hap))
    want = np.array([O.forward(s, q.astype(np.uint8), h, 0.001, 0.1, anchored) for s, q, h in pairs])
    np.testing.assert_allclose(_with(fp64, 0.001, 0.1).score(pairs, anchored), want, atol=FP64_ATOL_LN * 10, rtol=0)
    assert_mixed_close(_with(mixed, 0.001, 0.1).score(pairs, anchored), want)


def test_pairs_regions_and_chunking_agree():
    w = S.batched_regions(n_regions=200)
    eng = CudaPairHMM(memory_mb=4096, gap=w.gap, ext=w.ext)
    regions = eng.score_packed(_packed(w))
    pr, ph = w.explicit_pairs()
    pairs_form = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                               pair_read=pr, pair_hap=ph)
    np.testing.assert_array_equal(eng.score_packed(pairs_form), regions)
    small = CudaPairHMM(memory_mb=8, gap=w.gap, ext=w.ext)
    chunked = small.score_packed(_packed(w))
    assert small.last["batches"] > 1
    np.testing.assert_array_equal(chunked, regions)
    chunked_pairs = small.score_packed(pairs_form)
    assert small.last["batches"] > 1
    np.testing.assert_array_equal(chunked_pairs, regions)


def test_pair_list_regrouping_gives_the_region_results():
    """score() on a pair list (validated, deduplicated and regrouped into regions in native
    code) gives the region form's results bit for bit, in any pair order, with repeated pairs
    and reads passed as different objects of equal content."""
    w = S.batched_regions(n_regions=60)
    eng = CudaPairHMM(memory_mb=4096, gap=w.gap, ext=w.ext)
    want = eng.score_packed(_packed(w))
    pairs, idx = [], []
    o = 0
    for g in range(w.n_regions):
        haps = [bytes(w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]).decode()
                for h in range(w.region_hap_off[g], w.region_hap_off[g + 1])]
        for r in range(w.region_read_off[g], w.region_read_off[g + 1]):
            a, b = w.read_off[r], w.read_off[r + 1]
            s = bytes(w.read_bases[a:b]).decode()
            q = bytes(w.read_quals[a:b]) if r % 2 else w.read_quals[a:b].tolist()
            for h in haps:
                pairs.append((s, q, h))
                idx.append(o)
                o += 1
    rng = np.random.default_rng(3)
    extra = rng.integers(0, len(pairs), 500)
    as_bytes = lambda q: q if isinstance(q, bytes) else bytes(np.asarray(q).astype(np.uint8))
    pairs += [(pairs[i][0][:], as_bytes(pairs[i][1]), pairs[i][2]) for i in extra]
    idx += [idx[i] for i in extra]
    perm = rng.permutation(len(pairs))
    got = eng.score([pairs[i] for i in perm])
    np.testing.assert_array_equal(got, want[np.asarray(idx)[perm]])
    assert eng.last["pairs"] == len(pairs)


def test_pair_kernel_tiles_agree():
    """The two tilings of the packed two-read kernels (pair_split 6 and 7: which rows-per-lane
    counts run at 12 or 16 warps per SM) run the same arithmetic: identical results."""
    w = S.batched_regions(n_regions=40)
    eng = native.Engine(0, 4096)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    a = eng.forward(_packed(w), params)[0]
    eng.set_tuning(pair_split=7)
    assert eng.tuning()["pair_split"] == 7
    np.testing.assert_array_equal(eng.forward(_packed(w), params)[0], a)
    with pytest.raises(ValueError):
        eng.set_tuning(pair_split=5)
    eng.close()


def test_pipelined_chunks_agree():
    """vd_forward's pipelined chunks (the first a quarter of the others, each chunk's
    primary tier ordered after the previous one's) give the single-chunk results bit for bit."""
    w = S.batched_regions(n_regions=300)
    eng = native.Engine(0, 8192)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    eng.set_tuning(pipeline_gcells=1_000_000)
    one, st1 = eng.forward(_packed(w), params)
    assert st1.batches == 1
    eng.set_tuning(pipeline_gcells=max(1, w.cells() // 6 // 10**9))
    assert eng.tuning()["pipeline_gcells"] >= 1
    many, stn = eng.forward(_packed(w), params)
    assert stn.batches >= 4 and stn.shared_cells == st1.shared_cells
    np.testing.assert_array_equal(many, one)
    with pytest.raises(ValueError):
        eng.set_tuning(pipeline_gcells=-1)
    eng.close()


def test_pipeline_chunks_with_long_reads_and_long_group():
    """vd_forward on a batch with reads longer than a strip: asking for many pipeline chunks gives
    one here (each chunk keeps at least 8 long-read items per warp, and 300 regions hold far
    fewer), with the single-chunk results bit for bit.  long_group takes 1..8 (0 = 8); another
    grouping of a long read's haplotypes moves its likelihoods within FP32 rounding only."""
    w = S.mixed_length_regions(n_regions=300, workers=1)
    assert (np.diff(w.read_off) > 256).any()
    eng = native.Engine(0, 8192)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    eng.set_tuning(pipeline_gcells=1_000_000)
    one, st1 = eng.forward(_packed(w), params)
    assert st1.batches == 1 and st1.long_strips > 0
    eng.set_tuning(pipeline_gcells=1)
    many, stn = eng.forward(_packed(w), params)
    assert stn.batches == 1
    np.testing.assert_array_equal(many, one)
    for bad in (-1, 9):
        with pytest.raises(ValueError):
            eng.set_tuning(long_group=bad)
    eng.set_tuning(long_group=1)
    assert eng.tuning()["long_group"] == 1
    single, st = eng.forward(_packed(w), params)
    assert st.long_strip_runs >= st.long_strips > st1.long_strips
    finite = np.isfinite(one)
    assert np.array_equal(finite, np.isfinite(single))
    np.testing.assert_allclose(single[finite], one[finite], rtol=0, atol=1e-4)
    eng.close()


def test_plan_graph_replay_is_deterministic():
    w = S.batched_regions(n_regions=16)
    eng = native.Engine(0, 4096)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    plan = eng.plan(_packed(w), params)
    outs = []
    for _ in range(3):
        st = plan.run()
        # two-read kernels (1-2), single reads, drift, FP64, FP64 strips
        assert st.kernel_launches in (4, 5, 6) and st.pairs == w.pairs()
        outs.append(plan.fetch())
    ref, _ = eng.forward(_packed(w), params)
    for o in outs:
        np.testing.assert_array_equal(o, ref)


@pytest.mark.parametrize("anchored", [False, True])
@pytest.mark.parametrize("precision", [native.VD_PRECISION_MIXED, native.VD_PRECISION_FLOAT64])
def test_plain_schedule_gives_identical_results(anchored, precision):
    """VD_SCHEDULE_PLAIN (one pair per item, fixed 8 rows per lane, input order) runs the same
    arithmetic as the batched schedule, so every pair agrees bit for bit; long reads included."""
    w = S.batched_regions(n_regions=40)
    eng = native.Engine(0, 4096)
    batched, _ = native.make_params(w.gap, w.ext, anchored, precision)
    plain, _ = native.make_params(w.gap, w.ext, anchored, precision, schedule=native.VD_SCHEDULE_PLAIN)
    a, st_a = eng.forward(_packed(w), batched)
    b, st_b = eng.forward(_packed(w), plain)
    np.testing.assert_array_equal(a, b)
    assert st_b.work_items == w.pairs() > st_a.work_items
    pr, ph = w.explicit_pairs()
    pairs_form = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                               pair_read=pr, pair_hap=ph)
    np.testing.assert_array_equal(eng.forward(pairs_form, plain)[0], a)
    plan = eng.plan(_packed(w), plain)
    plan.run()
    np.testing.assert_array_equal(plan.fetch(), a)
    plan.close()
    eng.close()


def test_reference_shaped_entry_points():
    """The C-ABI drop-ins for pairhmm_pairs / trie_many / read_haplotype_batch_mode / read_haplotype."""
    lib = native.library()
    d = golden("accel_seed31")
    pairs = golden_pairs(d)
    enc = [(s.encode(), np.ascontiguousarray(q, np.uint8).tobytes(), h.encode()) for s, q, h in pairs]
    count = len(enc)
    reads = (ctypes.c_char_p * count)(*(e[0] for e in enc))
    quals = (ctypes.c_char_p * count)(*(e[1] for e in enc))
    haps = (ctypes.c_char_p * count)(*(e[2] for e in enc))
    rn = (ctypes.c_int * count)(*(len(e[0]) for e in enc))
    hn = (ctypes.c_int * count)(*(len(e[2]) for e in enc))
    for mode, key in [(0, "semiglobal"), (2, "semiglobal"), (1, "anchored")]:
        out = np.empty(count)
        rc = lib.vd_pairhmm_pairs(reads, ctypes.cast(quals, ctypes.POINTER(native.c_u8p)), rn, haps, hn, count, mode,
                                  8, out.ctypes.data_as(native.c_dp))
        assert rc == 0, native.last_error()
        assert_mixed_close(out, d[key])
    # trie_many: reads x haplotypes of single_region at the production constants
    g = golden("single_region_q30")
    nr, nh = len(g["read_off"]) - 1, len(g["hap_off"]) - 1
    rb = [bytes(g["read_bases"][g["read_off"][i]:g["read_off"][i + 1]]) for i in range(nr)]
    qb = [bytes(g["read_quals"][g["read_off"][i]:g["read_off"][i + 1]]) for i in range(nr)]
    hb = [bytes(g["hap_bases"][g["hap_off"][i]:g["hap_off"][i + 1]]) for i in range(nh)]
    out = np.empty(nr * nh)
    cells = ctypes.c_uint64()
    rc = lib.vd_trie_many((ctypes.c_char_p * nr)(*rb), ctypes.cast((ctypes.c_char_p * nr)(*qb),
                          ctypes.POINTER(native.c_u8p)), (ctypes.c_int * nr)(*map(len, rb)), nr,
                          (ctypes.c_char_p * nh)(*hb), (ctypes.c_int * nh)(*map(len, hb)), nh, 0, 0,
                          out.ctypes.data_as(native.c_dp), ctypes.byref(cells))
    assert rc == 0 and cells.value == sum(map(len, rb)) * sum(map(len, hb))
    assert_mixed_close(out, g["semiglobal"])
    # read_haplotype_batch_mode with the benchmark's gap/ext
    q45 = golden("single_region_q45")
    s0 = rb[0]
    q0 = (ctypes.c_ubyte * len(qb[0]))(*qb[0])
    out2 = np.empty(nh)
    lib.vd_read_haplotype_batch_mode(s0, q0, len(s0), (ctypes.c_char_p * nh)(*hb), (ctypes.c_int * nh)(*map(len, hb)),
                                     nh, float(q45["gap"]), float(q45["ext"]), out2.ctypes.data_as(native.c_dp), 0)
    assert_mixed_close(out2, q45["semiglobal"][:nh])
    single = lib.vd_read_haplotype(s0, q0, len(s0), hb[0], len(hb[0]), float(q45["gap"]), float(q45["ext"]))
    assert abs(single - q45["semiglobal"][0]) / LN10 <= 1e-4
    anch = lib.vd_anchored_pairhmm(s0, q0, len(s0), hb[0], len(hb[0]), 0.001, 0.1)
    assert abs(anch - O.forward(s0, qb[0], hb[0], 0.001, 0.1, True, 0)) / LN10 <= 1e-4


def test_score_pairs_and_many_module_api(monkeypatch):
    monkeypatch.setenv("VARDEPTH_PAIRHMM_BACKEND", "cuda")
    reads = ["ACGT" * 8, "A" * 30, "GATTACA"]
    quals = [[30] * len(x) for x in reads]
    haps = ["TT" + r + "GG" for r in reads] + ["ACGT" * 10]
    got = score_many(reads, quals, haps)
    want = np.array([[O.forward(r, np.array(q, np.uint8), h) for h in haps] for r, q in zip(reads, quals)])
    assert got.shape == (3, 4)
    assert_mixed_close(got.ravel(), want.ravel())
    flat = score_pairs([(r, q, h) for r, q in zip(reads, quals) for h in haps])
    np.testing.assert_array_equal(flat, got.ravel())


@pytest.mark.parametrize("rows", [64, 128, 256])
@pytest.mark.parametrize("anchored", [False, True])
def test_long_read_strip_heights(rows, anchored):
    """vd_tuning.long_read_rows: reads over 256 bases in strips of 64/128/256 rows, including
    error-rich ones (8% substitutions at reported Q30) that underflow a 256-row FP32 strip."""
    rng = np.random.default_rng(7 + rows)
    pairs = []
    for n, m, err in [(300, 420, 0.01), (700, 900, 0.08), (1500, 1700, 0.08), (2100, 2300, 0.03), (257, 400, 0.0)]:
        hap = "".join(rng.choice(list("ACGT"), m))
        start = int(rng.integers(0, m - n + 1))
        read = list(hap[start:start + n])
        for i in np.flatnonzero(rng.random(n) < err):
            read[i] = "ACGT"[("ACGT".index(read[i]) + 1) % 4]
        pairs.append(("".join(read), np.full(n, 30, np.uint8), hap))
    want = np.array([O.forward(s, q, h, 0.001, 0.1, anchored) for s, q, h in pairs])
    rb = np.frombuffer("".join(p[0] for p in pairs).encode(), np.uint8)
    rq = np.concatenate([p[1] for p in pairs])
    hb = np.frombuffer("".join(p[2] for p in pairs).encode(), np.uint8)
    ro = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])])
    ho = np.concatenate([[0], np.cumsum([len(p[2]) for p in pairs])])
    idx = np.arange(len(pairs), dtype=np.int32)
    eng = native.Engine(0, 4096)
    eng.set_tuning(long_read_rows=rows)
    assert eng.tuning()["long_read_rows"] == rows
    pk = native.Packed(rb, rq, ro, hb, ho, pair_read=idx, pair_hap=idx)
    for precision in (native.VD_PRECISION_MIXED, native.VD_PRECISION_FLOAT64):
        params, _ = native.make_params(0.001, 0.1, anchored, precision)
        got, st = eng.forward(pk, params)
        if precision == native.VD_PRECISION_FLOAT64:
            np.testing.assert_allclose(got, want, rtol=0, atol=FP64_ATOL_LN * 10)
        else:
            assert_mixed_close(got, want)
            if not anchored:
                # the error-rich reads leave a 256-row FP32 strip's range; the drift tier
                # (per-row power-of-two boosts) resolves them in FP32 at every strip
                # height.  Anchored pairs here force 120+ deletions (likelihoods far below
                # the FP32 range) and are rescued in FP64 by design.
                assert st.rescued_fp64 + st.rescued_robust == 0
                if rows == 256:
                    assert st.rescued_fp32 > 0
    with pytest.raises(ValueError):
        eng.set_tuning(long_read_rows=96)
    eng.close()


def test_autotune_on_a_sample():
    from vardepth_b200 import autotune
    w = S.mixed_length_regions(n_regions=120, workers=1)
    sub = w.subset(autotune.sample_regions(w.region_read_off, w.region_hap_off, fraction=0.5, min_regions=40))
    eng = native.Engine(0, 8192)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    before, _ = eng.forward(_packed(w), params)
    log = []
    best = autotune.autotune(eng, _packed(sub), params, repeats=1, use_cache=False, log=log)
    assert set(autotune.DEFAULT) <= set(best) and len(log) >= 3
    assert {k: eng.tuning()[k] for k in autotune.DEFAULT} == {k: best[k] for k in autotune.DEFAULT}
    after, _ = eng.forward(_packed(w), params)
    assert_mixed_close(after, before)
    # stratified: the long-read knobs on the long-read regions, the others on the short ones
    log = []
    best = autotune.autotune(eng, _packed(w), params, repeats=1, use_cache=False, log=log, stratify=True)
    assert {t["sample"] for t in log} == {"long", "short"}
    assert_mixed_close(eng.forward(_packed(w), params)[0], before)
    eng.close()


def test_region_shards_score_like_the_whole_batch():
    """Each rank's shard (LPT by cells) scored on its own gives the whole batch's values."""
    from vardepth_b200 import shard
    w = S.batched_regions(n_regions=50, seed=9)
    pk = _packed(w)
    eng = native.Engine(0, 4096)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    whole, _ = eng.forward(pk, params)
    full = np.full(pk.n_outputs(), np.nan)
    for part in shard.shard_regions(shard.region_cells(pk), 3):
        sub, pos = shard.subset(pk, part)
        full[pos] = eng.forward(sub, params)[0]
    np.testing.assert_array_equal(full, whole)
    eng.close()


def _prefix_regions(seed):
    """Regions whose haplotypes repeat the previous one's first bases in every pattern the
    two-read kernel distinguishes: a snapshot taken while the previous haplotype streams, one
    kept from the previous haplotype's own start, none (a shorter shared prefix), identical
    haplotypes, a haplotype that is a prefix of the previous one or extends it, a share that
    leaves one column to stream, prefixes below the 32-column minimum, an empty haplotype."""
    rng = np.random.default_rng(seed)
    qf = S._q_standard(rng)

    def snv(h, p):
        h = h.copy()
        h[p] = S.ALPHABET[S.ALPHABET != h[p]][rng.integers(0, 3)]
        return h

    base = S._random_hap(rng, 400)
    chain = [base] + [snv(base, p) for p in (300, 100, 250, 250, 60, 380, 40, 40, 40, 200)]
    b2 = S._random_hap(rng, 300)
    nested = [b2, b2[:200], b2.copy(), b2.copy(), np.concatenate([b2, S._random_hap(rng, 50)])]
    b3 = S._random_hap(rng, 33)
    short = [b3, b3.copy(), snv(S._random_hap(rng, 40), 5), S._random_hap(rng, 20), S._random_hap(rng, 20)]
    b4 = S._random_hap(rng, 250)
    gapped = [b4, np.empty(0, np.uint8), b4.copy(), snv(b4, 120)]
    regions = []
    for haps in (chain, nested, short, gapped, [base]):
        src = [h for h in haps if len(h) > 0]
        nr = int(rng.integers(9, 15))
        lengths = np.repeat(rng.integers(20, 257, nr), 2)[:nr]  # pairs of reads with the same rows per lane
        lengths[0] = 300  # one read longer than a strip (its own items, no sharing)
        reads, quals = S._sim_reads(rng, src, nr, lengths, 0.01, 0.001, qf)
        regions.append((haps, reads, quals))
    return S._assemble("prefixes", regions, S.GAP_Q45, S.EXT_Q10, {"seed": seed})


@pytest.mark.parametrize("max_item_columns", [0, 450])
def test_shared_haplotype_prefixes(max_item_columns):
    """Two-read items start a haplotype past the prefix it shares with the previous haplotype
    of its region; the skipped columns are bit-identical to streaming them (the plain
    schedule shares nothing) and the scores match the FP64 oracle."""
    w = _prefix_regions(77)
    eng = native.Engine(0, 4096)
    eng.set_tuning(max_item_columns=max_item_columns)
    batched, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    plain, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED, schedule=native.VD_SCHEDULE_PLAIN)
    a, st_a = eng.forward(_packed(w), batched)
    b, st_b = eng.forward(_packed(w), plain)
    assert 0 < st_a.shared_cells < st_a.dp_cells and st_b.shared_cells == 0
    np.testing.assert_array_equal(a, b)
    assert_mixed_close(a, _oracle_workload(w))
    plan = eng.plan(_packed(w), batched)
    assert plan.run().shared_cells == st_a.shared_cells
    np.testing.assert_array_equal(plan.fetch(), a)
    plan.close()
    eng.close()


def test_drift_tier_error_rich_long_reads():
    """Long reads at 6% substitution and 2% indel error (the mixed-length workload's long-read regions) leave
    a 256-row FP32 strip's range; the drift tier rescores them in FP32 with per-row
    power-of-two boosts, matching the FP64 oracle, bit-identical under the plain schedule."""
    rng = np.random.default_rng(404)
    qf = S._q_standard(rng)
    regions = []
    for _ in range(2):
        hap0 = S._random_hap(rng, 2600)
        haps = [hap0] + [S._mutate(rng, hap0, 3, 6) for _ in range(2)]
        reads, quals = S._sim_reads(rng, haps, 4, rng.integers(1000, 2400, 4), 0.06, 0.02, qf)
        regions.append((haps, reads, quals))
    w = S._assemble("drift", regions, S.GAP_Q45, S.EXT_Q10, {})
    eng = native.Engine(0, 4096)
    eng.set_tuning(long_mode=native.VD_LONG_SINGLE)  # long reads in the single-read kernel, then the drift tier
    batched, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    plain, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED, schedule=native.VD_SCHEDULE_PLAIN)
    a, st = eng.forward(_packed(w), batched)
    assert st.rescued_fp32 >= 20 and st.rescued_fp64 + st.rescued_robust <= 2
    assert_mixed_close(a, _oracle_workload(w))
    np.testing.assert_array_equal(eng.forward(_packed(w), plain)[0], a)
    eng.close()


def test_drift_tier_one_strip_reads_below_the_fp32_range():
    """Reads of one strip (40-256 bases) carrying 8-36 Q40 mismatches against every
    haplotype: likelihoods 2^-120 .. 2^-540 below a perfect match, many under the primary
    tier's FP32 range.  The drift tier rescores them in FP32 with one boost per read, within
    1e-4 log10 of the FP64 oracle, bit-identical under the plain schedule, with none left to FP64."""
    rng = np.random.default_rng(77)
    regions = []
    for n in (40, 100, 150, 200, 256):
        hap0 = S._random_hap(rng, 420)
        haps = [hap0, S._mutate(rng, hap0, 2, 4)]
        reads, quals = [], []
        for k in range(8, 37, 4):
            a = int(rng.integers(0, 420 - n))
            r = hap0[a:a + n].copy()
            for p in rng.choice(n, size=min(k, n - 1), replace=False):
                r[p] = S.ALPHABET[S.ALPHABET != r[p]][rng.integers(0, 3)]
            reads.append(r)
            quals.append(np.full(n, 40, np.uint8))
        regions.append((haps, reads, quals))
    w = S._assemble("one-strip drift", regions, S.GAP_Q45, S.EXT_Q10, {})
    want = _oracle_workload(w)
    eng = native.Engine(0, 4096)
    batched, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    plain, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED, schedule=native.VD_SCHEDULE_PLAIN)
    got, st = eng.forward(_packed(w), batched)
    assert st.rescued_fp32 >= 20 and st.rescued_fp64 + st.rescued_robust == 0
    assert_mixed_close(got, want)
    np.testing.assert_array_equal(eng.forward(_packed(w), plain)[0], got)
    eng.close()


def _long_read_regions(seed, lengths, err, n_haps):
    """One region per read length: n_haps haplotypes (a base and edited copies of unequal
    lengths) and two reads of that length at substitution rate err (indels err / 4)."""
    rng = np.random.default_rng(seed)
    qf = S._q_standard(rng)
    regions = []
    for n in lengths:
        hap0 = S._random_hap(rng, n + int(rng.integers(100, 600)))
        haps = [hap0] + [S._mutate(rng, hap0, 3, int(rng.integers(1, 11))) for _ in range(n_haps - 1)]
        reads, quals = S._sim_reads(rng, haps, 2, np.full(2, n), err, err / 4, qf)
        regions.append((haps, reads, quals))
    return S._assemble("long", regions, S.GAP_Q45, S.EXT_Q10, {"seed": seed})


@pytest.mark.parametrize("err,n_haps", [(0.08, 3), (0.01, 4)])
def test_long_read_kernel_two_haplotypes_per_warp(err, n_haps):
    """Reads of 257, 1,500 and 10,000 bases in the long-read kernel (one read against up to
    eight haplotypes per warp item, two at a time, per-lane power-of-two boosts, the pairs
    after the first starting from its measured lane decays): within 1e-4 log10 of the FP64
    oracle with no pair left to FP64 and the genotype argmax unchanged, bit-identical under the
    plain schedule.  The same bound and the same plain/batched identity hold for items of two
    and three haplotypes, for the block-per-pair kernel (the CTA's 4 warps split each
    1,024-row strip), for 128-row strips and for the single-read path."""
    w = _long_read_regions(int(err * 1000) + n_haps, [257, 1500, 10000], err, n_haps)
    want = _oracle_workload(w)
    eng = native.Engine(0, 8192)
    batched, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    plain, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED, schedule=native.VD_SCHEDULE_PLAIN)
    got, st = eng.forward(_packed(w), batched)
    assert_mixed_close(got, want)
    assert st.rescued_fp64 + st.rescued_robust == 0 and st.rescued_fp32 == 0
    # every pair of haplotypes (two per pair, up to 8 per item) runs the read's strips at least once
    n_strips = sum(-(-int(n) // 256) * -(-int(w.region_hap_off[g + 1] - w.region_hap_off[g]) // 2)
                   for g in range(w.n_regions)
                   for n in np.diff(w.read_off)[w.region_read_off[g]:w.region_read_off[g + 1]])
    assert st.long_strips == n_strips and st.long_strip_runs >= st.long_strips
    assert _argmax_agree(w, got, want) == (w.n_regions, w.n_regions)
    np.testing.assert_array_equal(eng.forward(_packed(w), plain)[0], got)
    # other strip heights and the single-read path: within the bound, plain still bit-identical
    for rows, mode, group in [(256, native.VD_LONG_BLOCK, 0), (128, native.VD_LONG_BLOCK, 0),
                              (128, native.VD_LONG_WARP, 0), (256, native.VD_LONG_WARP, 2),
                              (256, native.VD_LONG_WARP, 3), (256, native.VD_LONG_SINGLE, 0),
                              (128, native.VD_LONG_SINGLE, 0), (64, native.VD_LONG_WARP, 0)]:
        eng.set_tuning(long_read_rows=rows, long_mode=mode, long_group=group)
        other = eng.forward(_packed(w), batched)[0]
        assert_mixed_close(other, want)
        np.testing.assert_array_equal(eng.forward(_packed(w), plain)[0], other)
    eng.close()


def test_long_reads_against_unrelated_haplotypes():
    """Reads of 300-2,000 bases against random haplotypes of other lengths (likelihoods thousands of
    bits below a perfect match, alignment families trading places across rows): the long-read
    kernel keeps what it holds exactly and hands the rest to the drift and FP64 tiers, every pair
    within 1e-4 log10 of the FP64 oracle, in items of 2 and of 8 haplotypes."""
    rng = np.random.default_rng(2718)
    regions = []
    for n in (300, 700, 1200, 2000):
        haps = [S._random_hap(rng, int(m)) for m in rng.integers(150, 2600, 5)]
        haps[0] = S._random_hap(rng, n + 200)
        reads = [S._random_hap(rng, n)]
        # and one read drawn from the first haplotype at 8% substitutions
        r = haps[0][100:100 + n].copy()
        for i in np.flatnonzero(rng.random(n) < 0.08):
            r[i] = S.ALPHABET[S.ALPHABET != r[i]][rng.integers(0, 3)]
        reads.append(r)
        quals = [rng.choice(S.Q_LEVELS, n).astype(np.uint8) for _ in reads]
        regions.append((haps, reads, quals))
    w = S._assemble("unrelated", regions, S.GAP_Q45, S.EXT_Q10, {})
    want = _oracle_workload(w)
    eng = native.Engine(0, 4096)
    batched, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    for group in (2, 8):
        eng.set_tuning(long_group=group)
        got, st = eng.forward(_packed(w), batched)
        assert_mixed_close(got, want)
        assert st.long_strips > 0
    eng.close()


@pytest.mark.parametrize("mode", ["warp", "block", "single"])
def test_error_rich_long_read_regions_every_long_path(mode):
    """The mixed-length workload's long-read regions (2-8 reads of 1-10 kb at 6% substitution and
    2% indel error, 2-32 haplotypes each): every long-read path within 1e-4 log10 of the FP64
    oracle on every pair, with the genotype argmax unchanged."""
    rng = np.random.default_rng(4242)
    w = S._mixed_regions(rng, 600, S.GAP_Q45, S.EXT_Q10)
    rl = np.diff(w.read_off)
    longest = np.maximum.reduceat(rl, w.region_read_off[:-1])
    sub = w.subset(np.flatnonzero(longest > 256)[:4])
    want = _oracle_workload(sub)
    eng = native.Engine(0, 8192)
    eng.set_tuning(long_mode={"warp": native.VD_LONG_WARP, "block": native.VD_LONG_BLOCK,
                              "single": native.VD_LONG_SINGLE}[mode])
    params, _ = native.make_params(sub.gap, sub.ext, False, native.VD_PRECISION_MIXED)
    got, _ = eng.forward(_packed(sub), params)
    assert_mixed_close(got, want)
    assert _argmax_agree(sub, got, want) == (sub.n_regions, sub.n_regions)
    eng.close()
