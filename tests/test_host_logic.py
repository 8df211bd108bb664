"""Host-side logic of the drop-in (no GPU): input guards, packing, backend choice, workloads."""
import numpy as np
import pytest

from vardepth_b200 import accelerator as A
from vardepth_b200 import synthetic as S


def test_input_guards():
    # caller/native/caller/tests/test_accelerator.py:29-32
    for pairs in [[("A", [256], "A")], [("A", [-1], "A")], [("A", [3.5], "A")], [("A", [], "A")], [("X", [30], "A")]]:
        with pytest.raises(ValueError):
            A.validate_pairs(pairs)
    with pytest.raises(ValueError):
        A.score_pairs([("A", [30], "A")], selection="fake")
    with pytest.raises(ValueError):
        A.validate_pairs([("a", [30], "A")])
    with pytest.raises(ValueError):
        A.validate_pairs([("A", [np.nan], "A")])


def test_cpu_backend_is_not_provided():
    with pytest.raises(RuntimeError, match="CPU"):
        A.score_pairs([("A", [30], "A")], selection="cpu")
    with pytest.raises(RuntimeError, match="CPU"):
        A.score_many(["A"], [[30]], ["A"], selection="cpu")


def test_backend_env(monkeypatch):
    monkeypatch.setenv("VARDEPTH_PAIRHMM_BACKEND", "bogus")
    with pytest.raises(ValueError):
        A.backend()
    monkeypatch.setenv("VARDEPTH_PAIRHMM_BACKEND", "auto")
    assert A.backend() == "auto"
    monkeypatch.delenv("VARDEPTH_PAIRHMM_BACKEND")
    assert A.backend() == "cuda"


def test_empty_batches_need_no_device():
    assert A.score_pairs([]).shape == (0,)
    assert A.score_many([], [], ["ACGT"]).shape == (0, 1)
    assert A.score_many(["ACGT"], [[30] * 4], []).shape == (1, 0)


def test_pack_pairs_layout_and_dedupe():
    pairs = A.validate_pairs([("ACNT", [0, 20, 60, 255], "GATTACA"), ("G", [3], "G"), ("TGA", [10, 20, 30], "ACTG"),
                              ("ACNT", [0, 20, 60, 255], "G"), ("", [], "A")])
    pk = A.pack_pairs(pairs)
    assert pk.batch.n_reads == 4 and pk.batch.n_haps == 4      # one ACNT read stored once
    assert list(pk.pair_read) == [0, 1, 2, 0, 3] and list(pk.pair_hap) == [0, 1, 2, 1, 3]
    assert bytes(pk.read_bases).decode() == "ACNTGTGA"
    assert list(pk.read_quals) == [0, 20, 60, 255, 3, 10, 20, 30]
    assert list(pk.read_off) == [0, 4, 5, 8, 8]
    assert bytes(pk.hap_bases).decode() == "GATTACAGACTGA"
    assert pk.n_outputs() == 5
    assert all(a.flags.c_contiguous for a in (pk.read_bases, pk.read_quals, pk.read_off, pk.hap_bases, pk.hap_off))


def test_quality_objects_are_validated_once_and_kept():
    q = bytes([30] * 4)
    out = A.validate_pairs([("ACGT", q, "ACGT"), ("ACGT", q, "TTTT")])
    assert out[0][1] is out[1][1] and out[0][1].dtype == np.uint8


def test_single_region_shape():
    w = S.single_region()
    assert w.n_regions == 1 and len(w.read_off) - 1 == 64 and list(w.hap_lengths()) == [300, 297]
    assert set(np.unique(w.read_quals)) <= {10, 20, 30, 40}
    assert w.pairs() == 128 and w.cells() == 64 * 150 * 597
    assert abs(w.gap - 10 ** -4.5) < 1e-18 and w.ext == 0.1


def test_batched_regions_shape_small():
    w = S.batched_regions(n_regions=40)
    nh = np.diff(w.region_hap_off)
    nr = np.diff(w.region_read_off)
    assert nh.min() >= 2 and nh.max() <= 16 and nr.min() >= 10 and nr.max() <= 500
    rl = w.read_lengths()
    assert rl.min() >= 1 and rl.max() <= 250
    pr, ph = w.explicit_pairs()
    assert len(pr) == w.pairs()
    cells = int(np.sum(rl[pr].astype(np.int64) * w.hap_lengths()[ph]))
    assert cells == w.cells()
    sub = w.subset([3, 1])
    assert sub.n_regions == 2 and sub.pairs() == nr[3] * nh[3] + nr[1] * nh[1]


def test_workloads_are_seeded():
    a, b = S.batched_regions(n_regions=5), S.batched_regions(n_regions=5)
    assert np.array_equal(a.read_bases, b.read_bases) and np.array_equal(a.hap_bases, b.hap_bases)


def _prefix_plan_mirror(haps, min_share=32):
    """The work-list rule of the two-read kernels restated: lexicographic order (shorter first on a
    common prefix, ties in input order); a position shares Q bases with the one before it when the
    snapshot can be laid down while that one streams (Q at or past the column it started from) or
    is still there (Q equal to its share); Q < its length and >= min_share."""
    order = sorted(range(len(haps)), key=lambda i: bytes(haps[i]))
    share, prev = [], -1
    for k, i in enumerate(order):
        q = -1
        if k > 0 and len(haps[i]) > 0 and len(haps[order[k - 1]]) > 0:
            a, b = haps[order[k - 1]], haps[i]
            lim = min(len(a), len(b) - 1)
            l = 0
            while l < lim and a[l] == b[l]:
                l += 1
            if l >= prev + 1:
                q = l
            elif prev >= 0 and l >= prev:
                q = prev
            if q < min_share:
                q = -1
        share.append(q)
        prev = q
    return np.array(order, np.int32), np.array(share, np.int32)


@pytest.mark.parametrize("seed", range(6))
def test_prefix_plan_matches_its_restatement(built_library, seed):
    """vd_prefix_plan (host only): the order and shared-prefix columns of one region's haplotypes
    follow the stated rule on families of edited haplotypes, identical copies, prefixes,
    extensions and empty haplotypes."""
    from vardepth_b200 import native
    rng = np.random.default_rng(seed)
    base = S._random_hap(rng, int(rng.integers(40, 600)))
    haps = [base]
    for _ in range(int(rng.integers(1, 20))):
        kind = rng.integers(0, 6)
        src = haps[int(rng.integers(0, len(haps)))]
        if kind == 0:
            h = src.copy()
        elif kind == 1:
            h = src[:int(rng.integers(0, len(src) + 1))]
        elif kind == 2:
            h = np.concatenate([src, S._random_hap(rng, int(rng.integers(1, 50)))])
        elif kind == 3:
            h = np.empty(0, np.uint8)
        else:
            h = S._mutate(rng, src, int(rng.integers(1, 4)), int(rng.integers(0, 8)))
        haps.append(h)
    off = np.concatenate([[0], np.cumsum([len(h) for h in haps])]).astype(np.int64)
    flat = np.concatenate(haps).astype(np.uint8) if off[-1] else np.zeros(1, np.uint8)
    order, share = native.prefix_plan(flat, off)
    want_order, want_share = _prefix_plan_mirror(haps)
    np.testing.assert_array_equal(order, want_order)
    np.testing.assert_array_equal(share, want_share)
    # every share is a true common prefix of the two neighbours
    for k in range(1, len(order)):
        if share[k] >= 0:
            a, b = haps[order[k - 1]], haps[order[k]]
            assert share[k] < len(b) and np.array_equal(a[:share[k]], b[:share[k]])


def test_prefix_plan_guards(built_library):
    from vardepth_b200 import native
    with pytest.raises(ValueError):
        native.prefix_plan(np.zeros(4, np.uint8), np.array([0, 3, 2], np.int64))
    order, share = native.prefix_plan(np.zeros(1, np.uint8), np.array([0], np.int64))
    assert len(order) == 0 and len(share) == 0


def _folded_forward(read, qual, hap, gap, ext, boost=None):
    """The kernels' folded, row-scaled semiglobal recurrence in float64 (per row i: mu = s_above x
    (hit | miss), om = mu_left + x om, u = mu + X nu, s = mu + K nu + k2 om; row 0 = c; the last
    row's X is alpha f_n, so its u is the scaled M + I), with optional per-row boosts 2^k_i on
    hit, miss, K and X as the drift tier applies them.  Returns ln L."""
    a, alpha = 1.0 - 2.0 * gap, 0.25 * gap
    k1, k2, x4 = (1.0 - ext) * alpha / a, (1.0 - ext) * gap / a, 0.25 * ext
    e = 10.0 ** (-np.minimum(np.asarray(qual, np.float64), 60.0) / 10.0)
    p1, p0 = 1.0 - e, e / 3.0
    mx = np.maximum(p1, p0)
    f = 1.0 / (a * mx)
    hit, miss, K, X = p1 / mx, p0 / mx, k1 * f, x4 * f
    X = X.copy()
    X[-1] = alpha * f[-1]
    k = np.zeros(len(read), np.int64) if boost is None else np.asarray(boost, np.int64)
    scale = np.ldexp(1.0, k)
    hit, miss, K, X = hit * scale, miss * scale, K * scale, X * scale
    c = 2.0 ** 20
    m = len(hap)
    s_prev = np.full(m + 1, c)   # row 0: s and u are c in every column
    u_prev = np.full(m + 1, c)
    hb = np.frombuffer(hap.encode(), np.uint8)
    rb = np.frombuffer(read.encode(), np.uint8)
    for i in range(len(read)):
        match = np.concatenate([[False], hb == rb[i]])   # column 0 has no base
        diag = np.concatenate([[0.0], s_prev[:-1]])
        mu = diag * np.where(match, hit[i], miss[i])
        nu = u_prev
        om = np.zeros(m + 1)
        for j in range(1, m + 1):
            om[j] = mu[j - 1] + ext * om[j - 1]
        u = mu + X[i] * nu
        s = mu + K[i] * nu + k2 * om
        s_prev, u_prev = s, u
    Z = u_prev.sum()
    return np.log(Z) - np.log(c) - np.log(m + 1) + np.sum(np.log(a * mx)) - k.sum() * np.log(2.0)


def test_drift_boosts_cancel_exactly():
    """The drift tier's per-row powers of two leave ln L unchanged: the folded recurrence with
    random boosts 2^k_i (k_i in 0..3) equals the unboosted one, and both equal the FP64 oracle."""
    from oracle import oracle as O
    rng = np.random.default_rng(11)
    for _ in range(4):
        hap = "".join(rng.choice(list("ACGT"), int(rng.integers(30, 80))))
        n = int(rng.integers(10, 40))
        start = int(rng.integers(0, len(hap) - n + 1))
        read = list(hap[start:start + n])
        for i in np.flatnonzero(rng.random(n) < 0.1):
            read[i] = "ACGT"[("ACGT".index(read[i]) + 1) % 4]
        read = "".join(read)
        qual = rng.choice([10, 20, 30, 40], n).astype(np.uint8)
        plain = _folded_forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10)
        boosted = _folded_forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10, boost=rng.integers(0, 4, n))
        want = O.forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10)
        assert abs(boosted - plain) <= 1e-12 * abs(plain)
        assert abs(plain - want) <= 1e-9 * abs(want)


def test_long_kernel_lane_boosts_cancel_exactly():
    """The long-read kernel's boosts: lane L scales everything its first row takes from above by
    2^k_L (folded into that row's hit, miss, K and X), i.e. a per-row boost on every R-th row
    only, with shares of either sign as a re-run's measured lane decays give them.  The folded
    recurrence with such boosts equals the unboosted one and the FP64 oracle."""
    from oracle import oracle as O
    rng = np.random.default_rng(29)
    for R in (4, 8):
        hap = "".join(rng.choice(list("ACGT"), 90))
        n = 60
        read = list(hap[10:10 + n])
        for i in np.flatnonzero(rng.random(n) < 0.08):
            read[i] = "ACGT"[("ACGT".index(read[i]) + 1) % 4]
        read = "".join(read)
        qual = rng.choice([10, 20, 30, 40], n).astype(np.uint8)
        boost = np.zeros(n, np.int64)
        boost[::R] = rng.integers(-20, 41, len(boost[::R]))
        plain = _folded_forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10)
        lanes = _folded_forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10, boost=boost)
        want = O.forward(read, qual, hap, S.GAP_Q45, S.EXT_Q10)
        assert abs(lanes - plain) <= 1e-12 * abs(plain)
        assert abs(plain - want) <= 1e-9 * abs(want)


def _pair_list_mirror(pairs):
    """The regrouping of vd_score_pair_list restated: distinct reads (bases, qualities) and
    haplotypes numbered in order of first appearance; reads asking for the same set of
    haplotypes form a region (regions in order of their first read); a pair's slot is its
    (read, haplotype) cell of its region's reads x haplotypes block, haplotypes in id order."""
    rid, hid, rlist = {}, {}, []
    pr, ph = [], []
    for s, q, h in pairs:
        rk = (s, q if isinstance(q, bytes) else bytes(np.asarray(q).astype(np.uint8)))
        pr.append(rid.setdefault(rk, len(rid)))
        ph.append(hid.setdefault(h, len(hid)))
    sets = [set() for _ in rid]
    for r, h in zip(pr, ph):
        sets[r].add(h)
    region_of, members, hapsets = {}, [], []
    read_region = []
    for r, hs in enumerate(sets):
        key = tuple(sorted(hs))
        if key not in region_of:
            region_of[key] = len(members)
            members.append([])
            hapsets.append(list(key))
        read_region.append(region_of[key])
        members[region_of[key]].append(r)
    off = np.concatenate([[0], np.cumsum([len(m) * len(hs) for m, hs in zip(members, hapsets)])])
    slot = [off[read_region[r]] + members[read_region[r]].index(r) * len(hapsets[read_region[r]])
            + hapsets[read_region[r]].index(h) for r, h in zip(pr, ph)]
    return pr, ph, [read_region[r] for r in pr], slot, len(members), int(off[-1])


def test_pair_list_plan_matches_its_restatement():
    from vardepth_b200 import native
    rng = np.random.default_rng(5)
    haps = ["".join(rng.choice(list("ACGT"), int(rng.integers(1, 40)))) for _ in range(9)] + [""]
    regions = [rng.choice(len(haps), size=int(rng.integers(1, 5)), replace=False) for _ in range(6)]
    pairs = []
    for g, hs in enumerate(regions):
        for _ in range(int(rng.integers(1, 6))):
            n = int(rng.integers(0, 12))
            s = "".join(rng.choice(list("ACGTN"), n))
            q = rng.integers(0, 61, n)
            # the same qualities as bytes, a list, a tuple or a numpy array of another dtype
            q = [bytes(q.astype(np.uint8)), q.tolist(), tuple(int(x) for x in q), q.astype(np.int64)][g % 4]
            for h in hs:
                pairs.append((s, q, haps[h]))
    pairs += pairs[3:7]                                   # repeated pairs
    pairs.append((pairs[0][0][:], list(pairs[0][1]), pairs[0][2]))  # equal content, other objects
    order = rng.permutation(len(pairs))
    pairs = [pairs[i] for i in order]
    got = native.pair_list_plan(pairs)
    pr, ph, preg, slot, ng, nslots = _pair_list_mirror(pairs)
    assert list(got["read"]) == pr and list(got["hap"]) == ph
    assert list(got["region"]) == preg and list(got["slot"]) == slot
    assert got["n_regions"] == ng and got["n_slots"] == nslots


def test_pair_list_validation_messages():
    from vardepth_b200 import native
    cases = [([("ACGT", [30, 30, 30], "A")], "Read/quality lengths differ"),
             ([("ACGT", [30, 30, 30, 256], "A")], "integer Phred"),
             ([("ACGT", [30, 30, 30, 2.5], "A")], "integer Phred"),
             ([("ACGT", np.array([[30, 30], [30, 30]]), "A")], "integer Phred"),
             ([("acgt", [30] * 4, "A")], "Uppercase DNA required"),
             ([("ACGT", [30] * 4, "AXA")], "Uppercase DNA required"),
             ([(b"ACGT", [30] * 4, "A")], "Uppercase DNA required"),
             ([("ACGTé", [30] * 5, "A")], "Uppercase DNA required")]
    for pairs, msg in cases:
        with pytest.raises(ValueError, match=msg):
            native.pair_list_plan(pairs)
    ok = native.pair_list_plan([("ACGTN", b"\x00\x01\x3c\xff\x1e", "N"), ("", b"", "ACGT"), ("A", [0], "")])
    assert ok["n_reads"] == 3 and ok["n_haps"] == 3


def test_autotune_samples_split_long_and_short_regions():
    from vardepth_b200 import autotune, native
    w = S.mixed_length_regions(n_regions=300, workers=1)
    pk = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                       region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    short, long_ = autotune.split_samples(pk, fraction=0.1, min_regions=10, long_items=50, short_items=1)
    longest = lambda p: [int(np.diff(p.read_off)[p.region_read_off[g]:p.region_read_off[g + 1]].max(initial=0))
                         for g in range(len(p.region_read_off) - 1)]
    assert max(longest(short)) <= 256 and min(longest(long_)) > 256
    n_long = sum(1 for v in longest(pk) if v > 256)
    assert 1 <= len(long_.region_read_off) - 1 <= n_long
    assert len(short.region_read_off) - 1 == max(10, round(0.1 * (len(w.region_read_off) - 1 - n_long)))
    # the short sample grows to hold the requested two-read items (half its reads, rounded up per region)
    big, _ = autotune.split_samples(pk, fraction=0.1, min_regions=10, long_items=50, short_items=2000)
    rr = big.region_read_off
    items = sum(int(rr[g + 1] - rr[g]) // 2 + 1 for g in range(len(rr) - 1))
    assert items >= 2000 or len(rr) - 1 == len(w.region_read_off) - 1 - n_long
