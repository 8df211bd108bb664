"""vd_region_genotypes: the forward pass followed on the device by normalized_rows and the
diploid genotype log-likelihoods of every region, against the reference's own results
(genotypes_seed4242: molecule_rows.py, triangular.py, mixture_general.cpp) and the oracle."""
import numpy as np
import pytest

from conftest import FP64_ATOL_LN, LN10, golden
from oracle import oracle as O
from vardepth_b200 import native
from vardepth_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = native.Engine(0, 4096)
    yield e
    e.close()


def _packed(d):
    return native.Packed(d["read_bases"], d["read_quals"], d["read_off"], d["hap_bases"], d["hap_off"],
                         region_read_off=d["region_read_off"], region_hap_off=d["region_hap_off"])


def _oracle_post(ln, rro, rho, mq, prior):
    vals, cert, gl = [], [], []
    o = 0
    for g in range(len(rro) - 1):
        nr, H = int(rro[g + 1] - rro[g]), int(rho[g + 1] - rho[g])
        v, c = O.normalized_rows(ln[o:o + nr * H].reshape(nr, H), mq[rro[g]:rro[g + 1]])
        vals.append(v.ravel())
        cert.append(c)
        gl.append(O.diploid_gl(v, prior))
        o += nr * H
    return np.concatenate(vals), np.concatenate(cert), gl


@pytest.mark.parametrize("prior,key", [(None, "gl_none"), (0.0, "gl_prior0"), (0.001, "gl_prior001")])
def test_matches_reference_postprocessing(engine, prior, key):
    d = golden("genotypes_seed4242")
    params, _ = native.make_params(d["gap"], d["ext"], False, native.VD_PRECISION_FLOAT64)
    res = engine.region_genotypes(_packed(d), params, d["mapping_quality"], prior)
    np.testing.assert_allclose(res["ln"], d["semiglobal"], rtol=0, atol=FP64_ATOL_LN)
    np.testing.assert_allclose(res["values"], d["values"], rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(res["certainty"], d["certainty"], rtol=1e-7, atol=1e-7)
    want = d[key]
    got = np.concatenate(res["gl"])
    np.testing.assert_allclose(got, want, rtol=1e-8, atol=1e-7)
    # same inputs through the oracle: only the device's exp/log rounding differs
    v, c, gl = _oracle_post(res["ln"], d["region_read_off"], d["region_hap_off"], d["mapping_quality"], prior)
    np.testing.assert_allclose(res["values"], v, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(res["certainty"], c, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got, np.concatenate(gl), rtol=1e-12, atol=1e-10)
    # genotype calls agree with the reference's
    o = 0
    for g in res["gl"]:
        assert np.argmax(g) == np.argmax(want[o:o + len(g)])
        o += len(g)


def test_mixed_precision_calls_and_optional_outputs(engine):
    w = S.batched_regions(n_regions=40, seed=17)
    pk = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                       region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    params, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    mq = np.random.default_rng(3).integers(0, 61, len(w.read_off) - 1).astype(np.uint8)
    full = engine.region_genotypes(pk, params, mq, 0.001)
    lean = engine.region_genotypes(pk, params, mq, 0.001, values=False, certainty=False, ln=False)
    for a, b in zip(full["gl"], lean["gl"]):
        np.testing.assert_array_equal(a, b)
    fw, _ = engine.forward(pk, params)
    np.testing.assert_array_equal(full["ln"], fw)
    want = O.forward_pairs(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off, *w.explicit_pairs(),
                           w.gap, w.ext)
    assert np.max(np.abs(full["ln"] - want)) / LN10 <= 1e-4
    _, _, gl = _oracle_post(want, w.region_read_off, w.region_hap_off, mq, 0.001)
    assert all(np.argmax(a) == np.argmax(b) for a, b in zip(full["gl"], gl))
    assert full["stats"].kernel_launches >= 5
    with pytest.raises(ValueError):
        pr, ph = w.explicit_pairs()
        engine.region_genotypes(native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                                              pair_read=pr, pair_hap=ph), params)


def test_near_tie_guard_rescores_tied_regions_in_fp64(engine):
    """partial_anchor.py:120-133 as a device flag: a region whose haplotypes are all identical ties
    every genotype and is rescored in FP64; a region with a clear call keeps its mixed-precision result."""
    w = S.batched_regions(n_regions=6, seed=21)
    # every haplotype of region 0 is a copy of its first: all its genotypes tie
    haps = [w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]] for h in range(len(w.hap_off) - 1)]
    h0 = w.region_hap_off[0]
    for h in range(h0 + 1, w.region_hap_off[1]):
        haps[h] = haps[h0].copy()
    hap_bases = np.concatenate(haps)
    hap_off = np.concatenate([[0], np.cumsum([len(h) for h in haps])])
    pk = native.Packed(w.read_bases, w.read_quals, w.read_off, hap_bases, hap_off,
                       region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)
    mq = np.full(len(w.read_off) - 1, 60, np.uint8)
    mixed, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_MIXED)
    fp64, _ = native.make_params(w.gap, w.ext, False, native.VD_PRECISION_FLOAT64)
    plain = engine.region_genotypes(pk, mixed, mq, 0.001)
    guarded = engine.region_genotypes(pk, mixed, mq, 0.001, near_tie_guard=True)
    exact = engine.region_genotypes(pk, fp64, mq, 0.001)
    assert guarded["guarded"][0] and guarded["stats"].rescued_fp64 > 0
    for g in range(w.n_regions):
        want = exact if guarded["guarded"][g] else plain
        np.testing.assert_array_equal(guarded["gl"][g], want["gl"][g])
    nr, H = int(w.region_read_off[1]), int(w.region_hap_off[1])
    np.testing.assert_array_equal(guarded["ln"][:nr * H], exact["ln"][:nr * H])
    np.testing.assert_array_equal(guarded["certainty"][:nr], exact["certainty"][:nr])


@pytest.mark.parametrize("prior", [None, 0.0, 0.01])
def test_edge_regions(engine, prior):
    """Regions with one haplotype, with no reads, and with an empty read, against the oracle."""
    rng = np.random.default_rng(4)
    hap = S.ALPHABET[rng.integers(0, 4, 90)]
    reads = [hap[10:60], hap[30:80], np.empty(0, np.uint8), hap[5:45]]
    rb = np.concatenate(reads)
    rq = np.full(len(rb), 30, np.uint8)
    ro = np.concatenate([[0], np.cumsum([len(r) for r in reads])])
    haps = [hap, hap[:70], hap[20:], hap]
    hb = np.concatenate(haps)
    ho = np.concatenate([[0], np.cumsum([len(h) for h in haps])])
    # region 0: reads 0-1 x hap 0 (H = 1); region 1: no reads x haps 1-2; region 2: reads 2-3 x haps 2-3
    rro, rho = [0, 2, 2, 4], [0, 1, 3, 4]
    pk = native.Packed(rb, rq, ro, hb, ho, region_read_off=rro, region_hap_off=rho)
    params, _ = native.make_params(0.001, 0.1, False, native.VD_PRECISION_FLOAT64)
    mq = np.array([60, 20, 60, 5], np.uint8)
    res = engine.region_genotypes(pk, params, mq, prior)
    assert [len(g) for g in res["gl"]] == [1, 3, 1]
    np.testing.assert_allclose(res["gl"][1], np.zeros(3), atol=1e-15)
    v, c, gl = _oracle_post(res["ln"], np.array(rro), np.array(rho), mq, prior)
    for a, b in zip(res["gl"], gl):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    assert np.isneginf(res["ln"][2]) and np.isnan(res["certainty"][2]) == np.isnan(c[2])
