"""The CPU oracle against the golden vectors the reference itself produced.

The fixtures in tests/golden/ come from VarDepth's own Python and C++
(tests/golden/make_golden.py); here the plain-C restatement in
oracle/pairhmm_oracle.c must reproduce them before it is trusted as the
checker of the CUDA path.
"""
import numpy as np
import pytest

from conftest import golden, golden_pairs
from oracle import oracle as O


def _oracle(d, anchored, scaling, extended=False):
    return O.forward_pairs(d["read_bases"], d["read_quals"], d["read_off"], d["hap_bases"], d["hap_off"],
                           d["pair_read"], d["pair_hap"], float(d["gap"]), float(d["ext"]), anchored, scaling,
                           extended, threads=2)


@pytest.mark.parametrize("name", ["accel_seed31", "accel_seed17391"])
def test_restatement_reproduces_reference_cpu_pairs(name):
    d = golden(name)
    # cpu_pairs: wide.cpp read_haplotype (2^512 rescale) and anchored.cpp (row division)
    np.testing.assert_array_equal(_oracle(d, False, O.SEMIGLOBAL_POW2), d["semiglobal"])
    np.testing.assert_array_equal(_oracle(d, True, O.SEMIGLOBAL_ROW_DIVIDE), d["anchored"])


def test_restatement_reproduces_core_pair_scores():
    d = golden("base_seed712")
    np.testing.assert_array_equal(_oracle(d, False, O.SEMIGLOBAL_ROW_DIVIDE), d["semiglobal"])


def test_restatement_reproduces_anchored_catalog():
    d = golden("catalog_seed7713")
    np.testing.assert_array_equal(_oracle(d, True, O.SEMIGLOBAL_ROW_DIVIDE), d["anchored"])
    # the reference's canonical batch mode 1 equals its scalar anchored kernel
    np.testing.assert_array_equal(d["canonical"], d["anchored"])


def test_restatement_edge_cases():
    d = golden("edge_cases")
    np.testing.assert_array_equal(_oracle(d, False, O.SEMIGLOBAL_POW2), d["semiglobal"])
    np.testing.assert_array_equal(_oracle(d, True, O.SEMIGLOBAL_ROW_DIVIDE), d["anchored"])
    # Prepared (read_haplotype_batch_mode lanes) agrees with the scalar path within the reference's 1e-11
    n = int(d["n_prepared"])
    np.testing.assert_allclose(d["prepared"], d["semiglobal"][:n], atol=1e-11, rtol=0)
    assert np.isneginf(O.forward("", b"", "A")) and np.isneginf(O.forward("A", b"\x1e", ""))


def _region_pairs(d):
    return O.region_pairs(d["region_read_off"], d["region_hap_off"])


def test_restatement_single_region_q45_and_production():
    for name in ("single_region_q45", "single_region_q30"):
        d = golden(name)
        pr, ph = _region_pairs(d)
        got = O.forward_pairs(d["read_bases"], d["read_quals"], d["read_off"], d["hap_bases"], d["hap_off"], pr, ph,
                              float(d["gap"]), float(d["ext"]), False, O.SEMIGLOBAL_POW2, threads=2)
        # batch_mode lanes and trie prefix sharing reorder FP64 operations (~1e-13)
        np.testing.assert_allclose(got, d["semiglobal"], atol=1e-11, rtol=0)


def test_extended_precision_agrees():
    d = golden("accel_seed31")
    fp64 = _oracle(d, False, O.SEMIGLOBAL_POW2)
    ld = _oracle(d, False, O.SEMIGLOBAL_POW2, extended=True)
    np.testing.assert_allclose(ld, fp64, atol=1e-9, rtol=0)
    fp64a = _oracle(d, True, O.SEMIGLOBAL_ROW_DIVIDE)
    lda = _oracle(d, True, O.SEMIGLOBAL_ROW_DIVIDE, extended=True)
    np.testing.assert_allclose(lda, fp64a, atol=1e-9, rtol=0)


def test_planted_mistake_is_caught():
    """A checker that cannot fail proves nothing: perturb the oracle's inputs on the CPU."""
    d = golden("accel_seed31")
    bad = dict(d)
    bad["read_quals"] = d["read_quals"].copy()
    bad["read_quals"][5] ^= 7
    with pytest.raises(AssertionError):
        np.testing.assert_array_equal(_oracle(bad, False, O.SEMIGLOBAL_POW2), d["semiglobal"])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
def test_reference_libraries_reproduce_golden():
    d = golden("accel_seed31")
    pairs = golden_pairs(d)
    np.testing.assert_array_equal([O.ref_read_haplotype(s, q, h) for s, q, h in pairs], d["semiglobal"])
    np.testing.assert_array_equal([O.ref_anchored(s, q, h) for s, q, h in pairs], d["anchored"])
    got = O.ref_pairhmm_pairs(pairs, mode=1)
    np.testing.assert_allclose(got, d["anchored"], atol=1e-9, rtol=0)


def test_restatement_reproduces_region_postprocessing():
    """normalized_rows (molecule_rows.py:6-14), _diploid_likelihood_numpy (triangular.py:13-16) and
    mixture_general (mixture_general.cpp:9-37) as the reference computed them (genotypes_seed4242)."""
    d = golden("genotypes_seed4242")
    rro, rho = d["region_read_off"], d["region_hap_off"]
    o = p0 = 0
    for g in range(len(rro) - 1):
        nr, H = int(rro[g + 1] - rro[g]), int(rho[g + 1] - rho[g])
        v, c = O.normalized_rows(d["semiglobal"][o:o + nr * H].reshape(nr, H), d["mapping_quality"][rro[g]:rro[g + 1]])
        np.testing.assert_array_equal(v.ravel(), d["values"][o:o + nr * H])
        np.testing.assert_array_equal(c, d["certainty"][rro[g]:rro[g + 1]])
        P = H * (H + 1) // 2
        np.testing.assert_allclose(O.diploid_gl(v), d["gl_none"][p0:p0 + P], rtol=1e-13, atol=0)
        np.testing.assert_allclose(O.diploid_gl(v, 0.0), d["gl_prior0"][p0:p0 + P], rtol=1e-12, atol=0)
        np.testing.assert_allclose(O.diploid_gl(v, 0.001), d["gl_prior001"][p0:p0 + P], rtol=1e-12, atol=0)
        o += nr * H
        p0 += P
