"""The gradient checker itself, on the CPU: the long-double expected-count gradient of the
oracle against central finite differences of the FP64 forward restatement (h = 1e-3 on
the Phred-scale parameters), and the the planted-error-model workload simulator's shape."""
import numpy as np
import pytest

from oracle import oracle as O
from vardepth_b200 import synthetic as S


def _pairs(w, k):
    pr, ph = w.explicit_pairs()
    out = []
    for p in range(k):
        r, h = pr[p], ph[p]
        out.append((w.read_bases[w.read_off[r]:w.read_off[r + 1]], w.read_quals[w.read_off[r]:w.read_off[r + 1]],
                    w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]]))
    return out


@pytest.mark.parametrize("anchored", [False, True])
@pytest.mark.parametrize("theta", [(45.0, 10.0, 0.0, 0.0, 0.0, 0.0), (40.0, 8.0, 2.0, -1.0, 0.0, 3.0)])
def test_expected_count_gradient_matches_finite_differences(anchored, theta):
    theta = np.array(theta)
    g, x = O.phred_to_prob(theta[0]), O.phred_to_prob(theta[1])
    for read, qual, hap in _pairs(S.single_region(), 6):
        ln, jac = O.grad(read, qual, hap, g, x, anchored, theta[2:])
        fd = O.fd_grad(read, qual, hap, theta, anchored=anchored)
        assert np.isclose(ln, O.forward(read, qual, hap, g, x, anchored, O.SEMIGLOBAL_ROW_DIVIDE, offsets=theta[2:]),
                          rtol=0, atol=1e-9)
        # central differences carry an O(h^2) truncation error
        np.testing.assert_allclose(jac, fd, rtol=1e-6, atol=1e-7)


def test_low_quality_bases_and_two_sided_emissions():
    rng = np.random.default_rng(5)
    hap = S.ALPHABET[rng.integers(0, 4, 120)]
    read = hap[30:90].copy()
    read[::7] = S.ALPHABET[(np.searchsorted(S.ALPHABET, read[::7]) + 1) % 4]
    qual = rng.integers(1, 12, 60).astype(np.uint8)  # Phred 1 has P(error) > 3/4: two-sided rows
    theta = np.array([38.0, 9.0, 0.7, 0.0, 0.0, 0.0])
    g, x = O.phred_to_prob(theta[0]), O.phred_to_prob(theta[1])
    ln, jac = O.grad(read, qual, hap, g, x, False, theta[2:])
    np.testing.assert_allclose(jac, O.fd_grad(read, qual, hap, theta), rtol=1e-6, atol=1e-7)


def test_batch_gradient_matches_single_pairs():
    w = S.single_region()
    pr, ph = w.explicit_pairs()
    pr, ph = pr[:10], ph[:10]
    theta = np.array([42.0, 9.0, 1.0, -0.5, 0.25, 2.0])
    g, x = O.phred_to_prob(theta[0]), O.phred_to_prob(theta[1])
    ln, jac = O.grad_pairs(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off, pr, ph, g, x,
                           offsets=theta[2:], threads=2)
    for k, (read, qual, hap) in enumerate(_pairs(w, 10)):
        l1, j1 = O.grad(read, qual, hap, g, x, False, theta[2:])
        assert ln[k] == l1
        np.testing.assert_array_equal(jac[k], j1)


def test_planted_simulation_shape():
    w = S.planted_error_model(n_regions=20)
    assert w.meta["planted"] == [40.0, 8.0, 2.0, -1.0, 0.0, 3.0]
    n = np.diff(w.read_off)
    assert n.min() >= 1 and n.max() <= 250
    assert set(np.unique(w.read_quals)) <= {10, 20, 30, 40}
    assert w.n_regions == 20
    # reproducible from the seed
    w2 = S.planted_error_model(n_regions=20)
    np.testing.assert_array_equal(w.read_bases, w2.read_bases)


def test_phred_floor_gives_a_zero_offset_derivative():
    # Phred 0 bases with a negative offset sit on the floor (error 1): no NaN, no offset gradient
    rng = np.random.default_rng(8)
    hap = S.ALPHABET[rng.integers(0, 4, 80)]
    read = hap[10:50].copy()
    qual = np.zeros(40, np.uint8)
    ln, jac = O.grad(read, qual, hap, 1e-4, 0.1, False, np.array([-0.5, 0.0, 0.0, 0.0]))
    assert np.isfinite(ln) and np.all(np.isfinite(jac))
    assert jac[2] == 0.0
