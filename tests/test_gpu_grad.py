"""The reverse-wavefront gradient (vd_forward_backward) and its torch.autograd.Function.

Checks, all through the C ABI on the GPU:
  * the Jacobian d ln L / d(Qg, Qx, o0..o3) against the oracle's long-double
    expected-count gradient: the summed gradient d(sum ln L)/d theta within 1e-6
    relative in the mixed (FP32 + FP64) path, every pair within 1e-10 relative in
    the FP64 path, and every pair of the mixed path within 1e-4 of max(|J|, 1e-2);
  * ln L against the forward (|delta log10 L| <= 1e-4) and the oracle;
  * sqrt-L checkpointing and storing every anti-diagonal give identical results;
  * central finite differences (h = 1e-3) of the FP64 forward;
  * the autograd wrapper's backward (grad_output @ Jacobian) and a fit that
    recovers planted parameters.
"""
import numpy as np
import pytest
import torch

from conftest import LN10
from oracle import oracle as O
from vardepth_b200 import autograd as AG
from vardepth_b200 import native
from vardepth_b200 import synthetic as S

pytestmark = pytest.mark.gpu

THETA = np.array([45.0, 10.0, 0.5, -0.7, 0.3, 1.2])


@pytest.fixture(scope="module")
def engine():
    e = native.Engine(0, 4096)
    yield e
    e.close()


def _packed(w):
    return native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off,
                         region_read_off=w.region_read_off, region_hap_off=w.region_hap_off)


def _oracle(w, theta):
    pr, ph = w.explicit_pairs()
    return O.grad_pairs(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off, pr, ph,
                        O.phred_to_prob(theta[0]), O.phred_to_prob(theta[1]), False, theta[2:])


def _fb(engine, packed, theta, precision=native.VD_PRECISION_MIXED, checkpoint=native.VD_CHECKPOINT_SQRT):
    params, _keep = AG.params_from_theta(theta, precision)
    return engine.forward_backward(packed, params, checkpoint)


@pytest.mark.parametrize("theta", [THETA, np.array([40.0, 8.0, 2.0, -1.0, 0.0, 3.0])])
def test_jacobian_matches_expected_count_oracle(engine, theta):
    w = S.batched_regions(n_regions=6)
    lo, jo = _oracle(w, theta)
    ln, jac, st = _fb(engine, _packed(w), theta)
    assert st.failed_pairs == 0 and st.pairs == w.pairs()
    assert np.max(np.abs(ln - lo)) / LN10 <= 1e-4
    total, want = jac.sum(0), jo.sum(0)
    assert np.all(np.abs(total - want) <= 1e-6 * np.abs(want)), (total, want)
    assert np.all(np.abs(jac - jo) <= 1e-4 * np.maximum(np.abs(jo), 1e-2))
    ln64, jac64, st64 = _fb(engine, _packed(w), theta, native.VD_PRECISION_FLOAT64)
    assert st64.fp64_pairs == w.pairs()
    np.testing.assert_allclose(ln64, lo, rtol=0, atol=1e-9)
    np.testing.assert_allclose(jac64, jo, rtol=1e-10, atol=1e-12)
    print(f"pairs {st.pairs} fp64 {st.fp64_pairs} rel err of the summed gradient "
          f"{np.max(np.abs(total - want) / np.abs(want)):.2e}")


def test_ln_matches_forward(engine):
    w = S.batched_regions(n_regions=20)
    params, _keep = AG.params_from_theta(THETA)
    fw, _ = engine.forward(_packed(w), params)
    ln, _, _ = _fb(engine, _packed(w), THETA)
    assert np.max(np.abs(ln - fw)) / LN10 <= 1e-6


@pytest.mark.parametrize("precision", [native.VD_PRECISION_MIXED, native.VD_PRECISION_FLOAT64])
def test_sqrt_checkpointing_equals_storing_every_antidiagonal(engine, precision):
    w = S.batched_regions(n_regions=12)
    a = _fb(engine, _packed(w), THETA, precision, native.VD_CHECKPOINT_SQRT)
    b = _fb(engine, _packed(w), THETA, precision, native.VD_CHECKPOINT_ALL)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2].scratch_bytes * 4 < b[2].scratch_bytes


def test_central_differences(engine):
    w = S.single_region()
    pr, ph = w.explicit_pairs()
    sel = np.arange(0, len(pr), 16)
    pk = native.Packed(w.read_bases, w.read_quals, w.read_off, w.hap_bases, w.hap_off, pair_read=pr[sel],
                       pair_hap=ph[sel])
    _, jac, _ = _fb(engine, pk, THETA, native.VD_PRECISION_FLOAT64)
    for k, p in enumerate(sel):
        r, h = pr[p], ph[p]
        fd = O.fd_grad(w.read_bases[w.read_off[r]:w.read_off[r + 1]], w.read_quals[w.read_off[r]:w.read_off[r + 1]],
                       w.hap_bases[w.hap_off[h]:w.hap_off[h + 1]], THETA)
        np.testing.assert_allclose(jac[k], fd, rtol=1e-6, atol=1e-7)


def test_low_qualities_two_sided_rows_and_floor(engine):
    """Phred 0/1 bases (P(error) > 3/4), offsets that push a bin across that point, and the
    Phred floor at 0, which zeroes the offset derivative."""
    rng = np.random.default_rng(11)
    pairs = []
    for k in range(24):
        m = int(rng.integers(60, 300))
        hap = S.ALPHABET[rng.integers(0, 4, m)]
        n = int(rng.integers(20, min(m, 250)))
        a = int(rng.integers(0, m - n + 1))
        read = hap[a:a + n].copy()
        flip = rng.random(n) < 0.1
        read[flip] = S.ALPHABET[(np.searchsorted(S.ALPHABET, read[flip]) + 1) % 4]
        pairs.append((read, rng.integers(0, 14, n).astype(np.uint8), hap))
    read_off = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])])
    hap_off = np.concatenate([[0], np.cumsum([len(p[2]) for p in pairs])])
    rb = np.concatenate([p[0] for p in pairs])
    rq = np.concatenate([p[1] for p in pairs])
    hb = np.concatenate([p[2] for p in pairs])
    idx = np.arange(len(pairs), dtype=np.int32)
    pk = native.Packed(rb, rq, read_off, hb, hap_off, pair_read=idx, pair_hap=idx)
    for theta in (np.array([42.0, 9.0, 0.4, 0.0, 0.0, 0.0]), np.array([42.0, 9.0, -0.6, 0.5, 0.0, 0.0])):
        lo, jo = O.grad_pairs(rb, rq, read_off, hb, hap_off, idx, idx, O.phred_to_prob(theta[0]),
                              O.phred_to_prob(theta[1]), False, theta[2:])
        ln64, jac64, _ = _fb(engine, pk, theta, native.VD_PRECISION_FLOAT64)
        np.testing.assert_allclose(jac64, jo, rtol=1e-9, atol=1e-10)
        ln, jac, _ = _fb(engine, pk, theta)
        assert np.max(np.abs(ln - lo)) / LN10 <= 1e-4
        assert np.all(np.abs(jac - jo) <= 1e-4 * np.maximum(np.abs(jo), 1e-2))


def _anchored_windows(seed, sites=12, reads=10):
    """Read spans against haplotype windows of about their length, as indel refinement scores them
    (caller/native/caller/indel_refine.py:143-151)."""
    rng = np.random.default_rng(seed)
    rb, rq, hb, ro, ho = [], [], [], [0], [0]
    for _ in range(sites):
        ref = S.ALPHABET[rng.integers(0, 4, 300)]
        p, k = int(rng.integers(120, 180)), int(rng.integers(1, 8))
        alt = np.concatenate([ref[:p], ref[p + k:]]) if rng.random() < 0.5 else \
            np.concatenate([ref[:p], S.ALPHABET[rng.integers(0, 4, k)], ref[p:]])
        for _ in range(reads):
            src = alt if rng.random() < 0.5 else ref
            a = int(rng.integers(10, 80))
            b = int(rng.integers(p + 20, min(p + 110, a + 250)))
            read = src[a:b].copy()
            flip = rng.random(len(read)) < 0.02
            read[flip] = S.ALPHABET[(np.searchsorted(S.ALPHABET, read[flip]) + 1) % 4]
            for hap in (ref, alt):
                rb.append(read)
                rq.append(rng.choice([10, 20, 30, 40], len(read), p=[.05, .15, .5, .3]).astype(np.uint8))
                ro.append(ro[-1] + len(read))
                w = hap[a:b + len(hap) - len(src)]
                hb.append(w)
                ho.append(ho[-1] + len(w))
    idx = np.arange(len(rb), dtype=np.int32)
    return np.concatenate(rb), np.concatenate(rq), np.array(ro), np.concatenate(hb), np.array(ho), idx


def test_anchored_jacobian(engine):
    """The anchored (global) model: ln L of the end cell and its gradient, with the row-0 emulator."""
    rb, rq, ro, hb, ho, idx = _anchored_windows(3)
    pk = native.Packed(rb, rq, ro, hb, ho, pair_read=idx, pair_hap=idx)
    g, x = O.phred_to_prob(THETA[0]), O.phred_to_prob(THETA[1])
    lo, jo = O.grad_pairs(rb, rq, ro, hb, ho, idx, idx, g, x, True, THETA[2:])
    p64, _ = native.make_params(g, x, True, native.VD_PRECISION_FLOAT64, quality_offsets=THETA[2:])
    ln64, jac64, _ = engine.forward_backward(pk, p64)
    np.testing.assert_allclose(ln64, lo, rtol=0, atol=1e-9)
    np.testing.assert_allclose(jac64, jo, rtol=1e-9, atol=1e-10)
    pm, _ = native.make_params(g, x, True, native.VD_PRECISION_MIXED, quality_offsets=THETA[2:])
    ln, jac, st = engine.forward_backward(pk, pm)
    assert np.max(np.abs(ln - lo)) / LN10 <= 1e-4
    total, want = jac.sum(0), jo.sum(0)
    assert np.all(np.abs(total - want) <= 1e-6 * np.abs(want)), (total, want)
    fw, _ = engine.forward(pk, pm)
    assert np.max(np.abs(ln - fw)) / LN10 <= 1e-6
    every = engine.forward_backward(pk, pm, native.VD_CHECKPOINT_ALL)
    np.testing.assert_array_equal(every[1], jac)


def test_empty_inputs_and_argument_errors(engine):
    rb = np.frombuffer(b"ACGTACGT", np.uint8)
    rq = np.full(8, 30, np.uint8)
    hb = np.frombuffer(b"ACGTACGTAC", np.uint8)
    pk = native.Packed(rb, rq, [0, 0, 8], hb, [0, 10, 10], region_read_off=[0, 2], region_hap_off=[0, 2])
    ln, jac, st = _fb(engine, pk, THETA)
    assert np.isneginf(ln[[0, 1, 3]]).all() and np.isfinite(ln[2])
    assert not jac[[0, 1, 3]].any() and jac[2].any()
    long_read = native.Packed(np.full(300, 65, np.uint8), np.full(300, 30, np.uint8), [0, 300], hb, [0, 10],
                              region_read_off=[0, 1], region_hap_off=[0, 1])
    with pytest.raises(ValueError):
        _fb(engine, long_read, THETA)
    params, _keep = native.make_params(0.001, 0.1, True, native.VD_PRECISION_MIXED)
    with pytest.raises(ValueError):
        engine.forward_backward(long_read, params)
    ok = native.Packed(np.full(255, 65, np.uint8), np.full(255, 30, np.uint8), [0, 255], hb, [0, 10],
                       region_read_off=[0, 1], region_hap_off=[0, 1])
    engine.forward_backward(ok, params)  # 255 bases + the row-0 emulator fill one strip


def test_autograd_backward_is_grad_output_times_jacobian(engine):
    w = S.batched_regions(n_regions=4)
    batch = AG.Batch(engine, _packed(w))
    theta = torch.tensor(THETA, dtype=torch.float32, requires_grad=True)
    ln = AG.loglik(theta, batch)
    weights = torch.linspace(0.5, 1.5, ln.numel(), dtype=torch.float64)
    (weights * ln).sum().backward()
    _, jo = _oracle(w, THETA.astype(np.float32).astype(np.float64))
    want = weights.numpy() @ jo
    np.testing.assert_allclose(theta.grad.numpy(), want, rtol=2e-6)
    with torch.no_grad():
        plain = AG.loglik(theta, batch)
    np.testing.assert_allclose(plain.numpy(), ln.detach().numpy(), rtol=0, atol=1e-5)


def test_fit_recovers_planted_parameters(engine):
    """the planted-error-model workload shape at 300 regions: reads simulated at gap-open Q40, gap-continuation Q8 and
    offsets (+2, -1, 0, +3); L-BFGS from Q45 / Q10 / zeros lands within 1 Phred of each."""
    w = S.planted_error_model(n_regions=300)
    batch = AG.Batch(engine, _packed(w))
    hist = []
    theta = AG.fit_error_model(batch, w.region_read_off, w.region_hap_off, [45.0, 10.0, 0, 0, 0, 0], history=hist)
    planted = np.array(w.meta["planted"])
    print("fit", theta.numpy().round(3), "planted", planted, "evaluations", len(hist))
    assert np.all(np.abs(theta.numpy() - planted) <= 1.0), theta
