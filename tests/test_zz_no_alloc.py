"""vd_forward_region_noalloc: the entry point that allocates nothing.

It scores one region (every read against every haplotype) from device buffers
the caller owns, with all scratch in the library's fixed static device array.
Its results must agree with vd_forward on the same region and with the FP64
oracle, within the tests' tolerances: |delta log10 L| <= 1e-4 per pair for
precision 'mixed' and 2e-9 in ln for 'float64', with identical -inf entries,
on two calls in a row (the second call finds the first call's contents still
in the shared array).  A call after the first leaves the device's free memory
unchanged, and host pointers are refused before anything runs.

The file name sorts last so that it also runs after every other test in the
same process; it must pass alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from conftest import FP64_ATOL_LN, LN10
from oracle import oracle as O
from vardepth_b200 import native

pytestmark = pytest.mark.gpu

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def make_region(seed: int, n_reads: int, n_haps: int, anchored: bool):
    """A region of reads sampled from its haplotypes (with errors), a few
    unrelated reads that underflow FP32 and need the FP64 rescue, one empty
    read and one empty haplotype.  Lengths stay within the entry point's
    limits (reads <= 255, haplotypes <= 1023)."""
    rng = np.random.default_rng(seed)
    hap_len = 48 if anchored else 400
    base = rng.choice(BASES, hap_len + 40)
    haps = []
    for h in range(n_haps):
        s = base[rng.integers(0, 20):][:hap_len + int(rng.integers(-8, 9))].copy()
        for _ in range(3):  # a few variants per haplotype
            s[rng.integers(0, len(s))] = rng.choice(BASES)
        haps.append(s)
    haps[n_haps // 2] = np.zeros(0, np.uint8)
    reads, quals = [], []
    for r in range(n_reads):
        src = haps[r % n_haps] if len(haps[r % n_haps]) else haps[0]
        n = int(rng.integers(20, 60)) if anchored else int(rng.integers(60, 256))
        n = min(n, len(src))
        if anchored:
            seq = src[:n].copy()
        else:
            start = int(rng.integers(0, len(src) - n + 1))
            seq = src[start:start + n].copy()
        if r % 17 == 5:  # unrelated read: FP32 underflows, the FP64 tier takes it
            seq = rng.choice(BASES, n)
        q = rng.integers(2, 41, n).astype(np.uint8)
        err = rng.random(n) < 0.02
        seq[err] = rng.choice(BASES, int(err.sum()))
        if r % 23 == 7:
            q[:3] = [0, 1, 2]  # Phred 0/1: the two-sided emission branch
        reads.append(seq)
        quals.append(q)
    reads[3], quals[3] = np.zeros(0, np.uint8), np.zeros(0, np.uint8)
    read_off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    hap_off = np.concatenate([[0], np.cumsum([len(x) for x in haps])]).astype(np.int64)
    return (np.concatenate(reads).astype(np.uint8), np.concatenate(quals).astype(np.uint8), read_off,
            np.concatenate(haps).astype(np.uint8), hap_off)


def expected(region, anchored: bool, precision: int) -> np.ndarray:
    rb, rq, ro, hb, ho = region
    nr, nh = len(ro) - 1, len(ho) - 1
    pk = native.Packed(rb, rq, ro, hb, ho, region_read_off=np.array([0, nr]), region_hap_off=np.array([0, nh]))
    params, _keep = native.make_params(0.001, 0.1, anchored, precision)
    eng = native.Engine(0, 256)
    try:
        out = np.empty(nr * nh, np.float64)
        native.check(native.library().vd_forward(eng.handle, ctypes.byref(pk.batch), ctypes.byref(params),
                                                 out.ctypes.data_as(native.c_dp), None), "vd_forward")
    finally:
        eng.close()
    return out


def oracle_region(region, anchored: bool) -> np.ndarray:
    """The FP64 oracle on every (read, haplotype) pair, reads x haplotypes row-major."""
    rb, rq, ro, hb, ho = region
    nr, nh = len(ro) - 1, len(ho) - 1
    pr = np.repeat(np.arange(nr, dtype=np.int32), nh)
    ph = np.tile(np.arange(nh, dtype=np.int32), nr)
    return O.forward_pairs(rb, rq, ro, hb, ho, pr, ph, 0.001, 0.1, anchored=anchored, threads=0)


def call_noalloc(region, anchored: bool, precision: int, stream=None):
    """Upload the region into caller-owned device buffers and score it."""
    import torch
    rb, rq, ro, hb, ho = region
    nr, nh = len(ro) - 1, len(ho) - 1
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rb, rq, ro, hb, ho)]
    out = torch.full((nr * nh,), 7.0, dtype=torch.float64, device="cuda")  # overwritten by the call
    params, _keep = native.make_params(0.001, 0.1, anchored, precision)
    torch.cuda.synchronize()
    rc = native.library().vd_forward_region_noalloc(
        0, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), nr, dev[3].data_ptr(), dev[4].data_ptr(), nh,
        ctypes.byref(params), out.data_ptr(), stream)
    return rc, out.cpu().numpy()


def assert_agree(got, want, precision):
    assert np.array_equal(np.isneginf(got), np.isneginf(want))
    assert np.all(np.isfinite(got) | np.isneginf(got))
    fin = np.isfinite(want)
    if precision == native.VD_PRECISION_MIXED:
        err = np.abs(got[fin] - want[fin]) / LN10
        assert err.max() <= 1e-4, f"max |dlog10| {err.max():.3e}"
    else:
        np.testing.assert_allclose(got[fin], want[fin], atol=FP64_ATOL_LN, rtol=0)


@pytest.mark.parametrize("precision", [native.VD_PRECISION_MIXED, native.VD_PRECISION_FLOAT64])
@pytest.mark.parametrize("anchored", [False, True])
def test_noalloc_matches_vd_forward_and_the_oracle_twice(anchored, precision):
    region = make_region(11 + int(anchored), 96, 12, anchored)
    want = expected(region, anchored, precision)
    oracle = oracle_region(region, anchored)
    for _ in range(2):  # the second call finds the first call's scratch contents
        rc, got = call_noalloc(region, anchored, precision)
        assert rc == native.VD_OK, native.last_error()
        assert_agree(got, want, precision)
        assert_agree(got, oracle, precision)


def test_noalloc_leaves_free_device_memory_unchanged():
    """After a first call (which loads the kernels), a call changes neither the device's free
    memory (cudaMemGetInfo) nor torch's allocator: all of its scratch is the static array."""
    import torch
    region = make_region(21, 120, 10, False)
    rb, rq, ro, hb, ho = region
    nr, nh = len(ro) - 1, len(ho) - 1
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rb, rq, ro, hb, ho)]
    out = torch.empty(nr * nh, dtype=torch.float64, device="cuda")
    params, _keep = native.make_params(0.001, 0.1, False, native.VD_PRECISION_MIXED)
    lib = native.library()
    args = (0, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), nr, dev[3].data_ptr(), dev[4].data_ptr(),
            nh, ctypes.byref(params), out.data_ptr(), None)
    assert lib.vd_forward_region_noalloc(*args) == native.VD_OK, native.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    assert lib.vd_forward_region_noalloc(*args) == native.VD_OK, native.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert torch.cuda.memory_reserved() == reserved0
    assert_agree(out.cpu().numpy(), oracle_region(region, False), native.VD_PRECISION_MIXED)


def test_noalloc_refuses_host_pointers():
    """Host buffers are refused with VD_EINVAL before anything is enqueued."""
    import torch
    rb, rq, ro, hb, ho = make_region(22, 16, 3, False)
    nr, nh = len(ro) - 1, len(ho) - 1
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rb, rq, ro, hb, ho)]
    out_dev = torch.empty(nr * nh, dtype=torch.float64, device="cuda")
    out_host = np.empty(nr * nh, np.float64)
    params, _keep = native.make_params(0.001, 0.1, False, native.VD_PRECISION_MIXED)
    lib = native.library()
    host_reads = np.ascontiguousarray(rb)
    rc = lib.vd_forward_region_noalloc(0, host_reads.ctypes.data, dev[1].data_ptr(), dev[2].data_ptr(), nr,
                                       dev[3].data_ptr(), dev[4].data_ptr(), nh, ctypes.byref(params),
                                       out_dev.data_ptr(), None)
    assert rc == native.VD_EINVAL and "read_bases" in native.last_error()
    rc = lib.vd_forward_region_noalloc(0, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), nr,
                                       dev[3].data_ptr(), dev[4].data_ptr(), nh, ctypes.byref(params),
                                       out_host.ctypes.data, None)
    assert rc == native.VD_EINVAL and "out" in native.last_error()


def test_noalloc_on_a_caller_stream_after_a_different_region():
    import torch
    big = make_region(5, 300, 16, False)
    small = make_region(6, 40, 5, False)
    s = torch.cuda.Stream()
    for region in (big, small):
        want = expected(region, False, native.VD_PRECISION_MIXED)
        rc, got = call_noalloc(region, False, native.VD_PRECISION_MIXED, stream=s.cuda_stream)
        assert rc == native.VD_OK, native.last_error()
        assert_agree(got, want, native.VD_PRECISION_MIXED)


def test_noalloc_rejects_sizes_beyond_its_limits():
    lib = native.library()
    params, _keep = native.make_params(0.001, 0.1, False, native.VD_PRECISION_MIXED)
    # counts are checked on the host before anything runs
    assert lib.vd_forward_region_noalloc(0, 1, 1, 1, 131073, 1, 1, 1, ctypes.byref(params), 1, None) \
        == native.VD_EINVAL
    assert lib.vd_forward_region_noalloc(0, 1, 1, 1, 64, 1, 1, 4097, ctypes.byref(params), 1, None) \
        == native.VD_EINVAL
    assert lib.vd_forward_region_noalloc(0, 1, 1, 1, 1024, 1, 1, 1024, ctypes.byref(params), 1, None) \
        == native.VD_EINVAL
    assert "split the region" in native.last_error()
    # lengths are checked on the device: a 256-base read, then a 1024-base haplotype
    rb, rq, ro, hb, ho = make_region(8, 20, 4, False)
    long_read = (np.concatenate([rb, np.full(256, 65, np.uint8)]), np.concatenate([rq, np.full(256, 30, np.uint8)]),
                 np.concatenate([ro, [ro[-1] + 256]]).astype(np.int64), hb, ho)
    rc, _ = call_noalloc(long_read, False, native.VD_PRECISION_MIXED)
    assert rc == native.VD_EINVAL and "255" in native.last_error()
    long_hap = (rb, rq, ro, np.concatenate([hb, np.full(1024, 67, np.uint8)]),
                np.concatenate([ho, [ho[-1] + 1024]]).astype(np.int64))
    rc, _ = call_noalloc(long_hap, False, native.VD_PRECISION_MIXED)
    assert rc == native.VD_EINVAL and "1023" in native.last_error()
    # a rejected call leaves the next one correct
    region = (rb, rq, ro, hb, ho)
    rc, got = call_noalloc(region, False, native.VD_PRECISION_MIXED)
    assert rc == native.VD_OK, native.last_error()
    assert_agree(got, expected(region, False, native.VD_PRECISION_MIXED), native.VD_PRECISION_MIXED)
