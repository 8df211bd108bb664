"""The C-ABI library loads and exports every entry point include/vardepth_pairhmm.h declares.

No compute call runs here: on a machine without a GPU, engine creation must
fail loudly (VD_ENODEV -> RuntimeError) rather than fall back to the CPU.
"""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "vardepth_pairhmm.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"\b(vd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_drop_ins():
    names = declared_functions()
    for n in ("vd_pairhmm_pairs", "vd_trie_many", "vd_read_haplotype_batch_mode", "vd_read_haplotype",
              "vd_anchored_pairhmm", "vd_forward", "vd_plan_run"):
        assert n in names


def test_library_exports_every_declared_symbol(built_library):
    lib = ctypes.CDLL(str(built_library))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header(built_library):
    from vardepth_b200 import native
    assert set(declared_functions()) == set(native.SIGNATURES)
    lib = native.library()
    assert lib.vd_version().startswith(b"vardepth-pairhmm-b200")


def test_no_gpu_fails_loudly(built_library):
    from vardepth_b200 import native
    if native.library().vd_device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="GPU"):
        native.Engine(0, 256)
    from vardepth_b200.accelerator import CudaPairHMM
    with pytest.raises(RuntimeError):
        CudaPairHMM()


def test_engine_argument_errors(built_library):
    from vardepth_b200 import native
    lib = native.library()
    h = ctypes.c_void_p()
    assert lib.vd_engine_create(0, 4, ctypes.byref(h)) == native.VD_EINVAL  # budget below 8 MiB
    assert b"8 MiB" in lib.vd_last_error()
    # reference return code 1 for bad arguments (batch_hmm.cpp:194)
    assert lib.vd_pairhmm_pairs(None, None, None, None, None, -1, 0, 0, None) == 1
    assert lib.vd_pairhmm_pairs(None, None, None, None, None, 1, 3, 0, None) == 1
    assert lib.vd_trie_many(None, None, None, -1, None, None, 0, 0, 0, None, None) == 1
    assert lib.vd_pairhmm_pairs(None, None, None, None, None, 0, 0, 0, None) == 0


def test_noalloc_limits_are_checked_on_the_host(built_library):
    from vardepth_b200 import native
    lib = native.library()
    params, _keep = native.make_params(0.001, 0.1, False, native.VD_PRECISION_MIXED)
    # 1024 reads x 1024 haplotypes is beyond the 131072-pair scratch: rejected before any CUDA call
    assert lib.vd_forward_region_noalloc(0, 1, 1, 1, 1024, 1, 1, 1024, ctypes.byref(params), 1, None) \
        == native.VD_EINVAL
    assert b"split the region" in lib.vd_last_error()
    assert lib.vd_forward_region_noalloc(0, None, None, None, 0, None, None, 0, None, None, None) \
        == native.VD_EINVAL
    if lib.vd_device_count() == 0:
        # a valid request with no GPU fails loudly instead of computing on the CPU
        assert lib.vd_forward_region_noalloc(0, 1, 1, 1, 4, 1, 1, 4, ctypes.byref(params), 1, None) \
            == native.VD_ENODEV
