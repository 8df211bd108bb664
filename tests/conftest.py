"""Shared test setup: the gpu marker, the repository on sys.path, golden fixtures."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

LN10 = float(np.log(10.0))
# |delta log10 L| <= 1e-4 per pair for the FP32-scaled path, stated in ln
MIXED_ATOL_LN = 1e-4 * LN10
# the reference's own FP64 CUDA-vs-CPU tolerance (tests/test_accelerator.py:50)
FP64_ATOL_LN = 2e-9


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built CUDA library")


def golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as d:
        return {k: d[k] for k in d.files}


def golden_pairs(d: dict):
    """(read, quals, hap) triples of a pair-form golden fixture."""
    out = []
    for p in range(len(d["pair_read"])):
        r, h = int(d["pair_read"][p]), int(d["pair_hap"][p])
        a, b = d["read_off"][r], d["read_off"][r + 1]
        c, e = d["hap_off"][h], d["hap_off"][h + 1]
        out.append((bytes(d["read_bases"][a:b]).decode(), d["read_quals"][a:b].copy(),
                    bytes(d["hap_bases"][c:e]).decode()))
    return out


@pytest.fixture(scope="session")
def built_library():
    from vardepth_b200 import build
    return build.build()
