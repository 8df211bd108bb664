"""Builds libvardepth_pairhmm.so in-tree for sm_100a (B200).

The four kernel instantiations (FP32/FP64 x semiglobal/anchored) compile in
parallel; a stamp of the sources and flags skips rebuilds when nothing
changed.  Run ``python -m vardepth_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
ROOT = HERE.parent
INCLUDE = ROOT / "include"
LIB = HERE / "libvardepth_pairhmm.so"
OBJ = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
           "--expt-relaxed-constexpr"] + ARCH

UNITS = [
    ("inst_f32_sg", "pairhmm_inst.cu", ["-DVD_FP64=0", "-DVD_ANCH=0"]),
    ("inst_f32_an", "pairhmm_inst.cu", ["-DVD_FP64=0", "-DVD_ANCH=1"]),
    ("inst_f64_sg", "pairhmm_inst.cu", ["-DVD_FP64=1", "-DVD_ANCH=0"]),
    ("inst_f64_an", "pairhmm_inst.cu", ["-DVD_FP64=1", "-DVD_ANCH=1"]),
    ("drift", "pairhmm_drift.cu", []),
    ("long", "pairhmm_long_inst.cu", []),
    ("launch", "pairhmm_launch.cu", []),
    ("host", "pairhmm_host.cu", []),
    ("peak", "pairhmm_peak.cu", []),
    ("noalloc", "pairhmm_noalloc.cu", []),
    ("grad", "pairhmm_grad.cu", []),
    ("genotype", "pairhmm_genotype.cu", []),
    ("pairlist", "pairhmm_pairlist.cu", []),
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libvardepth_pairhmm.so")
    return path


def _fingerprint() -> str:
    h = hashlib.sha256()
    for p in sorted(CSRC.glob("*")) + sorted(INCLUDE.glob("*.h")):
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    h.update(repr(NVFLAGS).encode())
    h.update(repr(UNITS).encode())
    return h.hexdigest()


def _compile(unit, log):
    name, src, defs = unit
    out = OBJ / f"{name}.o"
    cmd = [nvcc(), *NVFLAGS, *defs, f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(out)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    log[name] = proc.stdout + proc.stderr
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{proc.stderr[-4000:]}")
    return out


def build_pairlist(force: bool = False) -> Path:
    """The CPython helper of the pair-list drop-in (csrc/pairlist_py.c -> _pairlist*.so)."""
    import sysconfig
    out = HERE / ("_pairlist" + sysconfig.get_config_var("EXT_SUFFIX"))
    src = CSRC / "pairlist_py.c"
    if not force and out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        raise RuntimeError("a C compiler is required to build vardepth_b200._pairlist")
    tmp = out.with_name(out.name + f".{os.getpid()}.tmp")
    cmd = [cc, "-O2", "-shared", "-fPIC", "-Wall", f"-I{sysconfig.get_paths()['include']}", str(src), "-o", str(tmp)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"building _pairlist failed:\n{proc.stderr[-4000:]}")
    tmp.replace(out)
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile (if needed) and return the path of the shared library."""
    build_pairlist(force)
    stamp = HERE / "libvardepth_pairhmm.sha256"
    fp = _fingerprint()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text().strip() == fp:
        return LIB
    OBJ.mkdir(exist_ok=True)
    log: dict[str, str] = {}
    with ThreadPoolExecutor(max_workers=len(UNITS)) as pool:
        objs = list(pool.map(lambda u: _compile(u, log), UNITS))
    tmp = LIB.with_name(LIB.name + f".{os.getpid()}.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp), "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stderr[-4000:]}")
    tmp.replace(LIB)
    stamp.write_text(fp + "\n")
    (OBJ / "ptxas.log").write_text("\n".join(f"== {k}\n{v}" for k, v in sorted(log.items())))
    if verbose:
        for k, v in sorted(log.items()):
            for line in v.splitlines():
                if "registers" in line or "spill" in line and "0 bytes spill" not in line:
                    print(k, line.strip())
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
