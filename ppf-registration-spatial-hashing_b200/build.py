"""Builds libppf_b200.so in this directory from csrc/ (nvcc for sm_100a).

The hot-path translation units are compiled with the reference's arithmetic
flags (--ftz=true --prec-div=false --prec-sqrt=false, contraction on), which
the bit-exact parity of feature keys and alpha bins depends on.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "ppf_b200"
LIB = PKG / "libppf_b200.so"
# measurement probe used by bench.py (not part of the engine's C ABI)
PEAKS_SRC = PKG / "peaks" / "shared_atomic_peak.cu"
PEAKS_LIB = PKG / "libppf_peaks.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--ftz=true",
    "--prec-div=false",
    "--prec-sqrt=false",
    "-Xcompiler",
    "-fPIC",
    "-I",
    str(ROOT / "include"),
    "-diag-suppress=177",
]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "include")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _needs(obj: Path, src: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "ppf_b200.h"]
    jobs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        if force or _needs(obj, src, headers):
            if src.suffix == ".cu":
                cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            else:
                cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)
    objs = [BUILD / (s.name + ".o") for s in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))]

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, file=sys.stderr)

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(run, jobs))
    if jobs or force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)]
        run(cmd)
    if force or _needs(PEAKS_LIB, PEAKS_SRC, []):
        run([nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", str(PEAKS_SRC), "-o",
             str(PEAKS_LIB)])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
