"""Builds libso3gpu.so in-tree (so3_b200/lib/) for sm_100a with nvcc.

Every translation unit under so3_b200/csrc is compiled in parallel into
so3_b200/_build/ and linked into one shared library with the CUDA runtime
linked statically.  A rebuild happens when any source or header is newer than
the library.  Usage: ``python -m so3_b200.build [--force]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "lib")
OBJ_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(OUT_DIR, "libso3gpu.so")
PEAKS_SRC = os.path.join(PKG, "peaks", "peaks.cu")
PEAKS_LIB = os.path.join(OUT_DIR, "libso3peaks.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return (_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True) + [__file__])


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"] if verbose else []
    else:
        cmd += ["-x", "cu"]  # host sources include the device headers
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build_peaks(force: bool = False) -> str:
    """The benchmark's throughput probes (not part of the product library)."""
    deps = [PEAKS_SRC, os.path.join(CSRC, "tc_sm100.cuh"), __file__]
    if not force and os.path.exists(PEAKS_LIB) and all(
            os.path.getmtime(d) <= os.path.getmtime(PEAKS_LIB) for d in deps):
        return PEAKS_LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = PEAKS_LIB + ".tmp"
    cmd = [NVCC] + ARCH + FLAGS + ["-shared", "-cudart", "static", PEAKS_SRC, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {PEAKS_SRC}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, PEAKS_LIB)
    return PEAKS_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_peaks(force)
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), _sources()))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
