"""Build the CUDA library of the critical-point path (libftk2b.so, sm_100a).

Compiles every translation unit under ftk2_b200/csrc with nvcc for
compute_100a/sm_100a into ftk2_b200/_lib/libftk2b.so.  Runs without a GPU
(nvcc cross-compiles).  Incremental: objects are rebuilt when their source or
any header changed.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libftk2b.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


# The checked build: the same sources with the device bounds checks compiled
# in (-DFTK2B_CHECKED: a failed index check sets an error bit and the call
# returns FTK2B_INTERNAL), loaded instead of LIB when FTK2B_CHECKED=1.
CHECKED_DIR = os.path.join(OUT_DIR, "checked")
CHECKED_LIB = os.path.join(CHECKED_DIR, "libftk2b.so")


def build(verbose: bool = False, checked: bool = False) -> str:
    out_dir = CHECKED_DIR if checked else OUT_DIR
    obj_dir = os.path.join(out_dir, "obj")
    lib = CHECKED_LIB if checked else LIB
    flags = NVCC_FLAGS + (["-DFTK2B_CHECKED"] if checked else [])
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0)
    objs = []
    for src in srcs:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmd = [nvcc()] + ARCH + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


DROPIN_SRC = os.path.join(ROOT, "tests", "cpp", "dropin_c1.cpp")
DROPIN_BIN = os.path.join(OUT_DIR, "dropin_c1")


def build_dropin_test(verbose: bool = False) -> str:
    """C++ program using include/ftk2b/engine.hpp exactly like the reference's
    examples use engine.hpp; linked against libftk2b.so (rpath = _lib)."""
    lib = build(verbose)
    if os.path.exists(DROPIN_BIN) and os.path.getmtime(DROPIN_BIN) >= max(
            os.path.getmtime(DROPIN_SRC), os.path.getmtime(lib),
            os.path.getmtime(os.path.join(ROOT, "include", "ftk2b", "engine.hpp"))):
        return DROPIN_BIN
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "oracle", "shim"), DROPIN_SRC, "-o", DROPIN_BIN,
           "-L", OUT_DIR, "-lftk2b", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return DROPIN_BIN


TRACKER_SRC = os.path.join(ROOT, "tests", "cpp", "tracker_run.cpp")
TRACKER_BIN = os.path.join(OUT_DIR, "tracker_run")


def build_tracker_test(verbose: bool = False) -> str:
    """C++ program driving include/ftk2b/feature_tracker.hpp from a YAML
    configuration, as a reference caller drives ftk2::FeatureTracker."""
    lib = build(verbose)
    hdrs = [os.path.join(ROOT, "include", "ftk2b", h) for h in ("engine.hpp", "feature_tracker.hpp",
                                                              "tracking_config.hpp")]
    if os.path.exists(TRACKER_BIN) and os.path.getmtime(TRACKER_BIN) >= max(
            [os.path.getmtime(TRACKER_SRC), os.path.getmtime(lib)] + [os.path.getmtime(h) for h in hdrs]):
        return TRACKER_BIN
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), TRACKER_SRC, "-o", TRACKER_BIN,
           "-L", OUT_DIR, "-lftk2b", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return TRACKER_BIN


CONTOUR_SRC = os.path.join(ROOT, "tests", "cpp", "contour_run.cpp")
CONTOUR_BIN = os.path.join(OUT_DIR, "contour_run")


def build_contour_test(verbose: bool = False) -> str:
    """C++ program running level sets through include/ftk2b/engine.hpp's
    SimplicialEngine<T, ContourPredicate<T>>."""
    lib = build(verbose)
    hdr = os.path.join(ROOT, "include", "ftk2b", "engine.hpp")
    if os.path.exists(CONTOUR_BIN) and os.path.getmtime(CONTOUR_BIN) >= max(
            os.path.getmtime(CONTOUR_SRC), os.path.getmtime(lib), os.path.getmtime(hdr)):
        return CONTOUR_BIN
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), CONTOUR_SRC, "-o", CONTOUR_BIN,
           "-L", OUT_DIR, "-lftk2b", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return CONTOUR_BIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
