"""Builds libfew_b200.so in-tree with nvcc for sm_100a (B200).

    python -m fastemriwaveforms_b200.build [--force] [--verbose]

The library lands in fastemriwaveforms_b200/lib/ next to the sources, so it
travels with the source tree; it is not installed anywhere else.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIBNAME = "libfew_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

SOURCES = ["api.cu", "plan.cpp", "spline.cu", "modesum.cu", "probe.cu", "noalloc.cu", "adjoint.cu", "mixed.cu",
           "mixed_adjoint.cu", "mixed_phase.cu", "amplitude.cu", "geodesic.cu", "fdsum.cu", "ylm.cu", "modeselect.cu", "aak.cu", "directsum.cu",
           "dopr853.cu"]
HEADERS = ["few_common.cuh", "few_internal.h", "few_tc.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.isfile(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libfew_b200.so")


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "few_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.isfile(LIBPATH):
        return False
    t = os.path.getmtime(LIBPATH)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a (one object per source, in
    parallel) and link them into one shared library."""
    if not force and up_to_date():
        return LIBPATH
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = nvcc_path()
    objdir = os.path.join(LIBDIR, "_build", f"obj{os.getpid()}")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]

    def compile_one(src):
        obj = os.path.join(objdir, src + ".o")
        cmd = [*common, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    log = ""
    for src, (obj, res) in zip(SOURCES, results):
        log += res.stdout + res.stderr
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    tmp = LIBPATH + f".tmp{os.getpid()}"
    link = [nvcc, *ARCH, "-shared", "-o", tmp, *(obj for obj, _ in results), "-lcudart"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_verbose:
        sys.stderr.write(log + res.stdout + res.stderr)
    os.replace(tmp, LIBPATH)
    shutil.rmtree(objdir, ignore_errors=True)
    return LIBPATH


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print registers / spills per kernel")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose, ptxas_verbose=args.ptxas))
