"""Builds the CUDA library ``libbe_b200.so`` (kernels + C ABI) and the ``labeling`` CLI in-tree.

Every ``.cu`` file under ``csrc/`` is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); the shared library links the CUDA runtime
statically so it loads without a CUDA toolkit on the library path.

    python -m labeling_b200.build [--verbose]
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
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libbe_b200.so")
LIB_CHECK = os.path.join(PKG, "libbe_b200_check.so")   # bounds-checked debug build
CLI = os.path.join(PKG, "labeling")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
LIB_SOURCES = ["be_uf2d.cu", "be_uf3d.cu", "be_scan.cu", "be_iter.cu", "be_api.cu",
               "be_batch.cu", "be_server.cu", "be_tune.cu", "be_noalloc.cu", "be_io.cu", "be_slab.cu"]
CLI_SOURCES = ["labeling.cpp", "cli_main.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, checked: bool = False) -> str:
    """Builds libbe_b200.so, or with checked=True the bounds-checked libbe_b200_check.so
    (-DBE_BOUNDS_CHECK: failed index checks are recorded and skipped, see be_check_status)."""
    build_dir = BUILD + ("_check" if checked else "")
    lib_path = LIB_CHECK if checked else LIB
    flags = NVCC_FLAGS + (["-DBE_BOUNDS_CHECK"] if checked else [])
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".hpp"))]
    headers.append(os.path.join(ROOT, "include", "be.h"))
    objs = []
    jobs = []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(build_dir, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([nvcc(), *ARCH, *flags, *extra, "-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda c: _run(c, verbose or ptxas_info), jobs):
            pass
    if jobs or _stale(lib_path, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", lib_path, *objs, "-Xcompiler", "-fPIC"], verbose)
    if checked:
        return lib_path
    cli_srcs = [os.path.join(CSRC, s) for s in CLI_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if len(cli_srcs) == len(CLI_SOURCES) and _stale(CLI, cli_srcs + headers + [LIB]):
        _run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
              *cli_srcs, "-o", CLI, "-L" + PKG, "-lbe_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"],
             verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    ap.add_argument("--checked", action="store_true", help="build the bounds-checked debug library")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.checked))
    sys.exit(0)
