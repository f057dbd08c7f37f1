"""Build recipe for libcdock_b200.so (sm_100a) -- run `python -m cdocker_b200.build`.

The library is built in-tree (cdocker_b200/libcdock_b200.so) so that it travels with the
repository snapshot; objects go to cdocker_b200/_build/. nvcc cross-compiles for sm_100a
without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcdock_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
              "--expt-relaxed-constexpr"] + ARCH
# the host helpers decide which rotations survive filtering: no contraction, as in the
# reference's host build; C++14 keeps std::random_shuffle
CXX_FLAGS = ["-O2", "-std=c++14", "-fPIC", "-ffp-contract=off", "-Wno-deprecated-declarations",
             "-pthread"]

CU_SOURCES = ["search_kernels.cu", "compat_kernels.cu", "capi.cu", "noalloc.cu", "server.cu", "tc_xpass.cu", "umma_xpass.cu",
              "cluster.cu", "stream_xpass.cu", "hankel_xpass.cu", "receptor_grids.cu"]
CPP_SOURCES = ["host/reference_api.cpp"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cxx() -> str:
    # /usr/bin/g++ is the system compiler nvcc itself uses on this image
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _headers() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(CSRC, "host"), INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def _run(cmd: list[str], log: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = _headers()
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.basename(s).replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([_nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.basename(s).replace(".cpp", ".o"))
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([_cxx()] + CXX_FLAGS + ["-I", INCLUDE, "-c", src, "-o", obj])
    log: list[str] = []
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, log), jobs))
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"], log)
    with open(os.path.join(BUILD, "build.log"), "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
