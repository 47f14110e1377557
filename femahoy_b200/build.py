"""Build libfemgpu.so (the CUDA library behind include/femgpu.h) in-tree for sm_100a.

    python -m femahoy_b200.build

Each translation unit is compiled to an object under femahoy_b200/_build/ and linked with nvcc
into femahoy_b200/libfemgpu.so. assemble.cu, noalloc.cu, recover.cu, transient.cu and modes.cu
are compiled with -fmad=false so that the element arithmetic keeps the reference's separate roundings;
hierarchy.cpp with -ffp-contract=off for the same reason.
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
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfemgpu.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
               "-I", INCLUDE, "-I", CSRC]

UNITS = [
    ("assemble.cu", ["-fmad=false"]),
    ("solver.cu", []),
    ("capi.cu", []),
    ("noalloc.cu", ["-fmad=false"]),
    ("server.cu", []),
    ("batch.cu", []),
    ("recover.cu", ["-fmad=false"]),
    ("transient.cu", ["-fmad=false"]),
    ("modes.cu", ["-fmad=false"]),
    ("reactions.cu", ["-fmad=false"]),
    ("coarsen.cu", []),
    ("sparse_direct.cu", []),
    ("dense_eigen.cu", []),
    ("dense_factor.cu", []),
    ("offsets.cu", []),
    ("extrude.cu", ["-fmad=false"]),
    ("boxgrid.cu", ["-fmad=false"]),
    ("pcg.cu", ["-fmad=false"]),
    ("rect.cu", ["-fmad=false"]),
]
CXX_UNITS = [("hierarchy.cpp", ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread"]),
             ("symbolic.cpp", ["-O3", "-std=c++17", "-fPIC"]),
             ("order.cpp", ["-O3", "-std=c++17", "-fPIC", "-pthread"]),
             ("mesh2d.cpp", ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off"]),
             ("prism.cpp", ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off"]),
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(src_files, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in src_files)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    return hs + [os.path.join(INCLUDE, "femgpu.h")]


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for name, extra in UNITS:
        src = os.path.join(CSRC, name)
        obj = os.path.join(OUT, name + ".o")
        objs.append(obj)
        if force or _stale([src] + headers, obj):
            jobs.append([nvcc, *ARCH, *NVCC_COMMON, *extra, "-c", src, "-o", obj])
    for name, flags in CXX_UNITS:
        src = os.path.join(CSRC, name)
        obj = os.path.join(OUT, name + ".o")
        objs.append(obj)
        if force or _stale([src] + headers, obj):
            jobs.append([os.environ.get("CXX", "g++"), *flags, "-I", INCLUDE, "-I", CSRC, "-c",
                         src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for err in ex.map(run, jobs):
            if verbose and err:
                print(err)
    if force or jobs or _stale(objs, LIB):
        # Link beside the library and rename it into place, so that the file is never seen
        # half written.
        tmp = LIB + ".tmp"
        run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lpthread"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
