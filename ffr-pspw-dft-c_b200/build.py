"""Build the engine's shared libraries in-tree for sm_100a.

    python ffr-pspw-dft-c_b200/build.py [--force] [-j N]

Outputs (git-ignored, shipped with the tree):
    ffr-pspw-dft-c_b200/lib/libpspw_gpu.so     the C ABI (include/pspw_gpu.h)
    ffr-pspw-dft-c_b200/lib/libpspw_dropin.so  the reference-signature drop-in

Objects go to _build/ at the repository root.  A source is recompiled when it
or any header it can include is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(ROOT, "_build", "obj")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
                  "--expt-relaxed-constexpr", "-I", INC, "-I", CSRC]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-I", INC,
            "-I", CSRC]

# libpspw_gpu.so
GPU_SOURCES = ["basis.cpp", "cell.cu", "hpsi.cu", "fftpath_f32.cu", "fftpath_f64.cu", "capi.cu",
               "noalloc.cu", "gemm.cu", "heev.cu", "dense.cu", "solvers.cu", "capi_solvers.cu", "nl_tc.cu",
               "scf.cu", "scf_driver.cu", "input.cpp", "geom.cu", "serve.cpp", "batch.cu"]
GPU_LIBS = ["-lcusolver", "-lcublas", "-lcudart"]
# libpspw_dropin.so (links libpspw_gpu.so)
DROPIN_SOURCES = ["dropin.cpp"]


def _headers():
    hs = []
    for d in (CSRC, INC):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                hs.append(os.path.join(d, f))
    return hs


def _stale(src, obj, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers)


def _compile(src, force, headers):
    name = os.path.basename(src)
    obj = os.path.join(OBJ, name + ".o")
    if not force and not _stale(src, obj, headers):
        return obj, None
    if name.endswith(".cu"):
        cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXXFLAGS + ["-I", os.path.join(CUDA, "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def _link(objs, out, extra):
    cmd = [NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-L", os.path.join(CUDA, "lib64")] + extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force=False, jobs=8, verbose=True):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    headers = _headers()
    sources = [s for s in GPU_SOURCES + DROPIN_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    errs = []
    objs = {}
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {ex.submit(_compile, os.path.join(CSRC, s), force, headers): s for s in sources}
        for f in cf.as_completed(futs):
            obj, err = f.result()
            objs[futs[f]] = obj
            if err:
                errs.append(err)
    if errs:
        raise RuntimeError("compilation failed:\n" + "\n".join(errs))
    gpu_objs = [objs[s] for s in GPU_SOURCES if s in objs]
    gpu_so = os.path.join(LIB, "libpspw_gpu.so")
    if force or not os.path.exists(gpu_so) or any(
            os.path.getmtime(o) > os.path.getmtime(gpu_so) for o in gpu_objs):
        _link(gpu_objs, gpu_so, GPU_LIBS)
        if verbose:
            print("built", gpu_so)
    drop_objs = [objs[s] for s in DROPIN_SOURCES if s in objs]
    if drop_objs:
        drop_so = os.path.join(LIB, "libpspw_dropin.so")
        if force or not os.path.exists(drop_so) or any(
                os.path.getmtime(o) > os.path.getmtime(drop_so) for o in drop_objs + [gpu_so]):
            _link(drop_objs, drop_so, ["-L", LIB, "-lpspw_gpu", "-Xlinker", "-rpath,$ORIGIN"])
            if verbose:
                print("built", drop_so)
    return gpu_so


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    try:
        build(a.force, a.j)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
