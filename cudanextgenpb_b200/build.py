"""Build the native libraries in-tree.

* ``cudanextgenpb_b200/lib/libpbgpu.so``  – the sm_100a CUDA path (C ABI in include/pbgpu.h)
* ``cudanextgenpb_b200/lib/libpbhost.so`` – the host pb_class mirror (C API in include/pbhost.h)
* ``cudanextgenpb_b200/lib/ngpb``         – command-line driver (same flags as the reference's ngpb)
* ``oracle/lib/liboracle.so``             – the CPU oracle (test infrastructure)

Kernels that reproduce the reference's own floating-point expressions
(markers, density, assembly) are compiled without FMA contraction so their
results match the sequential CPU restatement bit for bit; the Krylov and
energy kernels keep FMA.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cudanextgenpb_b200")
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
LIB = os.path.join(PKG, "lib")
ORACLE = os.path.join(ROOT, "oracle")
BUILD = os.path.join(ROOT, "_build")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
# the system g++ (OpenMP runtime included); PBGPU_CXX overrides
CXX = os.environ.get("PBGPU_CXX") or shutil.which("g++") or "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include")]
NO_FMA = {"k_markers.cu", "k_density.cu", "k_assemble.cu", "k_mesh.cu"}
CXXFLAGS = ["-O3", "-std=c++17", "-fopenmp", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
            "-I" + os.path.join(ROOT, "include")]

GPU_SOURCES = ["pbgpu_api.cu", "k_markers.cu", "k_density.cu", "k_assemble.cu", "k_krylov.cu", "k_energy.cu",
               "k_static.cu", "k_batch.cu", "pbgpu_server.cu", "k_multi.cu", "k_tune.cu", "k_mesh.cu",
               "k_potfield.cu"]
HOST_SOURCES = ["octree.cpp", "surface.cpp", "options.cpp", "pb_class.cpp", "pbhost_capi.cpp", "vtu.cpp"]


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers(d):
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))] + \
        [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]


def build_gpu(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    hdrs = _headers(CSRC)
    objs, jobs = [], []
    for src in GPU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            flags = list(NVFLAGS) + (["-fmad=false"] if src in NO_FMA else [])
            if ptxas_info:
                flags += ["-Xptxas", "-v"]
            jobs.append([NVCC] + ARCH + flags + ["-c", s, "-o", o])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    so = os.path.join(LIB, "libpbgpu.so")
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", so] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"], verbose)
    return so, "\n".join(logs)


def build_host(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers(HOST)
    objs, jobs = [], []
    for src in HOST_SOURCES:
        s = os.path.join(HOST, src)
        o = os.path.join(BUILD, "host_" + src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([CXX] + CXXFLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    so = os.path.join(LIB, "libpbhost.so")
    gpu = os.path.join(LIB, "libpbgpu.so")
    if _stale(so, objs + [gpu]):
        _run([CXX, "-shared", "-fopenmp", "-o", so] + objs +
             ["-L" + LIB, "-lpbgpu", "-Wl,-rpath,$ORIGIN"], verbose)
    exe = os.path.join(LIB, "ngpb")
    main = os.path.join(HOST, "ngpb_main.cpp")
    if os.path.exists(main) and _stale(exe, [main, so]):
        _run([CXX] + CXXFLAGS + [main, "-o", exe, "-L" + LIB, "-lpbhost", "-lpbgpu", "-Wl,-rpath,$ORIGIN"], verbose)
    return so


def build_oracle(verbose=False):
    out = os.path.join(ORACLE, "lib")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "liboracle.so")
    src = os.path.join(ORACLE, "pb_oracle.cpp")
    deps = [src, os.path.join(ORACLE, "pb_oracle.h"), os.path.join(ORACLE, "mc_tri_table.h"),
            os.path.join(ROOT, "include", "pbgpu.h")]
    if _stale(so, deps):
        _run([CXX] + CXXFLAGS + ["-shared", src, "-o", so], verbose)
    return so


def build_all(verbose=False, ptxas_info=False):
    gpu, log = build_gpu(verbose, ptxas_info)
    host = build_host(verbose)
    orc = build_oracle(verbose)
    return {"gpu": gpu, "host": host, "oracle": orc, "ptxas": log}


if __name__ == "__main__":
    res = build_all(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    if "--ptxas" in sys.argv:
        print(res["ptxas"])
    print({k: v for k, v in res.items() if k != "ptxas"})
