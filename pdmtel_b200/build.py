"""Builds libpdmtel_b200.so in-tree (nvcc for sm_100a, g++ for the host side).

    python -m pdmtel_b200.build [--verbose]

The FP64 kernels of the drop-in path (csrc/pd_exact.cu) are compiled with
-fmad=false so that no multiply-add is contracted: their arithmetic is then
rounded exactly as the reference's C++ rounds it.  The host C++ is compiled
with -ffp-contract=off for the same reason (its MLS and boundary-factor setup
must reproduce the reference bit for bit).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpdmtel_b200.so")
CLI = os.path.join(HERE, "pdmtel_run")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                  "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
            "-Wno-unused-parameter", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

CUDA_UNITS = {
    "pd_exact.cu": ["-fmad=false"],
    "pd_ai.cu": ["-fmad=false"],
    "pd_f32c.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "pd_fast.cu": [],
    "pd_capi.cu": [],
    "pd_adjoint.cu": [],
}
HOST_UNITS = ["host/pd_deck.cpp", "host/pd_setup.cpp", "host/pd_ai_plan.cpp", "host/pdDataManager.cpp",
              "host/pd_host_capi.cpp"]


def _newer(src_list, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 or (verbose and (r.stdout or r.stderr)):
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r


def headers():
    out = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    for d in (CSRC, os.path.join(CSRC, "host")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh", ".hpp"))]
    return out


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = headers()
    objs = []
    for unit, extra in CUDA_UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        if _newer([src] + hdr, obj) or ptxas_info:
            cmd = [NVCC] + NVFLAGS + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
            _run(cmd, verbose or ptxas_info)
        objs.append(obj)
    for unit in HOST_UNITS:
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, os.path.basename(unit).replace(".cpp", ".o"))
        if _newer([src] + hdr, obj):
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    if _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"], verbose)
    main = os.path.join(CSRC, "host", "pdmtel_main.cpp")
    if os.path.exists(main) and _newer([main, LIB], CLI):
        _run([CXX] + CXXFLAGS + [main, "-o", CLI, "-L" + HERE, "-lpdmtel_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
