"""Build libpathed.so (sm_100a kernels + host runtime + C ABI) in-tree.

    python gpu-pathed_b200/build.py          # incremental
    python gpu-pathed_b200/build.py --clean  # from scratch

CUDA sources are compiled with nvcc for sm_100a only; host C++ with g++ and
-ffp-contract=off (the host-side scene arithmetic stays IEEE single without contraction).
Objects go to gpu-pathed_b200/_build/, the library to gpu-pathed_b200/libpathed.so.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpathed.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["wavefront.cu", "guide.cu", "bvh_gpu.cu", "probe.cu"]
# The integrator's kernels are compiled without FMA contraction: every FP32 operation rounds
# on its own, as in the oracle (-ffp-contract=off), so the kernels specialised per material
# class, per batch and per node format compute bit-identical paths (contraction would fuse
# differently in each instantiation), at about 2% of the shade stage's time.
CU_FLAGS = {"wavefront.cu": ["-fmad=false"]}
CPP_SOURCES = ["host_scene.cpp", "bvh_build.cpp", "host_util.cpp", "assets.cpp", "session.cpp", "session_batch.cpp",
               "capi.cpp"]
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] if os.path.isdir(CSRC) else []


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and r.stdout.strip():
        print(r.stdout)
    return r.stdout


def build(verbose: bool = False, clean: bool = False, ptxas_info: bool = False) -> str:
    """Compile every source that changed and relink libpathed.so. Returns the library path."""
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "pathed.h")]
    objs = []
    relink = not os.path.exists(LIB)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer([s] + headers, o):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", *CU_FLAGS.get(src, []), "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            out = _run(cmd, verbose)
            if ptxas_info:
                print(out)
            relink = True
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer([s] + headers, o):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread",
                  "-I", os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o], verbose)
            relink = True
    if relink:
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-lpthread", "-lz"], verbose)
    build_module(verbose, relink)
    return LIB


def build_module(verbose: bool = False, force: bool = False) -> str:
    """The pybind11 module `path_tracer` (the reference GUI's binding surface) over
    libpathed.so, next to it in the package directory."""
    import pybind11

    src = os.path.join(CSRC, "path_tracer_module.cpp")
    out = os.path.join(HERE, "path_tracer" + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [src, LIB, os.path.join(HERE, "..", "include", "pathed.h")]
    if force or _newer(deps, out):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I", pybind11.get_include(),
              "-I", sysconfig.get_paths()["include"], src, "-o", out, "-L", HERE, "-lpathed",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return out


if __name__ == "__main__":
    build(verbose=True, clean="--clean" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print("built", LIB)
