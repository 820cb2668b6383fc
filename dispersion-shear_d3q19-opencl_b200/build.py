"""Build recipe of the native parts, in-tree:

  lib/libd3q19_b200.so   CUDA kernels + C ABI (nvcc, sm_100a, static cudart)
  lib/libd3q19_b200_checked.so   the same with -DD3Q19_BOUNDS_CHECK=1 (device index
                         checks that record D3Q19_EBOUNDS instead of faulting)
  lib/libd3q19_host.so   C host routines (parser, initial state, outputs)
  bin/d3q19_b200         the simulation program (drop-in for the reference's binary)

Usage: python build.py [--force]
"""
import concurrent.futures
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
CUDA_LIB = os.path.join(LIB, "libd3q19_b200.so")
CHECKED_LIB = os.path.join(LIB, "libd3q19_b200_checked.so")
HOST_LIB = os.path.join(LIB, "libd3q19_host.so")
MAIN = os.path.join(BIN, "d3q19_b200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SRC = [os.path.join(PKG, "csrc", f) for f in ("d3q19_kernels.cu", "d3q19_api.cu", "d3q19_exact.cu", "d3q19_tma.cu")]
# Translation units compiled without floating-point contraction: the
# reference-exact arithmetic.
NO_CONTRACT = {"d3q19_exact.cu"}
OBJ = os.path.join(PKG, "_build")
CU_HDR = [os.path.join(PKG, "csrc", "d3q19_internal.h"), os.path.join(PKG, "csrc", "d3q19_device.cuh"),
          os.path.join(REPO, "include", "d3q19_b200.h")]
HOST_SRC = [os.path.join(PKG, "host", "d3q19_host.c")]
HOST_HDR = [os.path.join(PKG, "host", "d3q19_host.h"), os.path.join(REPO, "include", "d3q19_b200.h")]
MAIN_SRC = [os.path.join(PKG, "host", "d3q19_main.c")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _cuda_lib(target, objdir, defines, force, verbose_ptxas):
    if not (force or _stale(target, CU_SRC + CU_HDR + [__file__])):
        return
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src in CU_SRC:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"] + defines + ["-c", "-o", obj,
                                                                                                   src]
        if os.path.basename(src) in NO_CONTRACT:
            cmd.insert(1, "--fmad=false")
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    # The translation units are independent: compile them concurrently.
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        list(ex.map(_run, cmds))
    _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", target] + objs)


def build(force: bool = False, verbose_ptxas: bool = False, checked: bool = True):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    jobs = [(CUDA_LIB, OBJ, [])]
    if checked:
        jobs.append((CHECKED_LIB, os.path.join(OBJ, "checked"), ["-DD3Q19_BOUNDS_CHECK=1"]))
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        list(ex.map(lambda j: _cuda_lib(*j, force, verbose_ptxas), jobs))
    if force or _stale(HOST_LIB, HOST_SRC + HOST_HDR + [__file__]):
        _run(["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-Wall", "-Wno-unused-result", "-o", HOST_LIB]
             + HOST_SRC + ["-lm"])
    if force or _stale(MAIN, MAIN_SRC + HOST_SRC + HOST_HDR + [CUDA_LIB, __file__]):
        _run(["gcc", "-O2", "-std=gnu11", "-Wall", "-Wno-unused-result", "-o", MAIN] + MAIN_SRC + HOST_SRC
             + ["-L" + LIB, "-ld3q19_b200", "-Wl,-rpath,$ORIGIN/../lib", "-lm", "-lstdc++", "-lpthread", "-ldl",
                "-lrt"])
    return CUDA_LIB, HOST_LIB, MAIN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
