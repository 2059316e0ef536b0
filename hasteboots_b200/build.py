"""Build libhb_gpu.so in-tree: CUDA kernels for sm_100a (nvcc) + host client code (g++).

Usage: python -m hasteboots_b200.build [--force]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libhb_gpu.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["hb_api.cu", "hb_serve.cu", "hb_trace.cu"]
CPP_SOURCES = ["hb_client.cpp"]


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "hb_gpu.h")]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _run_all(cmds):
    """Runs the compile commands concurrently; raises if any fails."""
    procs = []
    for cmd in cmds:
        print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])


def build(force=False, verbose_ptxas=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs, cmds = [], []
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        cmds.append([CXX, "-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-fno-fast-math",
                     "-I", "/usr/local/cuda/include", "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    _run_all(cmds)
    tmp = OUT + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread"])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
