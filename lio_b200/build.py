"""Builds lio_b200/libg2g_b200.so in-tree (host C++ + sm_100a CUDA, one C-ABI library).

    python -m lio_b200.build            # incremental
    python -m lio_b200.build --force    # rebuild everything

Host sources are compiled with the system g++ and -ffp-contract=off (the grid
partition must reproduce the reference's FP64 results bit for bit, so no fused
multiply-add may be formed and no -march is given). CUDA sources are compiled
for sm_100a only. The CUDA runtime is linked statically so the library has no
dependency on a particular libcudart.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libg2g_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

HOST_SRCS = ["partition.cpp", "g2g_abi.cpp", "serve.cpp", "batch.cpp"]
CUDA_SRCS = ["engine.cu", "tc_selftest.cu"]
HEADERS = ["system.h", "partition.h", "engine.h", "molecule.h", "xc_functionals.cuh", "umma.cuh", "density_tc.cuh", "fock_tc.cuh", "force_tc.cuh"]

CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fvisibility=hidden",
            "-I" + os.path.join(CUDA_HOME, "include"),
            "-Wall", "-Wextra", "-Wno-unused-parameter"]
NVCCFLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
             "-Xcompiler", "-fPIC,-fvisibility=hidden,-fopenmp", "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], log: list[str]) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd))
    if p.stdout:
        log.append(p.stdout)
    if p.stderr:
        log.append(p.stderr)
    if p.returncode != 0:
        sys.stderr.write("\n".join(log[-3:]) + "\n")
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", h)
                                                       for h in ("g2g.h", "lio_serve.h")]
    objs, log = [], []
    for s in HOST_SRCS:
        src, obj = os.path.join(CSRC, s), os.path.join(OBJ, s + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([CXX, *CXXFLAGS, "-c", src, "-o", obj], log)
        objs.append(obj)
    for s in CUDA_SRCS:
        src, obj = os.path.join(CSRC, s), os.path.join(OBJ, s + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([NVCC, *NVCCFLAGS, "-c", src, "-o", obj], log)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([CXX, "-shared", "-o", LIB, *objs, f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-lrt", "-ldl",
              "-lpthread", "-fopenmp", "-Wl,--no-undefined"], log)
    with open(os.path.join(OBJ, "build.log"), "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
