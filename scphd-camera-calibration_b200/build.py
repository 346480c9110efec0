"""Build recipe of the CUDA library: one nvcc invocation for sm_100a, output in-tree
(csrc/libscphd_b200.so) so that it travels with the repository snapshot."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(CSRC, "libscphd_b200.so")
CLI = os.path.join(CSRC, "scphd_calibrate")   # command-line driver (links LIB)
SOURCES = ["scphd_filter.cu", "scphd_server.cu", "scphd_io.cpp"]
DEPS = SOURCES + ["scphd_kernels.cuh", "scphd_device.cuh", "scphd_cli.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", h)
                                                    for h in ("scphd.h", "scphd_io.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB,
           *[os.path.join(CSRC, s) for s in SOURCES], "-lz"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libscphd_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    build_cli()
    return LIB


def build_cli() -> str:
    """The command-line driver: host C++ over the C ABI, rpath to the library beside it."""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), os.path.join(CSRC, "scphd_cli.cpp"),
           "-L", CSRC, "-lscphd_b200", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("g++ failed building scphd_calibrate")
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
