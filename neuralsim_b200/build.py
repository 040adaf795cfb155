"""Builds the in-tree CUDA library libneuralsim.so for sm_100a with nvcc.

Usage: python -m neuralsim_b200.build   (or build() from Python)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libneuralsim.so")

SOURCES = ["ns_core.cu", "ns_gen.cu", "ns_noalloc.cu", "ns_surrogate.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false",            # one rounding per float op: the drive/neuron spec
    "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
    "-Xptxas", "-v",
]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "neuralsim.h"))
    deps.append(os.path.abspath(__file__))
    if not force and not _newer(LIB, deps):
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-shared", "-o", LIB]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    cmd += ["-lgomp", "-ccbin", "g++"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed building libneuralsim.so")
    with open(os.path.join(HERE, "ptxas_info.txt"), "w") as f:
        f.write(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
