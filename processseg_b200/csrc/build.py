"""Builds libpsgcuda.so in-tree (processseg_b200/libpsgcuda.so) with nvcc for
sm_100a. Usage: python processseg_b200/csrc/build.py [--force]"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(PKG, "libpsgcuda.so")
SOURCES = ["psg_cuda.cu", "psg_plan.cpp"]
DEPS = SOURCES + ["psg_device.cuh", "psg_internal.h", "psg_dft_consts.h", os.path.join("..", "..", "include", "psg.h")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    cmd = [NVCC, *FLAGS, "-o", OUT, *[os.path.join(HERE, s) for s in SOURCES]]
    r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libpsgcuda.so")
    with open(os.path.join(HERE, "ptxas.log"), "w") as f:
        f.write(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
