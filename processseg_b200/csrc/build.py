"""Builds libpsgcuda.so in-tree (processseg_b200/libpsgcuda.so) with nvcc for
sm_100a: each source compiles to an object in parallel (the float32 and
float64 pipeline kernels in their own units), then one link.
Usage: python processseg_b200/csrc/build.py [--force]"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(PKG, "libpsgcuda.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["psg_pipe_f32.cu", "psg_recipe_f32.cu", "psg_pipe_f64.cu", "psg_recipe_f64.cu", "psg_cuda.cu",
           "psg_plan.cpp"]
DEPS = SOURCES + ["psg_kernel.cuh", "psg_device.cuh", "psg_internal.h", "psg_dft_consts.h",
                  os.path.join("..", "..", "include", "psg.h")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-Xptxas", "-v"]


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in DEPS)


def _compile(src):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    r = subprocess.run([NVCC, *FLAGS, "-c", "-o", obj, os.path.join(HERE, src)], cwd=HERE,
                       capture_output=True, text=True)
    return src, obj, r


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(len(SOURCES)) as ex:
        results = list(ex.map(_compile, SOURCES))
    log = []
    for src, _, r in results:
        log.append(f"== {src}\n{r.stdout}{r.stderr}")
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    r = subprocess.run([NVCC, *ARCH, "-shared", "-o", OUT, *[o for _, o, _ in results]], cwd=HERE,
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libpsgcuda.so")
    with open(os.path.join(HERE, "ptxas.log"), "w") as f:
        f.write("\n".join(log))
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
