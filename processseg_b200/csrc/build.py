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
TRACE_UNITS = ["psg_trace_f32.cu", "psg_trace_m1944.cu", "psg_trace_m1125.cu", "psg_trace_m3375.cu"]
SOURCES = ["psg_pipe_f32.cu", "psg_recipe_f32.cu", "psg_pipe_f64.cu", "psg_recipe_f64.cu", *TRACE_UNITS,
           "psg_cuda.cu", "psg_plan.cpp"]
PUBLIC = os.path.join("..", "..", "include", "psg.h")
# the headers each unit includes (a unit recompiles when it or one of them changes)
KERNEL_HEADERS = ["psg_kernel.cuh", "psg_device.cuh", "psg_internal.h", "psg_dft_consts.h", "psg_trace.h", PUBLIC]
HEADERS = {src: KERNEL_HEADERS for src in SOURCES}
for _u in TRACE_UNITS:
    HEADERS[_u] = KERNEL_HEADERS + ["psg_trace.cuh"]
HEADERS["psg_plan.cpp"] = ["psg_internal.h", PUBLIC]
DEPS = SOURCES + sorted({h for hs in HEADERS.values() for h in hs})
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-Xptxas", "-v"]


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in DEPS)


def _obj(src):
    return os.path.join(OBJ, os.path.splitext(src)[0] + ".o")


def _unit_stale(src, force):
    obj = _obj(src)
    if force or not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in [src] + HEADERS[src])


class _Done:
    returncode, stdout, stderr = 0, "", "(up to date)\n"


def _compile(args):
    src, force = args
    obj = _obj(src)
    if not _unit_stale(src, force):
        return src, obj, _Done()
    r = subprocess.run([NVCC, *FLAGS, "-c", "-o", obj, os.path.join(HERE, src)], cwd=HERE,
                       capture_output=True, text=True)
    return src, obj, r


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(len(SOURCES)) as ex:
        results = list(ex.map(_compile, [(src, force) for src in SOURCES]))
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
