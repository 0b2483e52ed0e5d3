"""Builds the in-tree CUDA library ``libpigment_mpm.so`` for sm_100a (B200).

    python -m pigment_mixing_b200.build        # or: python pigment_mixing_b200/build.py

nvcc compiles the kernels and the C-ABI host runtime in ``csrc/`` into one shared library
next to this file; the Python package loads it with ctypes.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpigment_mpm.so")
SOURCES = ["pm_kernels.cu", "pm_api.cu", "pm_mlp.cu", "pm_noalloc.cu", "pm_splat.cu", "pm_sampling.cu", "pm_render.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "pigment_mpm.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, "_build", src.replace(".cu", ".o"))
        os.makedirs(os.path.dirname(obj), exist_ok=True)
        cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart", "-ccbin", "/usr/bin/g++"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
