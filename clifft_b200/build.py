"""Build recipe for the in-tree CUDA library.

    python -m clifft_b200.build          # builds clifft_b200/libclifft_gpu.so

Compiles the sm_100a kernels with nvcc (no JIT cache, no torch extension
machinery) so the shared object lives next to the package and travels with
the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libclifft_gpu.so")

SOURCES = ["clifft_gpu.cu", "svm_kernels_f32.cu", "svm_kernels_f64.cu", "svm_grad.cu", "svm_sample_k.cu"]
HEADERS = ["svm_kernel.cuh", "svm_dispatch.h", "svm_instantiate.cuh", "svm_grad.h", "svm_sample_k.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _inputs():
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps += [os.path.join(ROOT, "include", h) for h in ("clifft_gpu.h", "clifft_program_image.h")]
    deps.append(os.path.abspath(__file__))
    return deps


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(ROOT, "_build", "clifft_b200")
    os.makedirs(objdir, exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *flags, *inc, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    for src, pr in procs:
        if pr.wait() != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs,
                    "-o", OUT + ".tmp"], check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
