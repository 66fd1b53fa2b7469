"""Builds the sm_100a shared library ``libscft_b200.so`` and the drop-in
executable ``scft_b200`` in-tree with nvcc (no JIT cache, no CPU fallback)."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscft_b200.so")
EXE = os.path.join(HERE, "scft_b200")
def _nvcc() -> str:
    """nvcc from $NVCC, else $CUDA_HOME/bin, else the PATH."""
    if os.environ.get("NVCC"):
        return os.environ["NVCC"]
    home = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if home and os.path.exists(os.path.join(home, "bin", "nvcc")):
        return os.path.join(home, "bin", "nvcc")
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: set NVCC or CUDA_HOME, or put nvcc on the PATH")
    return found


NVCC = _nvcc()
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["scft_ctx.cu", "props_kernels.cu", "field_kernels.cu", "stress_kernels.cu", "noalloc.cu",
              "density_ckpt.cu", "reg64.cu"]
HEADERS = ["common.cuh", "fft.cuh", "kernels.h", "tma.cuh", "reg64.cuh", "step_order.cuh"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "scft_b200.h"))
    if force or _stale(LIB, deps):
        # one nvcc per translation unit, in parallel, then one link
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs, procs = [], []
        for f in CU_SOURCES:
            o = os.path.join(objdir, f.replace(".cu", ".o"))
            objs.append(o)
            cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-c",
                   "-o", o, os.path.join(CSRC, f)]
            if verbose:
                print(" ".join(cmd))
            procs.append(subprocess.Popen(cmd))
        if any(p.wait() != 0 for p in procs):
            raise RuntimeError("nvcc failed")
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    main = os.path.join(CSRC, "scft_main.cpp")
    if os.path.exists(main) and (force or _stale(EXE, [main, LIB])):
        cmd = [NVCC, "-O2", "-std=c++17", *ARCH, "-o", EXE, main, "-L" + HERE, "-lscft_b200",
               "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
