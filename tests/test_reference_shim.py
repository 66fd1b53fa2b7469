"""The reference-side binding include/density_b200.h: the reference program's
own scft.cu, unchanged, compiles for sm_100a against it and links against
libscft_b200.so.  The build directory gets a density.h that holds only the
include of the shim, and the single-rank mpi.h stand-in that the reference
build recipe also uses.  The reference sources are read from
SCFT_REFERENCE_DIR into a temporary directory, never into the repository; the
test skips where they are absent.  Compile and link only: running the program
needs a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SCFT_REFERENCE_DIR", "/root/reference")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
PKG = os.path.join(ROOT, "scft_string_b200")

MPI_STUB = """#pragma once
#include <stdlib.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
static inline int MPI_Init(void *, void *) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int c) { exit(c); }
"""


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "scft.cu")), reason="reference sources absent")
def test_reference_main_builds_on_the_shim(built_lib, tmp_path):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc absent")
    shutil.copy(os.path.join(REF, "scft.cu"), tmp_path / "scft.cu")
    (tmp_path / "density.h").write_text('#include "density_b200.h"\n')
    (tmp_path / "mpi.h").write_text(MPI_STUB)
    exe = tmp_path / "scft_shim"
    cmd = [NVCC, "-O1", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(tmp_path),
           "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(tmp_path / "scft.cu"), "-L" + PKG,
           "-lscft_b200", "-Xlinker", "-rpath=" + PKG]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-4000:]
    assert exe.exists()
    # the program's undefined symbols that the library resolves are the ABI calls
    nm = subprocess.run(["nm", "-u", str(exe)], capture_output=True, text=True).stdout
    used = sorted({ln.split()[-1] for ln in nm.splitlines() if ln.split()[-1].startswith("scft_")})
    assert used == ["scft_create", "scft_destroy", "scft_last_error", "scft_props_host", "scft_spline_derivs",
                    "scft_spline_redist", "scft_status_string"]
