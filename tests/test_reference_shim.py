"""The reference-side binding include/density_b200.h: the reference program's
own scft.cu, unchanged, compiles for sm_100a against it and links against
libscft_b200.so.  The build directory gets a density.h that holds only the
include of the shim, and the single-rank mpi.h stand-in that the reference
build recipe also uses.  The reference sources are read from
SCFT_REFERENCE_DIR into a temporary directory, never into the repository; the
test skips where they are absent.  Compile and link only: running the program
needs a GPU.  The binding's own host logic (when it makes, reuses and remakes
a context) is checked against a recording fake of the ABI."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SCFT_REFERENCE_DIR", "")
NVCC = os.environ.get("NVCC") or shutil.which("nvcc") or "nvcc"
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


FAKE_ABI = r"""
// records the ABI calls the shim makes; no device
#include <cstdio>
#include <vector>
#include <string>
#include "scft_b200.h"
struct scft_ctx { scft_problem p; };
static std::vector<std::string> calls;
extern "C" {
scft_status scft_create(const scft_problem *p, scft_ctx **out) {
    char b[160];
    snprintf(b, sizeof b, "create N=%d alpha=%g phidb=%g f=%g ens=%d strn=%d m=%d,%d,%d D=%g", p->N, p->alpha, p->phidb,
             p->f, p->ens, p->strn, p->m[0], p->m[1], p->m[2], p->D[0]);
    calls.push_back(b);
    *out = new scft_ctx{*p};
    return SCFT_OK;
}
void scft_destroy(scft_ctx *c) { calls.push_back("destroy"); delete c; }
const char *scft_last_error(const scft_ctx *) { return ""; }
const char *scft_status_string(scft_status) { return "fake"; }
scft_status scft_props_host(scft_ctx *, double *, double *lnQ, int, int Ns, double, double, double *, double f) {
    char b[80];
    snprintf(b, sizeof b, "props N=%d f=%g", Ns, f);
    calls.push_back(b);
    *lnQ = 1.5;
    return SCFT_OK;
}
scft_status scft_spline_derivs(scft_ctx *, const double *x, const double *const *, int, int, const int *, double *const *) {
    char b[64];
    snprintf(b, sizeof b, "derivs x0=%g", x[0]);
    calls.push_back(b);
    return SCFT_OK;
}
scft_status scft_spline_redist(scft_ctx *, const double *x, const double *xref, double *const *, int, int, const int *,
                               double) {
    char b[64];
    snprintf(b, sizeof b, "redist x0=%g xref0=%g", x[0], xref[0]);
    calls.push_back(b);
    return SCFT_OK;
}
}
int m[3] = {8, 6, 4}, N = 20, ens = 1;
double alpha = 0.1, phidb = 0.8;
constexpr int strn = 3;
#include "density_b200.h"
int main() {
    double D[3] = {2.5, 3, 4}, x[3] = {0, 0.5, 1}, xr[3] = {0.25, 0.5, 1}, lnQ, phis[5];
    double w[6] = {0}, *ww[3] = {w, w, w};
    int doiis[3] = {1, 1, 1};
    {
        density d(N, D);
        d.setSplineX(x);
        d.splineDerivsChunked(ww, nullptr, 0, 1, doiis, ww);   // before any props: a context of its own
        d.props(w, &lnQ, 0, N, alpha, phidb, phis, 0.45);      // chain parameters differ: made again
        d.props(w, &lnQ, 1, N, alpha, phidb, phis, 0.45);      // same: reused
        d.setSplineXRef(xr);
        d.splineRedistChunked(ww, x, nullptr, 0, 1, doiis, 0.1);
        d.props(w, &lnQ, 0, N, 0.2, phidb, phis, 0.45);        // other alpha: made again
    }
    for (auto &c : calls) printf("%s\n", c.c_str());
    return lnQ == 1.5 ? 0 : 1;
}
"""


def test_shim_makes_and_reuses_contexts(tmp_path):
    """The binding's own logic against a recording fake of the ABI (host
    only): the context is made by the first call that needs one, made again
    when props brings other chain parameters, reused otherwise; setSplineX /
    setSplineXRef values reach the spline calls that pass NULL."""
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ absent")
    src = tmp_path / "fake.cpp"
    src.write_text(FAKE_ABI)
    exe = tmp_path / "fake"
    out = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-3000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    calls = run.stdout.split("\n")[:-1]
    assert calls == [
        "create N=20 alpha=0 phidb=1 f=0.5 ens=1 strn=3 m=8,6,4 D=2.5",
        "derivs x0=0",
        "destroy",
        "create N=20 alpha=0.1 phidb=0.8 f=0.45 ens=1 strn=3 m=8,6,4 D=2.5",
        "props N=20 f=0.45",
        "props N=20 f=0.45",
        "redist x0=0 xref0=0.25",
        "destroy",
        "create N=20 alpha=0.2 phidb=0.8 f=0.45 ens=1 strn=3 m=8,6,4 D=2.5",
        "props N=20 f=0.45",
        "destroy",
    ], calls
