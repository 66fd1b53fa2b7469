#!/usr/bin/env bash
# Builds the reference SCFT_string CUDA program (scft.cu + density.h +
# GPU_kernels.h) from the reference sources for use as a parity oracle and as
# the reference arm of bench.py.  TEST INFRASTRUCTURE ONLY.
#
#   oracle/build_ref.sh STRN [NSTERP] [PRELUDE] [shim]
#
# With the fourth argument `shim`, the reference's density.h and
# GPU_kernels.h are left out: density.h becomes the one-line include of
# include/density_b200.h (the reference-side binding of this library) and
# the program links libscft_b200.so, so the reference's own main loop
# (scft.cu) drives this library's density class.  Output
# oracle/_ref/scft_shim_<tag>; the PROPS trace (printed from the reference's
# density.h) is absent from it.
#
# The sources are copied into a temporary directory (no reference source is
# kept or committed) and patched with sed only where the single-process,
# single-GPU run needs it:
#   * `constexpr int strn = 48;` (scft.cu:35) becomes -DSTRN (compile-time in
#     the reference; every replica count needs its own binary);
#   * `int nsterp=4000;` (scft.cu:1102) and the 5E3 prelude iteration cap
#     (scft.cu:1105) become -DNSTERP / -DPRELUDE;
#   * a single-rank mpi.h stub replaces MPI (one process owns every replica,
#     which is what scft.cu:952-975 computes for numprocs=1);
#   * trace lines (full-precision Q2, QC, lnQ, phis per props call; errs/errs3
#     per string iteration; FEs per FreeE; a monotonic timestamp at the start
#     of every string iteration) are printed to stdout.  They read values the
#     reference already computed and do not change its trajectory.
# The patched copy is compiled from a temporary directory that is removed
# afterwards; only the binary is kept.
# Output: oracle/_ref/scft_ref_s<STRN>_n<NSTERP>_p<PRELUDE>
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${SCFT_REFERENCE_DIR:?set SCFT_REFERENCE_DIR to the directory holding the reference scft.cu}"
STRN="${1:?usage: build_ref.sh STRN [NSTERP] [PRELUDE]}"
NSTERP="${2:-4000}"
PRELUDE="${3:-5000}"
MODE="${4:-ref}"
TAG="s${STRN}_n${NSTERP}_p${PRELUDE}"
OUT="$HERE/_ref/scft_ref_${TAG}"
[ "$MODE" = "shim" ] && OUT="$HERE/_ref/scft_shim_${TAG}"
SRC="$(mktemp -d)"
trap 'rm -rf "$SRC"' EXIT
NVCC="${NVCC:-nvcc}"

if [ ! -f "$REF/scft.cu" ]; then
    echo "reference sources not found at $REF" >&2
    exit 3
fi
mkdir -p "$HERE/_ref"
cp "$REF/scft.cu" "$REF/density.h" "$REF/GPU_kernels.h" "$SRC/"
chmod u+w "$SRC"/*

cat > "$SRC/mpi.h" <<'EOF'
/* single-rank stand-in for MPI: one process owns every replica */
#pragma once
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
EOF

S="$SRC/scft.cu"
D="$SRC/density.h"
# compile-time replica count, iteration caps
sed -i 's/^constexpr int strn = 48;/#include <time.h>\nconstexpr int strn = STRN;/' "$S"
sed -i 's/int nsterp=4000;/int nsterp=NSTERP;/' "$S"
sed -i 's/solve_field0(W, chi, f, D2, ii, 5E3, 1E-4); \/\/solve W_+ before we start/solve_field0(W, chi, f, D2, ii, PRELUDE, 1E-4); \/\/solve W_+ before we start/' "$S"
# traces
sed -i 's|^\(\s*\)//send stuff to host array|\1printf("PROPS %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\\n", Q2, QC, *lnQ, phis[0], phis[1], phis[2], phis[3], phis[4]);\n\1//send stuff to host array|' "$D"
sed -i 's|^\(\s*\)errs3\[0\]=errs\[0\]; errs3\[strn-1\]=errs\[strn-1\];.*$|\1errs3[0]=errs[0]; errs3[strn-1]=errs[strn-1];\n\1printf("ERRS %d", k); for(int _i=0;_i<strn;_i++) printf(" %.17g %.17g", errs[_i], errs3[_i]); printf("\\n");|' "$S"
sed -i 's|^\(\s*\)if(k>=springsteps \&\& doii==-1 \&\& dostring==1) {dospring=0; doredist=1; doperp=1;}|\1{ struct timespec _ts; clock_gettime(CLOCK_MONOTONIC, \&_ts); printf("KSTART %d %.9f\\n", k, _ts.tv_sec + 1e-9 * _ts.tv_nsec); fflush(stdout); }\n&|' "$S"
sed -i 's|^\(\s*\)FEs\[ii\] = FEs0\[ii\] + FEs1\[ii\];|&\n\1printf("FREEE %d %.17g %.17g %.17g\\n", ii, FEs0[ii], FEs1[ii], phctot[ii]);|' "$S"
sed -i 's|^\(\s*\)if (justFE!=1){$|\1{ struct timespec _ts; clock_gettime(CLOCK_MONOTONIC, \&_ts); printf("KEND %.9f\\n", _ts.tv_sec + 1e-9 * _ts.tv_nsec); fflush(stdout); }\n&|' "$S"

for pat in 'constexpr int strn = STRN;' 'int nsterp=NSTERP;' 'PRELUDE, 1E-4' 'printf("PROPS' 'printf("ERRS' 'printf("KSTART' 'printf("FREEE' 'printf("KEND'; do
    if ! grep -q -F "$pat" "$S" "$D"; then
        echo "patch did not apply: $pat" >&2
        exit 4
    fi
done

if [ "$MODE" = "shim" ]; then
    ROOT="$(dirname "$HERE")"
    rm -f "$SRC/GPU_kernels.h"
    echo '#include "density_b200.h"' > "$D"
    "$NVCC" -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
        -DSTRN="$STRN" -DNSTERP="$NSTERP" -DPRELUDE="$PRELUDE" \
        -I"$SRC" -I"$ROOT/include" -o "$OUT" "$S" -L"$ROOT/scft_string_b200" -lscft_b200 \
        -Xlinker -rpath='$ORIGIN/../../scft_string_b200' -w
else
    "$NVCC" -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
        -DSTRN="$STRN" -DNSTERP="$NSTERP" -DPRELUDE="$PRELUDE" \
        -I"$SRC" -o "$OUT" "$S" -lcufft -w
fi
echo "$OUT"
