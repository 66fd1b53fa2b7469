// kernels.h -- launch interfaces between the host solver (scft_ctx.cu) and the
// sm_100a kernels (props_kernels.cu, field_kernels.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace scft {

// per-replica scalar record in device memory (doubles)
enum {
    kRsQ2 = 0,
    kRsQC = 1,
    kRsLnQ = 2,
    kRsZB = 3,
    kRsZC = 4,
    kRsPhis = 5,  // 5 values
    kRsDev2 = 10, // sum over M of (chi*(phiA+phiB-1))^2 of the last props
    kRsStride = 16
};

// Arguments of every propagator kernel (passed by value).
template <typename T>
struct PropsArgs {
    Geo g;
    const int *slot_rep;    // slot -> replica index
    const double *W;        // [rep][2M]  W-, W+
    double *conc;           // [rep][4M]  phiA, phiB, phih, phicB
    double *rs;             // [rep][kRsStride]
    T *etab;                // [slot][2][M]  exp(-wA ds/4), exp(-wB ds/4)
    T *hist;                // [slot][Ns+1][2][M]  q(s), q^dagger(s)
    cplx<T> *spec;          // [slot][2 fields][2 spectra][Mk]
    T *pbuf;                // [slot][2][M]  E2 * full-step result
    const cplx<T> *tw;      // twiddles: x (m0) | y (m1) | z (m2)
    const T *kfac;          // per-axis diffusion factors: x (m0) | y (m1) | z (mk2), per replica
    int kf_stride;          // elements between replicas' factor blocks (0: one shared box)
    double *partials;       // [slot][npart_stride]
    int npart_stride;
    T invM, Mreal;
    double chi, phic, alpha;
    int ens;
    int *err;               // device error word (launch-geometry / plan errors)
    int slot0;              // first slot of this launch within the spectra tensor map
    T *jtab;                // [slot][M]  junction-step E4 (continuous A fraction only)
    int *sync;              // claim and completion counters of the persistent step kernel (reg64.cu)
};

struct PropsLaunch {
    int slab_threads, slab_smem;
    int pencil_threads, pencil_smem;
    int ew_blocks;   // elementwise grid (per slot)
    int red_blocks;  // reduction grid (per slot)
    int big;         // FFT kernels need more than 256 threads per CTA
    int fixed;       // compile-time shape id (0: runtime-shaped kernels)
    int pf;          // prefetching (bulk-copy) slab kernels for the fixed shape
    int mid_pf_smem, combine_pf_smem;
    int tma_pencil;  // x pass through 2-D tensor-map tiles (fixed shapes)
    int pencil_tma_smem;
    const CUtensorMap *tmap;  // host copy of the spectrum tensor map
    int ptile_wide;  // tensor-map x pass with tiles of twice the default width
    int pencil_tma_smem_wide;
    const CUtensorMap *tmap_wide;  // the same spectra with the wide tile box
    int pencil_sh;   // m0 = 64: x pass as register transforms with warp-shuffle transposes (k_pencil_sh);
                     // tmap and tmap_wide are then the 128-byte-swizzled map of 128-byte boxes
    int reg;         // 64^3 FP32: register-resident step kernels (reg64.cu) instead of the shared-memory ones
    int persist;     // one persistent launch per contour step instead of four (register kernels, or the
                     // shared-memory kernels of the compile-time shapes)
    int step_grid;   // CTAs of the register kernels' persistent launch
    int step_grid_pf, step_pf_smem;  // CTAs and dynamic shared memory of the shared-memory kernels' one
};

// register-resident 64^3 FP32 step kernels (reg64.cu)
bool reg64_applicable(int m0, int m1, int m2);
int reg64_set_smem();
void reg64_combine(const PropsArgs<float> &a, int nslots, int s, int mode, cudaStream_t st);
void reg64_mid(const PropsArgs<float> &a, int nslots, int s, cudaStream_t st);
void reg64_pencil(const PropsArgs<float> &a, int nslots, int both, cudaStream_t st);
int reg64_sync_ints(int Ns, int nslots);
int reg64_step_grid();
void reg64_step(const PropsArgs<float> &a, int nslots, int s, int grid, cudaStream_t st);

void pf_smem_bytes(int id, int fp32, int &mid, int &comb);
// dynamic shared memory of k_pencil_sh for tiles of tc columns
int pencil_sh_smem_bytes(int fp32, int tc, int m0);

int fixed_shape_id(int m0, int m1, int m2);
int fixed_shape_threads(int id);

template <typename T>
int launch_props(const PropsArgs<T> &a, const PropsLaunch &L, int nslots, cudaStream_t st);
template <typename T>
int launch_single_step(const PropsArgs<T> &a, const PropsLaunch &L, int s, cudaStream_t st);
template <typename T>
int set_props_smem(const PropsLaunch &L);
// CTAs of the persistent step kernel of the compile-time shapes (0: none)
template <typename T>
int props_step_grid(const PropsLaunch &L);
// chain segment of slot 0 (a.g.Ns steps; a.g.n1, n2 relative to the segment
// start), E tables of slot 0 from its replica, Q2/QC/lnQ of slot 0 from the
// store slices a.g.Ns (q) and a.g.Nh (q^dagger)
template <typename T>
int launch_chain(const PropsArgs<T> &a, const PropsLaunch &L, int first_mode, cudaStream_t st);
template <typename T>
int launch_prepare(const PropsArgs<T> &a, const PropsLaunch &L, cudaStream_t st);
template <typename T>
int launch_qsums(const PropsArgs<T> &a, const PropsLaunch &L, cudaStream_t st);
// one bounded wait on a barrier that nothing completes: error 3 after `polls` polls
int launch_wait_selftest(int *err, unsigned polls, cudaStream_t st);

// ------------------------------------------------------------------ stress (adjoint)
constexpr int kStressPairs = 16;

struct StressPairs {
    int n;
    int xs[kStressPairs], xf[kStressPairs];  // slice s and field (0 q, 1 q^dagger) of x
    int ys[kStressPairs], yf[kStressPairs];  // of the adjoint y
    int sel[kStressPairs];                   // E table of the step (0 A, 1 B)
};

template <typename T>
struct StressArgs {
    Geo g;
    int slot;
    const T *hist, *etab;
    const cplx<T> *tw;
    const T *kfac;
    cplx<T> *S4, *S2, *S4p;  // [pair][x,y][Mk]
    double *part;            // [pair][9][ntiles]
    double L[3];
    T invM;
    int *err;
    const T *jtab;           // [slot][M] junction-step E4 (table 2), continuous A fraction only
    T *rbuf;                 // [6][M] real work arrays of the junction derivative
    const double *wminus;    // W- of the replica (junction derivative)
};

template <typename T>
int launch_stress_chunk(const StressArgs<T> &a, const StressPairs &P, int slab_threads, int slab_smem,
                        int pencil_threads, int pencil_smem, double *out, cudaStream_t st);
template <typename T>
int set_stress_smem(int slab_smem, int pencil_smem);
// <y, dS_J/dtheta x> of the junction step (pair 0 of P, table 2) summed over
// the grid: block partials into `part` (nblk), then `out` (one double)
template <typename T>
int launch_junction_dtheta(const StressArgs<T> &a, const StressPairs &P, int slab_threads, int slab_smem,
                           int pencil_threads, int pencil_smem, double *part, int nblk, double *out,
                           cudaStream_t st);

// ------------------------------------------------------------------ checkpointed densities
constexpr int kDensPairs = 32;

// slice pairs of one accumulation launch: element offsets (from the launch's
// base pointer) of q(s) and q^dagger(N-s) (or q^dagger(j), q^dagger(Nh-j)),
// and the raw Simpson weight of the product in the A block, the B block and
// the homopolymer sum
struct DensPairs {
    int n;
    long long x[kDensPairs], y[kDensPairs];
    double wA[kDensPairs], wB[kDensPairs], wH[kDensPairs];
};

template <typename T>
int launch_density_acc(const T *base, size_t M, const DensPairs &P, double *acc, int nblk, cudaStream_t st);
int launch_density_final(const double *acc, size_t M, double *rs_row, double ds, double chi, double *conc,
                         double *part, int nblk, cudaStream_t st);

// ------------------------------------------------------------------ FP64 field kernels
constexpr int kMaxStrn = 64;

struct FieldArgs {
    int M;
    int strn;
    const int *rep_list;   // replicas processed by the launch (blockIdx.y)
    double *W;             // [rep][2M]
    const double *conc;    // [rep][4M]
    double *DEV;           // [rep][2M]
    double *dWda;          // [rep][M]
    double *partials;      // [slotq][nblk]
    double chi;
};

// coefficients of the natural cubic spline that depend on the knots only
struct SplineKnots {
    int strn;
    double h[kMaxStrn], l[kMaxStrn], u[kMaxStrn];
    int nm_d[kMaxStrn];     // interval of knot ev (derivative evaluation)
    double dx_d[kMaxStrn];
    int nm_v[kMaxStrn];     // interval of xref[ev] (value evaluation)
    double dx_v[kMaxStrn];
    int doiis[kMaxStrn];
};

void launch_dev(const FieldArgs &a, int nrep_launch, int nblk, int dospring, double eps,
                cudaStream_t st);
void launch_mix0(const FieldArgs &a, int nrep_launch, const double *lam, cudaStream_t st);
void launch_mix(const FieldArgs &a, double lambda, cudaStream_t st);
void launch_edist(const FieldArgs &a, int nblk, cudaStream_t st);
void launch_spline_deriv(const FieldArgs &a, const SplineKnots *knots, int nblk, cudaStream_t st);
void launch_dots(const FieldArgs &a, int nrep_launch, int nblk, cudaStream_t st);
void launch_perp(const FieldArgs &a, int nrep_launch, const double *coef, const double *ndev,
                 int nblk, cudaStream_t st);
void launch_redist(const FieldArgs &a, const SplineKnots *knots, double lambda, int nblk,
                   cudaStream_t st);
void launch_freee(const FieldArgs &a, int nrep_launch, double f, int nblk, cudaStream_t st);
void launch_reduce_final(const double *partials, int nrows, int nblk, double *out,
                         cudaStream_t st);
void launch_hist_dots(const double *Dh, size_t n2M, int k, const int *slots, int n, int nblk, double *partials,
                      cudaStream_t st);
void launch_anderson_update(double *W, const double *Xh, const double *Dh, size_t n2M, int k, int m,
                            const int *slots, const double *theta, double lam, cudaStream_t st);

}  // namespace scft
