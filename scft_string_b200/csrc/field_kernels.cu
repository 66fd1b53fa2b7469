// field_kernels.cu -- FP64 field updates and string coupling of solve_field on
// sm_100a: residuals (scft.cu:527-535, 604-608, 624-639), simple mixing
// (scft.cu:543, 691-693), arc length (EDist, scft.cu:351-355), the natural
// cubic spline across replicas with its derivative and equal-arc value
// (cubefit_chunk_g / eval_spline_*_chunk_g, GPU_kernels.h:232-329), the
// perpendicular projection (scft.cu:648-683) and the free-energy sums
// (scft.cu:823-828).  Every sum is a per-block partial in fixed order
// followed by k_reduce_final, so results are deterministic.
#include "kernels.h"

namespace scft {

namespace {

struct SmallVec {
    double v[kMaxStrn];
};

__device__ __forceinline__ double block_sum(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
    return t;
}

__device__ __forceinline__ void put_partial(double *partials, int row, double v, double *sh)
{
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) partials[(size_t)row * gridDim.x + blockIdx.x] = t;
}

// DEV- = chi (phiB - phiA) - 2 W- (+ spring), DEV+ = chi (phiB + phiA - 1)
// (scft.cu:604-608).  Partial rows: 2j -> sum_2M DEV^2, 2j+1 -> sum_M DEV-^2.
__global__ void k_dev(FieldArgs a, int dospring, double eps)
{
    __shared__ double sh[32];
    const int j = blockIdx.y, ii = a.rep_list[j];
    const size_t M = a.M;
    const double *W = a.W + ii * 2 * M;
    const double *phiA = a.conc + ii * 4 * M, *phiB = phiA + M;
    double *DEV = a.DEV + ii * 2 * M;
    const bool spring = dospring && ii > 0 && ii < a.strn - 1;
    const double *Wn = spring ? a.W + (ii + 1) * 2 * M : W, *Wp = spring ? a.W + (ii - 1) * 2 * M : W;
    double s2 = 0, sm = 0;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        double dm = a.chi * (phiB[r] - phiA[r]) - 2.0 * W[r];
        if (spring) dm += eps * (Wn[r] + Wp[r] - 2.0 * W[r]);
        const double dp = a.chi * (phiB[r] + phiA[r] - 1.0);
        DEV[r] = dm;
        DEV[r + M] = dp;
        s2 += dm * dm + dp * dp;
        sm += dm * dm;
    }
    put_partial(a.partials, 2 * j, s2, sh);
    put_partial(a.partials, 2 * j + 1, sm, sh);
}

// solve_field0 mixing: W += lambda * (0, chi (phiB + phiA - 1)) (scft.cu:528-529, 543)
__global__ void k_mix0(FieldArgs a, SmallVec lam)
{
    const int j = blockIdx.y, ii = a.rep_list[j];
    const size_t M = a.M;
    double *W = a.W + ii * 2 * M;
    const double *phiA = a.conc + ii * 4 * M, *phiB = phiA + M;
    const double l = lam.v[j];
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        W[r + M] = W[r + M] + l * (a.chi * (phiB[r] + phiA[r] - 1.0));
    }
}

// W[ii] += lambda DEV[ii] for every replica (scft.cu:691-693)
__global__ void k_mix(FieldArgs a, double lambda)
{
    const int ii = blockIdx.y;
    const size_t n = 2 * (size_t)a.M;
    double *W = a.W + ii * n;
    const double *D = a.DEV + ii * n;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x)
        W[r] = W[r] + lambda * D[r];
}

// partial sums of (W-[i] - W-[i+1])^2 (EDist, scft.cu:351-355); row i
__global__ void k_edist(FieldArgs a)
{
    __shared__ double sh[32];
    const int i = blockIdx.y;
    const size_t M = a.M;
    const double *w0 = a.W + i * 2 * M, *w1 = a.W + (i + 1) * 2 * M;
    double s = 0;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        const double d = w0[r] - w1[r];
        s += d * d;
    }
    put_partial(a.partials, i, s, sh);
}

// natural cubic spline of a[0..strn) over the knots (cubefit_chunk_g,
// GPU_kernels.h:232-284); on return zc holds the c coefficients
__device__ __forceinline__ void spline_fit(const SplineKnots &K, const double *a, double *zc)
{
    const int n = K.strn - 1;
    zc[0] = 0.0;
    for (int i = 1; i <= n - 1; ++i) {
        const double Ai = 3.0 * (a[i + 1] - a[i]) / K.h[i] - 3.0 * (a[i] - a[i - 1]) / K.h[i - 1];
        zc[i] = (Ai - K.h[i - 1] * zc[i - 1]) / K.l[i];
    }
    zc[n] = 0.0;  // z[n] = 0 and c[n] = 0
    for (int j = n - 1; j >= 0; --j) zc[j] = zc[j] - K.u[j] * zc[j + 1];
}

__device__ __forceinline__ void spline_bd(const SplineKnots &K, const double *a, const double *c,
                                          int j, double &b, double &d)
{
    if (j >= K.strn - 1) {
        b = 0.0;
        d = 0.0;
        return;
    }
    b = (a[j + 1] - a[j]) / K.h[j] - K.h[j] * (c[j + 1] + 2.0 * c[j]) / 3.0;
    d = (c[j + 1] - c[j]) / (3.0 * K.h[j]);
}

// dW-/dalpha at the knots for replicas with doiis == 1
// (eval_spline_deriv_chunk_g, GPU_kernels.h:286-306)
__global__ void k_spline_deriv(FieldArgs a, const SplineKnots *__restrict__ knots)
{
    __shared__ SplineKnots K;
    if (threadIdx.x == 0) K = *knots;
    __syncthreads();
    const size_t M = a.M;
    const int strn = K.strn;
    double av[kMaxStrn], zc[kMaxStrn];
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        for (int ii = 0; ii < strn; ii++) av[ii] = a.W[ii * 2 * M + r];
        spline_fit(K, av, zc);
        for (int ev = 0; ev < strn; ev++) {
            if (K.doiis[ev] != 1) continue;
            const int nm = K.nm_d[ev];
            const double dx = K.dx_d[ev];
            double b, d;
            spline_bd(K, av, zc, nm, b, d);
            a.dWda[ev * M + r] = b + 2.0 * dx * zc[nm] + 3.0 * dx * dx * d;
        }
    }
}

// per-replica sums for the projection: row 2j -> sum dWda^2, 2j+1 -> sum DEV- dWda
__global__ void k_dots(FieldArgs a)
{
    __shared__ double sh[32];
    const int j = blockIdx.y, ii = a.rep_list[j];
    const size_t M = a.M;
    const double *D = a.DEV + ii * 2 * M, *dw = a.dWda + ii * M;
    double s0 = 0, s1 = 0;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        s0 += dw[r] * dw[r];
        s1 += D[r] * dw[r];
    }
    put_partial(a.partials, 2 * j, s0, sh);
    put_partial(a.partials, 2 * j + 1, s1, sh);
}

// DEV- -= (dotW/normDER) dWda normDEV (scft.cu:672), then sum_2M DEV^2 (scft.cu:673)
__global__ void k_perp(FieldArgs a, SmallVec coef, SmallVec ndev)
{
    __shared__ double sh[32];
    const int j = blockIdx.y, ii = a.rep_list[j];
    const size_t M = a.M;
    double *D = a.DEV + ii * 2 * M;
    const double *dw = a.dWda + ii * M;
    const double cf = coef.v[j], nd = ndev.v[j];
    double s = 0;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        const double v = D[r] - cf * dw[r] * nd;
        D[r] = v;
        const double p = D[r + M];
        s += v * v + p * p;
    }
    put_partial(a.partials, j, s, sh);
}

// W-[ii] += lambda (S(xref[ii]) - W-[ii]) for interior replicas with doiis == 1
// (eval_spline_value_chunk_g, GPU_kernels.h:308-329; density.h:524-527)
__global__ void k_redist(FieldArgs a, const SplineKnots *__restrict__ knots, double lambda)
{
    __shared__ SplineKnots K;
    if (threadIdx.x == 0) K = *knots;
    __syncthreads();
    const size_t M = a.M;
    const int strn = K.strn;
    double av[kMaxStrn], zc[kMaxStrn];
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        for (int ii = 0; ii < strn; ii++) av[ii] = a.W[ii * 2 * M + r];
        spline_fit(K, av, zc);
        for (int ii = 1; ii < strn - 1; ii++) {
            if (K.doiis[ii] != 1) continue;
            const int nm = K.nm_v[ii];
            const double dx = K.dx_v[ii];
            double b, d;
            spline_bd(K, av, zc, nm, b, d);
            const double val = av[nm] + dx * b + dx * dx * zc[nm] + dx * dx * dx * d;
            a.W[ii * 2 * M + r] = av[ii] + (val - av[ii]) * lambda;
        }
    }
}

// free-energy sums (scft.cu:823-828): row 2j -> sum (chi phiA phiB - wa phiA - wb phiB)/M,
// row 2j+1 -> sum phiA/(M f)
__global__ void k_freee(FieldArgs a, double f)
{
    __shared__ double sh[32];
    const int j = blockIdx.y, ii = a.rep_list[j];
    const size_t M = a.M;
    const double *W = a.W + ii * 2 * M;
    const double *phiA = a.conc + ii * 4 * M, *phiB = phiA + M;
    double s0 = 0, s1 = 0;
    const double Md = (double)M;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        const double wa = W[r] + W[r + M], wb = W[r + M] - W[r];
        s0 += (a.chi * phiA[r] * phiB[r] - wa * phiA[r] - wb * phiB[r]) / Md;
        s1 += phiA[r] / (Md * f);
    }
    put_partial(a.partials, 2 * j, s0, sh);
    put_partial(a.partials, 2 * j + 1, s1, sh);
}

__global__ void k_reduce_final(const double *partials, int nrows, int nblk, double *out)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    double t = 0;
    for (int i = 0; i < nblk; i++) t += partials[(size_t)row * nblk + i];
    out[row] = t;
}

SmallVec to_vec(const double *v, int n)
{
    SmallVec s;
    for (int i = 0; i < kMaxStrn; i++) s.v[i] = i < n ? v[i] : 0.0;
    return s;
}

}  // namespace

constexpr int kThreads = 256;

void launch_dev(const FieldArgs &a, int n, int nblk, int dospring, double eps, cudaStream_t st)
{
    k_dev<<<dim3(nblk, n), kThreads, 0, st>>>(a, dospring, eps);
}

void launch_mix0(const FieldArgs &a, int n, const double *lam, cudaStream_t st)
{
    k_mix0<<<dim3(256, n), kThreads, 0, st>>>(a, to_vec(lam, n));
}

void launch_mix(const FieldArgs &a, double lambda, cudaStream_t st)
{
    k_mix<<<dim3(256, a.strn), kThreads, 0, st>>>(a, lambda);
}

void launch_edist(const FieldArgs &a, int nblk, cudaStream_t st)
{
    if (a.strn > 1) k_edist<<<dim3(nblk, a.strn - 1), kThreads, 0, st>>>(a);
}

void launch_spline_deriv(const FieldArgs &a, const SplineKnots *knots, int nblk, cudaStream_t st)
{
    k_spline_deriv<<<nblk, 128, 0, st>>>(a, knots);
}

void launch_dots(const FieldArgs &a, int n, int nblk, cudaStream_t st)
{
    k_dots<<<dim3(nblk, n), kThreads, 0, st>>>(a);
}

void launch_perp(const FieldArgs &a, int n, const double *coef, const double *ndev, int nblk,
                 cudaStream_t st)
{
    k_perp<<<dim3(nblk, n), kThreads, 0, st>>>(a, to_vec(coef, n), to_vec(ndev, n));
}

void launch_redist(const FieldArgs &a, const SplineKnots *knots, double lambda, int nblk,
                   cudaStream_t st)
{
    k_redist<<<nblk, 128, 0, st>>>(a, knots, lambda);
}

void launch_freee(const FieldArgs &a, int n, double f, int nblk, cudaStream_t st)
{
    k_freee<<<dim3(nblk, n), kThreads, 0, st>>>(a, f);
}

void launch_reduce_final(const double *partials, int nrows, int nblk, double *out, cudaStream_t st)
{
    k_reduce_final<<<(nrows + 127) / 128, 128, 0, st>>>(partials, nrows, nblk, out);
}

}  // namespace scft

// ------------------------------------------------------------------ Anderson mixing
// (no reference code; the reference keeps only scaffolding for it, scft.cu:30-31)
namespace scft {
namespace {

// partial sums of <d_k, d_j> for the n history slots listed in `slots`
__global__ void k_hist_dots(const double *Dh, size_t n2M, int k, SmallVec slots, double *partials)
{
    __shared__ double sh[32];
    const int j = blockIdx.y;
    const double *a = Dh + (size_t)k * n2M, *b = Dh + (size_t)(int)slots.v[j] * n2M;
    double s = 0;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n2M; r += (size_t)gridDim.x * blockDim.x)
        s += a[r] * b[r];
    put_partial(partials, j, s, sh);
}

// W = (x_k + lam d_k) - sum_i theta_i ((x_k + lam d_k) - (x_i + lam d_i))
__global__ void k_anderson_update(double *W, const double *Xh, const double *Dh, size_t n2M, int k, int m,
                                  SmallVec slots, SmallVec theta, double lam)
{
    const double *xk = Xh + (size_t)k * n2M, *dk = Dh + (size_t)k * n2M;
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n2M; r += (size_t)gridDim.x * blockDim.x) {
        const double yk = xk[r] + lam * dk[r];
        double v = yk;
        for (int i = 0; i < m; i++) {
            const size_t o = (size_t)(int)slots.v[i] * n2M + r;
            v -= theta.v[i] * (yk - (Xh[o] + lam * Dh[o]));
        }
        W[r] = v;
    }
}

}  // namespace

void launch_hist_dots(const double *Dh, size_t n2M, int k, const int *slots, int n, int nblk, double *partials,
                      cudaStream_t st)
{
    SmallVec sv;
    for (int i = 0; i < kMaxStrn; i++) sv.v[i] = i < n ? slots[i] : 0;
    k_hist_dots<<<dim3(nblk, n), kThreads, 0, st>>>(Dh, n2M, k, sv, partials);
}

void launch_anderson_update(double *W, const double *Xh, const double *Dh, size_t n2M, int k, int m,
                            const int *slots, const double *theta, double lam, cudaStream_t st)
{
    SmallVec sv, th;
    for (int i = 0; i < kMaxStrn; i++) {
        sv.v[i] = i < m ? slots[i] : 0;
        th.v[i] = i < m ? theta[i] : 0;
    }
    k_anderson_update<<<512, kThreads, 0, st>>>(W, Xh, Dh, n2M, k, m, sv, th, lam);
}

}  // namespace scft
