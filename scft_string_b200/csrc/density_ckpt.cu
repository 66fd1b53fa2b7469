// density_ckpt.cu -- the Simpson density pass of density::props
// (density.h:402-454) from propagator slices held only in recomputed segments
// (scft_props_ckpt): the terms w_s q(s) q^dagger(N-s) arrive in batches of
// slice pairs and are Kahan-accumulated per grid point in FP64; a final
// kernel scales them into phiA, phiB, phih, phicB and the phis averages.
#include "kernels.h"

namespace scft {

namespace {

__device__ __forceinline__ void kahan(double &sum, double &c, double term)
{
    const double y = term - c;
    const double t = sum + y;
    c = (t - sum) - y;
    sum = t;
}

__device__ __forceinline__ double bsum(double v, double *sh)
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

// acc per point: [sA, cA, sB, cB, sH, cH] x M (sums and Kahan compensations of
// the copolymer A block, the copolymer B block and the homopolymer)
template <typename T>
__global__ void k_dens_acc(const T *__restrict__ base, size_t M, DensPairs P, double *__restrict__ acc)
{
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        double s[6];
#pragma unroll
        for (int k = 0; k < 6; k++) s[k] = acc[k * M + r];
        for (int p = 0; p < P.n; p++) {
            const double t = (double)base[P.x[p] + r] * (double)base[P.y[p] + r];
            if (P.wA[p] != 0.0) kahan(s[0], s[1], P.wA[p] * t);
            if (P.wB[p] != 0.0) kahan(s[2], s[3], P.wB[p] * t);
            if (P.wH[p] != 0.0) kahan(s[4], s[5], P.wH[p] * t);
        }
#pragma unroll
        for (int k = 0; k < 6; k++) acc[k * M + r] = s[k];
    }
}

// densities (the scaling of density.h:430-431 and GPU_kernels.h:129-139) and
// per-block partial sums of rC, rA, rB, rhA, rhB and (chi (phiA+phiB-1))^2
__global__ void k_dens_final(const double *__restrict__ acc, size_t M, const double *__restrict__ rs, double ds,
                             double chi, double *__restrict__ conc, double *__restrict__ part)
{
    __shared__ double sh[32];
    const double zB = rs[kRsZB], zC = rs[kRsZC];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        const double rCA = acc[r] * zC * ds / 3.0;
        const double rCB = acc[2 * M + r] * zC * ds / 3.0;
        const double rhB = acc[4 * M + r] * zB * ds / 3.0;
        const double rhA = 0.0;  // scaled by zA = 0
        const double rA = rhA + rCA, rB = rhB + rCB;
        conc[r] = rA;
        conc[r + M] = rB;
        conc[r + 2 * M] = rhA + rhB;
        conc[r + 3 * M] = rCB;
        const double dv = chi * (rB + rA - 1.0);
        a[0] += rCA + rCB;
        a[1] += rA;
        a[2] += rB;
        a[3] += rhA;
        a[4] += rhB;
        a[5] += dv * dv;
    }
    for (int k = 0; k < 6; k++) {
        const double t = bsum(a[k], sh);
        if (threadIdx.x == 0) part[k * gridDim.x + blockIdx.x] = t;
    }
}

// phis and the W+ residual sum into the replica's scalar record
__global__ void k_dens_phis(const double *__restrict__ part, int nblk, size_t M, double *__restrict__ rs)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v[6];
    for (int k = 0; k < 6; k++) {
        double t = 0;
        for (int i = 0; i < nblk; i++) t += part[k * nblk + i];
        v[k] = t;
    }
    for (int k = 0; k < 5; k++) rs[kRsPhis + k] = v[k] / (double)M;
    rs[kRsDev2] = v[5];
}

}  // namespace

template <typename T>
int launch_density_acc(const T *base, size_t M, const DensPairs &P, double *acc, int nblk, cudaStream_t st)
{
    k_dens_acc<T><<<nblk, 256, 0, st>>>(base, M, P, acc);
    return 1;
}

int launch_density_final(const double *acc, size_t M, double *rs_row, double ds, double chi, double *conc,
                         double *part, int nblk, cudaStream_t st)
{
    k_dens_final<<<nblk, 256, 0, st>>>(acc, M, rs_row, ds, chi, conc, part);
    k_dens_phis<<<1, 32, 0, st>>>(part, nblk, M, rs_row);
    return 2;
}

template int launch_density_acc<float>(const float *, size_t, const DensPairs &, double *, int, cudaStream_t);
template int launch_density_acc<double>(const double *, size_t, const DensPairs &, double *, int, cudaStream_t);

}  // namespace scft
