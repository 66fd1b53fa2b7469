// common.cuh -- shared types of the sm_100a SCFT kernels.
//
// Layouts (same as the reference, scft.cu:462-464 and density.h:90):
//   real grid      r = z + m2*(y + m1*x)
//   half spectrum  k = kz + mk2*(ky + m1*kx),  mk2 = m2/2 + 1
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

namespace scft {

template <typename T>
struct cplx {
    T x, y;
};

template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename T>
__device__ __forceinline__ cplx<T> cmulc(cplx<T> a, cplx<T> b)
{
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b)
{
    return {a.x + b.x, a.y + b.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b)
{
    return {a.x - b.x, a.y - b.y};
}

constexpr int kMaxStages = 12;
constexpr int kPairLanes = 8;  // slab pack/unpack: mk2 <= 32*kPairLanes

// Mixed-radix factorisation of one FFT length (radices 2, 3, 4, 5, 7, 8).
struct Plan1D {
    int n;
    int nst;
    int radix[kMaxStages];
};

// Everything a propagator kernel needs to know about the grid.
struct Geo {
    int m0, m1, m2, mk2;
    int M, Mk;
    int npair;       // ceil(m1/2): packed real y-line pairs per x-slab
    int slab_c;      // complex elements of one slab buffer (m1*mk2 + slack)
    Plan1D px, py, pz;
    int Ns, n1, n2, Nh;
    int ncol_tiles;  // x-pencil tiles per field
    int tc;          // columns per x-pencil tile
    // continuous A fraction (off when jon == 0): q's step jq and q^dagger's
    // step jqd see the junction field theta wA + (1 - theta) wB (E table 2)
    int jon, jq, jqd;
    double theta;
};

// Raises a kernel's dynamic shared-memory limit to at least `bytes`, never
// lowers it.  The limit belongs to the kernel, not to a context: the
// runtime-shaped kernels serve every context of any grid, so a context that
// set it to its own (smaller) need would make the launches of an earlier,
// larger context fail.  Serialised, so concurrent context creation keeps
// the largest value.
template <typename F>
inline cudaError_t raise_dyn_smem(F *fn, int bytes)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes at;
    cudaError_t e = cudaFuncGetAttributes(&at, reinterpret_cast<const void *>(fn));
    if (e != cudaSuccess) return e;
    if (at.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(reinterpret_cast<const void *>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bytes);
}

}  // namespace scft
