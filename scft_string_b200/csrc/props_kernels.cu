// props_kernels.cu -- the contour-step pipeline of density::props on sm_100a.
//
// One Richardson step (density.h:129-220, GPU_kernels.h:175-203) advances q and
// q^dagger of every replica slot in the batch:
//   qs0 = IFFT(K2 FFT(E2 * IFFT(K2 FFT(E4 q))))      (two half steps)
//   qs1 = IFFT(K1 FFT(E2 q))                        (one full step)
//   q'  = (4 E4 qs0 - E2 qs1) / 3
// with E4 = exp(-w ds/4), E2 = E4^2, K2 = exp(-k^2 ds/12)/M, K1 = K2^2 M.
// Four launches per step, each over (slot, field, slab-or-tile):
//   pencil(both)  x-transform of the two spectra, times K2 / K1, back
//   mid           inverse slab of qs1 -> P = E2 qs1 (real, kept for the
//                 combine); inverse slab of the half step, times E2, forward
//   pencil(A)     x-transform, times K2, back
//   combine       inverse slab -> q' = (4 E4 qs0 - P)/3 -> propagator store;
//                 forward slabs of E4' q' and E2' q' for the next step
// The q(s) store (density.h:293-301 keeps every slice) feeds the Simpson
// density pass (density.h:402-430), done by k_density in FP64.
#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"
#include "tma.cuh"
#include "step_order.cuh"

namespace scft {

template <typename T>
__device__ __forceinline__ size_t hist_off(const Geo &g, int slot, int s, int fld)
{
    return (((size_t)slot * (g.Ns + 1) + s) * 2 + fld) * (size_t)g.M;
}

// E4 table (0: A field, 1: B field, 2: junction) for field fld (0: q,
// 1: q^dagger) at step s; q sees the A block for s < n1, q^dagger the B block
// for s < n2 (density.h:136-146).  With a continuous A fraction the step that
// holds the junction (q's jq, q^dagger's jqd) takes table 2.
__device__ __forceinline__ int etab_sel(const Geo &g, int fld, int s)
{
    if (g.jon && s == (fld == 0 ? g.jq : g.jqd)) return 2;
    return fld == 0 ? (s < g.n1 ? 0 : 1) : (s < g.n2 ? 1 : 0);
}

// the E4 table `sel` of slot `slot`
template <typename T>
__device__ __forceinline__ const T *etab_ptr(const PropsArgs<T> &a, int slot, int sel)
{
    return sel == 2 ? a.jtab + (size_t)slot * a.g.M : a.etab + ((size_t)slot * 2 + sel) * a.g.M;
}

template <typename T>
__device__ __forceinline__ void load_tw(cplx<T> *dst, const cplx<T> *src, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------- prepare
// E4 = exp(-wA ds/4), exp(-wB ds/4) with wA = W- + W+, wB = W+ - W-
// (Prepare_dev_dev_expWds2_dev_expWds, GPU_kernels.h:215-225)
template <typename T>
__global__ void k_prepare(PropsArgs<T> a)
{
    const Geo g = a.g;
    const int slot = blockIdx.y;
    const int rep = a.slot_rep[slot];
    const double *W = a.W + (size_t)rep * 2 * g.M;
    T *e = a.etab + (size_t)slot * 2 * g.M;
    const double ds = 1.0 / g.Ns;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < g.M; r += gridDim.x * blockDim.x) {
        const double wm = W[r], wp = W[r + g.M];
        e[r] = (T)exp(-(wm + wp) * ds / 4);
        e[r + g.M] = (T)exp(-(-wm + wp) * ds / 4);
        // junction step: theta wA + (1 - theta) wB = W+ + (2 theta - 1) W-
        if (g.jon) a.jtab[(size_t)slot * g.M + r] = (T)exp(-(wp + (2.0 * g.theta - 1.0) * wm) * ds / 4);
    }
}

// ---------------------------------------------------------------- shape dispatch
// Offset of packed z-row p (real lines 2p, 2p+1) in a slab buffer: stride
// M2 + 1 for the compile-time shapes, 2 mk2 for the runtime path.
template <int FM2>
__device__ __forceinline__ int prow(int p, int mk2)
{
    if constexpr (FM2 != 0)
        return p * PackedRows<FM2>::LSF;
    else
        return 2 * p * mk2;
}

// FM0/FM1/FM2 = 0: sizes from the runtime Geo; otherwise compile-time sizes
// (blockDim.x == MT, tile width from kTile<T>).
template <typename T>
struct kTile {
    static constexpr int value = sizeof(T) == 4 ? 32 : 16;
};

template <typename T, int MT, int FM1, int FM2>
__device__ __forceinline__ void slab_fwd(cplx<T> *buf, const Geo &g, const cplx<T> *twy,
                                         const cplx<T> *twz, int *err)
{
    if constexpr (FM1 != 0)
        slab_forward_fixed<T, FM1, FM2, MT>(buf, twy, twz);
    else
        slab_forward(buf, g, twy, twz, err);
}

template <typename T, int MT, int FM1, int FM2>
__device__ __forceinline__ void slab_inv(cplx<T> *buf, const Geo &g, const cplx<T> *twy,
                                         const cplx<T> *twz, int *err)
{
    if constexpr (FM1 != 0)
        slab_inverse_fixed<T, FM1, FM2, MT>(buf, twy, twz);
    else
        slab_inverse(buf, g, twy, twz, err);
}

// ---------------------------------------------------------------- combine
// mode 0: finishes step s (q(s+1) = Richardson combination);
// mode 1: q(s+1) = 1 (Array_set_value, density.h:368-369; called with s = -1);
// mode 2: q(s+1) is taken from the propagator store (single-step entry).
// Then starts step s+1 when s+1 < Ns.
template <typename T, int MT, int FM0, int FM1, int FM2>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 3 : 2) : 1) k_combine(PropsArgs<T> a, int s, int mode)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    constexpr bool FX = FM1 != 0;
    const int m1 = FX ? FM1 : g.m1, m2 = FX ? FM2 : g.m2, mk2 = m2 / 2 + 1;
    const int m0 = FX ? FM0 : g.m0, M = m0 * m1 * m2, Mk = m0 * m1 * mk2;
    const int slab_c = m1 * mk2 + m2 + 32;
    const int nthr = FX ? MT : (int)blockDim.x;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twy = buf + slab_c;
    cplx<T> *twz = twy + m1;
    for (int i = threadIdx.x; i < m1; i += nthr) twy[i] = a.tw[m0 + i];
    for (int i = threadIdx.x; i < m2; i += nthr) twz[i] = a.tw[m0 + m1 + i];
    const int x = blockIdx.x, fld = blockIdx.y, slot = blockIdx.z;
    const size_t slab_r = (size_t)x * m1 * m2;  // real offset of this slab
    const size_t slab_k = (size_t)x * m1 * mk2;
    cplx<T> *specA = a.spec + ((size_t)slot * 2 + fld) * 2 * Mk;
    cplx<T> *specB = specA + Mk;
    const int sn = s + 1;
    T *qn = a.hist + hist_off<T>(g, slot, sn, fld) + slab_r;
    const int npair = (m1 + 1) / 2, npz = npair * m2;

    if (mode == 0) {
        for (int i = threadIdx.x; i < m1 * mk2; i += nthr) buf[i] = specA[slab_k + i];
        __syncthreads();
        slab_inv<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
        const T *E4 = etab_ptr(a, slot, etab_sel(g, fld, s)) + slab_r;
        const T *P = a.pbuf + ((size_t)slot * 2 + fld) * M + slab_r;
        for (int e = threadIdx.x; e < npz; e += nthr) {
            const int p = e / m2, z = e - p * m2;
            cplx<T> &c = buf[prow<FM2>(p, mk2) + z];
            const int r0 = 2 * p * m2 + z;
            // Richardson, GPU_kernels.h:199-203
            c.x = (c.x * E4[r0] * (T)4 - P[r0]) / (T)3;
            qn[r0] = c.x;
            if (2 * p + 1 < m1) {
                const int r1 = r0 + m2;
                c.y = (c.y * E4[r1] * (T)4 - P[r1]) / (T)3;
                qn[r1] = c.y;
            } else {
                c.y = (T)0;
            }
        }
    } else if (mode == 1) {
        for (int e = threadIdx.x; e < npz; e += nthr) {
            const int p = e / m2, z = e - p * m2;
            const int r0 = 2 * p * m2 + z;
            const bool hb = 2 * p + 1 < m1;
            buf[prow<FM2>(p, mk2) + z] = {(T)1, hb ? (T)1 : (T)0};
            qn[r0] = (T)1;
            if (hb) qn[r0 + m2] = (T)1;
        }
    } else {
        for (int e = threadIdx.x; e < npz; e += nthr) {
            const int p = e / m2, z = e - p * m2;
            const int r0 = 2 * p * m2 + z;
            const bool hb = 2 * p + 1 < m1;
            buf[prow<FM2>(p, mk2) + z] = {qn[r0], hb ? qn[r0 + m2] : (T)0};
        }
    }
    if (sn >= g.Ns) return;
    __syncthreads();
    const T *E4n = etab_ptr(a, slot, etab_sel(g, fld, sn)) + slab_r;
    // half step input E4' q'
    for (int e = threadIdx.x; e < npz; e += nthr) {
        const int p = e / m2, z = e - p * m2;
        cplx<T> &c = buf[prow<FM2>(p, mk2) + z];
        const int r0 = 2 * p * m2 + z;
        c.x *= E4n[r0];
        if (2 * p + 1 < m1) c.y *= E4n[r0 + m2];
    }
    __syncthreads();
    slab_fwd<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
    for (int i = threadIdx.x; i < m1 * mk2; i += nthr) specA[slab_k + i] = buf[i];
    __syncthreads();
    // full step input E2' q' (q' re-read from the propagator store written above)
    for (int e = threadIdx.x; e < npz; e += nthr) {
        const int p = e / m2, z = e - p * m2;
        const int r0 = 2 * p * m2 + z;
        const T e0 = E4n[r0];
        T v0 = qn[r0] * (e0 * e0), v1 = (T)0;
        if (2 * p + 1 < m1) {
            const T e1 = E4n[r0 + m2];
            v1 = qn[r0 + m2] * (e1 * e1);
        }
        buf[prow<FM2>(p, mk2) + z] = {v0, v1};
    }
    __syncthreads();
    slab_fwd<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
    for (int i = threadIdx.x; i < m1 * mk2; i += nthr) specB[slab_k + i] = buf[i];
}

// ---------------------------------------------------------------- mid
template <typename T, int MT, int FM0, int FM1, int FM2>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 3 : 2) : 1) k_mid(PropsArgs<T> a, int s)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    constexpr bool FX = FM1 != 0;
    const int m1 = FX ? FM1 : g.m1, m2 = FX ? FM2 : g.m2, mk2 = m2 / 2 + 1;
    const int m0 = FX ? FM0 : g.m0, M = m0 * m1 * m2, Mk = m0 * m1 * mk2;
    const int slab_c = m1 * mk2 + m2 + 32;
    const int nthr = FX ? MT : (int)blockDim.x;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twy = buf + slab_c;
    cplx<T> *twz = twy + m1;
    for (int i = threadIdx.x; i < m1; i += nthr) twy[i] = a.tw[m0 + i];
    for (int i = threadIdx.x; i < m2; i += nthr) twz[i] = a.tw[m0 + m1 + i];
    const int x = blockIdx.x, fld = blockIdx.y, slot = blockIdx.z;
    const size_t slab_r = (size_t)x * m1 * m2;
    const size_t slab_k = (size_t)x * m1 * mk2;
    const T *E4 = etab_ptr(a, slot, etab_sel(g, fld, s)) + slab_r;
    cplx<T> *specA = a.spec + ((size_t)slot * 2 + fld) * 2 * Mk;
    cplx<T> *specB = specA + Mk;
    T *P = a.pbuf + ((size_t)slot * 2 + fld) * M + slab_r;
    const int npz = ((m1 + 1) / 2) * m2;

    // full step: P = E2 * qs1
    for (int i = threadIdx.x; i < m1 * mk2; i += nthr) buf[i] = specB[slab_k + i];
    __syncthreads();
    slab_inv<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
    for (int e = threadIdx.x; e < npz; e += nthr) {
        const int p = e / m2, z = e - p * m2;
        const cplx<T> c = buf[prow<FM2>(p, mk2) + z];
        const int r0 = 2 * p * m2 + z;
        const T e0 = E4[r0];
        P[r0] = c.x * (e0 * e0);
        if (2 * p + 1 < m1) {
            const T e1 = E4[r0 + m2];
            P[r0 + m2] = c.y * (e1 * e1);
        }
    }
    __syncthreads();
    // second half step input: E2 * (first half step)
    for (int i = threadIdx.x; i < m1 * mk2; i += nthr) buf[i] = specA[slab_k + i];
    __syncthreads();
    slab_inv<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
    for (int e = threadIdx.x; e < npz; e += nthr) {
        const int p = e / m2, z = e - p * m2;
        cplx<T> &c = buf[prow<FM2>(p, mk2) + z];
        const int r0 = 2 * p * m2 + z;
        const T e0 = E4[r0];
        c.x *= e0 * e0;
        if (2 * p + 1 < m1) {
            const T e1 = E4[r0 + m2];
            c.y *= e1 * e1;
        } else {
            c.y = (T)0;
        }
    }
    __syncthreads();
    slab_fwd<T, MT, FM1, FM2>(buf, g, twy, twz, a.err);
    for (int i = threadIdx.x; i < m1 * mk2; i += nthr) specA[slab_k + i] = buf[i];
}

// ---------------------------------------------------------------- pencil
// x-transform of a tile of tc consecutive (ky, kz) columns, times the
// diffusion factor (Mult_self, GPU_kernels.h:175-181), inverse x-transform.
// both != 0: spectrum A with K2 and spectrum B with K1; else A with K2 only.
template <typename T, int MT, int FM0, int FM1, int FM2>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 3 : 2) : 1) k_pencil(PropsArgs<T> a, int both)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    constexpr bool FX = FM0 != 0;
    constexpr int TCF = kTile<T>::value;
    const int tc = FX ? TCF : g.tc, m0 = FX ? FM0 : g.m0;
    const int m1 = FX ? FM1 : g.m1, mk2 = (FX ? FM2 : g.m2) / 2 + 1;
    const int Mk = m0 * m1 * mk2;
    const int nthr = FX ? MT : (int)blockDim.x;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twx = buf + tc * m0;
    T *colf = reinterpret_cast<T *>(twx + m0);
    T *gx = colf + tc;
    for (int i = threadIdx.x; i < m0; i += nthr) twx[i] = a.tw[i];
    const int tile = blockIdx.x, fld = blockIdx.y, slot = blockIdx.z;
    const int ncol = m1 * mk2;
    const int c0 = tile * tc;
    const T *kf = a.kfac + (size_t)a.slot_rep[slot] * a.kf_stride;  // the replica's box
    for (int t = threadIdx.x; t < tc; t += nthr) {
        const int c = c0 + t;
        const int y = c / mk2, kz = c - y * mk2;
        colf[t] = c < ncol ? kf[m0 + y] * kf[m0 + m1 + kz] : (T)0;
    }
    for (int i = threadIdx.x; i < m0; i += nthr) gx[i] = kf[i];
    const T invM = a.invM;
    cplx<T> *spec = a.spec + ((size_t)slot * 2 + fld) * 2 * Mk;
    const int npass = both ? 2 : 1;
    for (int pass = 0; pass < npass; pass++) {
        cplx<T> *sp = spec + (size_t)pass * Mk;
        __syncthreads();
        for (int e = threadIdx.x; e < tc * m0; e += nthr) {
            const int x = e / tc, t = e - x * tc;
            const int c = c0 + t;
            buf[e] = c < ncol ? sp[(size_t)x * ncol + c] : cplx<T>{(T)0, (T)0};
        }
        __syncthreads();
        if constexpr (FX)
            fft_fixed<T, FM0, TCF, TCF, 1, true, MT>(buf, twx, -1);
        else
            cta_fft(buf, g.px, tc, tc, 1, true, twx, -1, a.err);
        for (int e = threadIdx.x; e < tc * m0; e += nthr) {
            const int x = e / tc, t = e - x * tc;
            const T k2 = gx[x] * colf[t];
            // pass 0: K2 = g/M ; pass 1: K1 = g^2/M  (Prepare_dev_expKsq2_expKsq, GPU_kernels.h:207-213)
            const T f = pass == 0 ? k2 * invM : (k2 * invM) * (k2 * invM) * a.Mreal;
            buf[e].x *= f;
            buf[e].y *= f;
        }
        __syncthreads();
        if constexpr (FX)
            fft_fixed<T, FM0, TCF, TCF, 1, true, MT>(buf, twx, +1);
        else
            cta_fft(buf, g.px, tc, tc, 1, true, twx, +1, a.err);
        for (int e = threadIdx.x; e < tc * m0; e += nthr) {
            const int x = e / tc, t = e - x * tc;
            const int c = c0 + t;
            if (c < ncol) sp[(size_t)x * ncol + c] = buf[e];
        }
    }
}

// ---------------------------------------------------------------- prefetching slab kernels
// Compile-time shapes whose operands fit in shared memory.  One thread issues
// bulk asynchronous copies (TMA, cp.async.bulk) of every slab the kernel needs
// as soon as it starts; the transforms run while the later copies land, and
// the epilogues read their operands from shared memory.
// Shared-memory layout: [4 mbarriers | spectrum A | (spectrum B) | twiddles y, z |
// real slabs].
template <typename T, int M1, int M2>
struct SlabSmem {
    static constexpr int MK2 = M2 / 2 + 1;
    static constexpr int SLAB_C = M1 * MK2 + M2 + 32;              // complex elements per spectrum buffer
    static constexpr int SPEC_BYTES = M1 * MK2 * 2 * (int)sizeof(T); // bytes copied per spectrum slab
    static constexpr int REAL = M1 * M2;                           // reals per real slab
    static constexpr int REAL_BYTES = REAL * (int)sizeof(T);
    static constexpr int BARS = 128;
    static constexpr int mid_bytes() { return BARS + (2 * SLAB_C + M1 + M2) * 2 * (int)sizeof(T) + REAL_BYTES; }
    static constexpr int combine_bytes() { return BARS + (SLAB_C + M1 + M2) * 2 * (int)sizeof(T) + 2 * REAL_BYTES; }
};

// slab x of (slot, fld); the body of k_mid_pf and of the persistent step kernel
template <typename T, int MT, int FM0, int FM1, int FM2>
__device__ __forceinline__ void mid_pf_body(const PropsArgs<T> &a, int s, int x, int fld, int slot,
                                            unsigned char *smem_raw)
{
    using L = SlabSmem<T, FM1, FM2>;
    const Geo &g = a.g;
    constexpr int m1 = FM1, m2 = FM2, mk2 = L::MK2, M = FM0 * FM1 * FM2, Mk = FM0 * FM1 * L::MK2;
    constexpr int npz = ((m1 + 1) / 2) * m2;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw + L::BARS);
    cplx<T> *bufB = bufA + L::SLAB_C;
    cplx<T> *twy = bufB + L::SLAB_C;
    cplx<T> *twz = twy + m1;
    T *E4s = reinterpret_cast<T *>(twz + m2);
    const size_t slab_r = (size_t)x * m1 * m2, slab_k = (size_t)x * m1 * mk2;
    const T *E4g = etab_ptr(a, slot, etab_sel(g, fld, s)) + slab_r;
    cplx<T> *specA = a.spec + ((size_t)slot * 2 + fld) * 2 * Mk;
    cplx<T> *specB = specA + Mk;
    T *P = a.pbuf + ((size_t)slot * 2 + fld) * M + slab_r;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 3; i++) mbar_init(&bars[i], 1);
        mbar_fence_init();
        mbar_expect_tx(&bars[0], L::SPEC_BYTES);
        bulk_g2s(bufB, specB + slab_k, L::SPEC_BYTES, &bars[0]);
        mbar_expect_tx(&bars[1], L::REAL_BYTES);
        bulk_g2s(E4s, E4g, L::REAL_BYTES, &bars[1]);
        mbar_expect_tx(&bars[2], L::SPEC_BYTES);
        bulk_g2s(bufA, specA + slab_k, L::SPEC_BYTES, &bars[2]);
    }
    for (int i = threadIdx.x; i < m1; i += MT) twy[i] = a.tw[FM0 + i];
    for (int i = threadIdx.x; i < m2; i += MT) twz[i] = a.tw[FM0 + m1 + i];
    __syncthreads();
    // full step: P = E2 * qs1
    mbar_wait(&bars[0], 0, a.err);
    slab_inverse_fixed<T, m1, m2, MT>(bufB, twy, twz);
    mbar_wait(&bars[1], 0, a.err);
    for (int e = threadIdx.x; e < npz; e += MT) {
        const int p = e / m2, z = e - p * m2;
        const cplx<T> c = bufB[prow<FM2>(p, mk2) + z];
        const int r0 = 2 * p * m2 + z;
        const T e0 = E4s[r0];
        P[r0] = c.x * (e0 * e0);
        if (2 * p + 1 < m1) {
            const T e1 = E4s[r0 + m2];
            P[r0 + m2] = c.y * (e1 * e1);
        }
    }
    // second half step input: E2 * (first half step)
    mbar_wait(&bars[2], 0, a.err);
    slab_inverse_fixed<T, m1, m2, MT>(bufA, twy, twz);
    for (int e = threadIdx.x; e < npz; e += MT) {
        const int p = e / m2, z = e - p * m2;
        cplx<T> &c = bufA[prow<FM2>(p, mk2) + z];
        const int r0 = 2 * p * m2 + z;
        const T e0 = E4s[r0];
        c.x *= e0 * e0;
        if (2 * p + 1 < m1) {
            const T e1 = E4s[r0 + m2];
            c.y *= e1 * e1;
        } else {
            c.y = (T)0;
        }
    }
    __syncthreads();
    slab_forward_fixed<T, m1, m2, MT>(bufA, twy, twz);
    for (int i = threadIdx.x; i < m1 * mk2; i += MT) specA[slab_k + i] = bufA[i];
}

// combine with prefetch: mode 0 (Richardson), 1 (q = 1), 2 (q from the store)
template <typename T, int MT, int FM0, int FM1, int FM2>
__device__ __forceinline__ void combine_pf_body(const PropsArgs<T> &a, int s, int mode, int x, int fld, int slot,
                                                unsigned char *smem_raw)
{
    using L = SlabSmem<T, FM1, FM2>;
    const Geo &g = a.g;
    constexpr int m1 = FM1, m2 = FM2, mk2 = L::MK2, M = FM0 * FM1 * FM2, Mk = FM0 * FM1 * L::MK2;
    constexpr int npz = ((m1 + 1) / 2) * m2;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw + L::BARS);
    cplx<T> *twy = buf + L::SLAB_C;
    cplx<T> *twz = twy + m1;
    T *Q = reinterpret_cast<T *>(twz + m2);  // P, then q'
    T *E = Q + L::REAL;                        // E4 of step s (or of step s+1)
    const size_t slab_r = (size_t)x * m1 * m2, slab_k = (size_t)x * m1 * mk2;
    cplx<T> *specA = a.spec + ((size_t)slot * 2 + fld) * 2 * Mk;
    cplx<T> *specB = specA + Mk;
    const int sn = s + 1;
    T *qn = a.hist + hist_off<T>(g, slot, sn, fld) + slab_r;
    const bool next = sn < g.Ns;
    const int sel_n = next ? etab_sel(g, fld, sn) : 0;
    const int sel_s = mode == 0 ? etab_sel(g, fld, s) : sel_n;
    // E holds the table of step s; the next step reads it from shared memory
    // unless it switches blocks there (s+1 == n1 or n2), then from global
    const bool e_next_shared = sel_s == sel_n;
    const T *E4n_g = etab_ptr(a, slot, sel_n) + slab_r;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 3; i++) mbar_init(&bars[i], 1);
        mbar_fence_init();
        if (mode == 0) {
            mbar_expect_tx(&bars[0], L::SPEC_BYTES);
            bulk_g2s(buf, specA + slab_k, L::SPEC_BYTES, &bars[0]);
            mbar_expect_tx(&bars[1], L::REAL_BYTES);
            bulk_g2s(Q, a.pbuf + ((size_t)slot * 2 + fld) * M + slab_r, L::REAL_BYTES, &bars[1]);
        } else if (mode == 2) {
            mbar_expect_tx(&bars[1], L::REAL_BYTES);
            bulk_g2s(Q, qn, L::REAL_BYTES, &bars[1]);
        }
        if (mode == 0 || next) {
            mbar_expect_tx(&bars[2], L::REAL_BYTES);
            bulk_g2s(E, etab_ptr(a, slot, sel_s) + slab_r, L::REAL_BYTES, &bars[2]);
        }
    }
    for (int i = threadIdx.x; i < m1; i += MT) twy[i] = a.tw[FM0 + i];
    for (int i = threadIdx.x; i < m2; i += MT) twz[i] = a.tw[FM0 + m1 + i];
    __syncthreads();
    if (mode == 0) {
        mbar_wait(&bars[0], 0, a.err);
        slab_inverse_fixed<T, m1, m2, MT>(buf, twy, twz);
        mbar_wait(&bars[1], 0, a.err);
        mbar_wait(&bars[2], 0, a.err);
        for (int e = threadIdx.x; e < npz; e += MT) {
            const int p = e / m2, z = e - p * m2;
            const cplx<T> c = buf[prow<FM2>(p, mk2) + z];
            const int r0 = 2 * p * m2 + z;
            // Richardson, GPU_kernels.h:199-203
            const T q0 = (c.x * E[r0] * (T)4 - Q[r0]) / (T)3;
            Q[r0] = q0;
            qn[r0] = q0;
            if (2 * p + 1 < m1) {
                const int r1 = r0 + m2;
                const T q1 = (c.y * E[r1] * (T)4 - Q[r1]) / (T)3;
                Q[r1] = q1;
                qn[r1] = q1;
            }
        }
    } else if (mode == 1) {
        for (int r = threadIdx.x; r < m1 * m2; r += MT) {
            Q[r] = (T)1;
            qn[r] = (T)1;
        }
    } else {
        mbar_wait(&bars[1], 0, a.err);
    }
    if (!next) return;
    if (mode != 0) mbar_wait(&bars[2], 0, a.err);
    __syncthreads();
    const T *En = e_next_shared ? E : E4n_g;
    // half step input E4' q'
    for (int e = threadIdx.x; e < npz; e += MT) {
        const int p = e / m2, z = e - p * m2;
        const int r0 = 2 * p * m2 + z;
        const bool hb = 2 * p + 1 < m1;
        buf[prow<FM2>(p, mk2) + z] = {Q[r0] * En[r0], hb ? Q[r0 + m2] * En[r0 + m2] : (T)0};
    }
    __syncthreads();
    slab_forward_fixed<T, m1, m2, MT>(buf, twy, twz);
    for (int i = threadIdx.x; i < m1 * mk2; i += MT) specA[slab_k + i] = buf[i];
    __syncthreads();
    // full step input E2' q'
    for (int e = threadIdx.x; e < npz; e += MT) {
        const int p = e / m2, z = e - p * m2;
        const int r0 = 2 * p * m2 + z;
        const T e0 = En[r0];
        T v1 = (T)0;
        if (2 * p + 1 < m1) {
            const T e1 = En[r0 + m2];
            v1 = Q[r0 + m2] * (e1 * e1);
        }
        buf[prow<FM2>(p, mk2) + z] = {Q[r0] * (e0 * e0), v1};
    }
    __syncthreads();
    slab_forward_fixed<T, m1, m2, MT>(buf, twy, twz);
    for (int i = threadIdx.x; i < m1 * mk2; i += MT) specB[slab_k + i] = buf[i];
}

// ---------------------------------------------------------------- TMA pencil
// The x pass of a compile-time shape with the column tiles moved by 2-D
// tensor-map copies: the spectra of every slot are one 2-D array of
// (nslots*2*2*m0) rows by 2*m1*mk2 reals; a tile is the box {2*tc, m0}.
// Both spectra of a both-pass are requested at kernel start, so the second
// one lands while the first is transformed; results leave through tile stores.
template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__device__ __forceinline__ void pencil_tma_body(const CUtensorMap &tmap, const PropsArgs<T> &a, int both, int tile,
                                                int fld, int slot, unsigned char *smem_raw)
{
    constexpr int m0 = FM0, m1 = FM1, mk2 = FM2 / 2 + 1;
    constexpr int BOX = TC * m0;                      // complex elements per tile
    constexpr uint32_t BOX_BYTES = BOX * 2 * sizeof(T);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    cplx<T> *bufA = reinterpret_cast<cplx<T> *>(smem_raw + 128);
    cplx<T> *bufB = bufA + BOX;
    cplx<T> *twx = bufB + BOX;
    T *colf = reinterpret_cast<T *>(twx + m0);
    T *gx = colf + TC;
    const int ncol = m1 * mk2, c0 = tile * TC;
    const int x = 2 * c0;
    const int y0 = (((a.slot0 + slot) * 2 + fld) * 2) * m0;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
        mbar_expect_tx(&bars[0], BOX_BYTES);
        tma_load_2d(bufA, &tmap, x, y0, &bars[0]);
        if (both) {
            mbar_expect_tx(&bars[1], BOX_BYTES);
            tma_load_2d(bufB, &tmap, x, y0 + m0, &bars[1]);
        }
    }
    const T *kf = a.kfac + (size_t)a.slot_rep[slot] * a.kf_stride;  // the replica's box
    for (int i = threadIdx.x; i < m0; i += MT) {
        twx[i] = a.tw[i];
        gx[i] = kf[i];
    }
    for (int t = threadIdx.x; t < TC; t += MT) {
        const int c = c0 + t;
        const int yy = c / mk2, kz = c - yy * mk2;
        colf[t] = c < ncol ? kf[m0 + yy] * kf[m0 + m1 + kz] : (T)0;
    }
    __syncthreads();
    const T invM = a.invM;
    const int npass = both ? 2 : 1;
    for (int pass = 0; pass < npass; pass++) {
        cplx<T> *buf = pass == 0 ? bufA : bufB;
        mbar_wait(&bars[pass], 0, a.err);
        // x forward, times the diffusion factor, x inverse; bin xx of column t:
        // pass 0: K2 = g/M ; pass 1: K1 = g^2/M  (Prepare_dev_expKsq2_expKsq, GPU_kernels.h:207-213)
        const T Mreal = a.Mreal;
        fft_fwd_mul_inv<T, m0, TC, TC, 1, true, MT>(buf, twx, [&](cplx<T> &v, int t, int xx) {
            const T k2 = gx[xx] * colf[t];
            const T f = pass == 0 ? k2 * invM : (k2 * invM) * (k2 * invM) * Mreal;
            v.x *= f;
            v.y *= f;
        });
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) tma_store_2d(&tmap, x, y0 + pass * m0, buf);
    }
    if (threadIdx.x == 0) tma_store_wait_read();
}

template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 3 : 2) : 1)
    k_pencil_tma(const __grid_constant__ CUtensorMap tmap, PropsArgs<T> a, int both)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    pencil_tma_body<T, MT, FM0, FM1, FM2, TC>(tmap, a, both, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ---------------------------------------------------------------- shuffle pencil (m0 = 64)
// Opt-in (SCFT_PENCIL_SHUFFLE=1): on the 16-replica 64^3 string it measured
// as fast as the Stockham pencil at the same tile width and 2 % slower than
// its wide tiles, because in the full pipeline the x pass is bound by moving
// the spectra, not by its barriers.
// The x pass of the m0 = 64 shapes with the transforms in registers: each
// column of a tile is one octet of lanes (octet_fft64_fwd / _inv), so a
// transform, the diffusion factor and the inverse transform run without a
// shared-memory round trip or a CTA barrier.  The tiles arrive through the
// spectrum tensor map with 128-byte swizzling, in boxes of 128 bytes by m0
// rows: element (x, c) of a box sits in 16-byte chunk (c-chunk XOR x mod 8)
// of row x, so the eight lanes of an octet, which read rows s + 8 j of one
// column, hit eight different chunks (ncu still counts about a fifth of the
// FP32 tile wavefronts as bank conflicts).  Shared layout: mbarriers at 0, the x factors at 128, the
// column factors at 640, the tiles from the next 1024-byte boundary (the
// swizzle pattern repeats every 1024 bytes).
template <typename T>
struct PencilSh {
    static constexpr int CPB = 128 / (int)sizeof(cplx<T>);  // complex elements per box row
    static constexpr int BOXW = 128 / (int)sizeof(T);        // box width in reals
    static constexpr int HEADER = 1024;
    // dynamic shared memory of a tile of tc columns and m0 rows, both spectra
    static __host__ __device__ constexpr int smem(int tc, int m0)
    {
        return HEADER + 1023 + 2 * tc * m0 * (int)sizeof(cplx<T>);
    }
    // complex index of element (x, c) of a tile
    static __device__ __forceinline__ int at(int x, int c, int m0)
    {
        const int b = c / CPB, cc = c % CPB;
        const int chunk = sizeof(T) == 4 ? cc >> 1 : cc;
        const int sw = chunk ^ (x & 7);
        return b * CPB * m0 + x * CPB + (sizeof(T) == 4 ? (sw << 1) | (cc & 1) : sw);
    }
};

template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__device__ __forceinline__ void pencil_sh_body(const CUtensorMap &tmap, const PropsArgs<T> &a, int both, int tile,
                                               int fld, int slot, unsigned char *smem_raw)
{
    static_assert(FM0 == 64, "octet transforms are 64-point");
    using P = PencilSh<T>;
    static_assert(TC % P::CPB == 0 && (TC % 4) == 0, "tile of whole boxes and whole warps");
    constexpr int m0 = FM0, m1 = FM1, mk2 = FM2 / 2 + 1;
    constexpr int NBOX = TC / P::CPB;
    constexpr int TILE = TC * m0;  // complex elements per spectrum tile
    constexpr uint32_t BOX_BYTES = 128u * m0;
    constexpr int NO = MT / 8;  // octets
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    T *gx = reinterpret_cast<T *>(smem_raw + 128);
    T *colf = reinterpret_cast<T *>(smem_raw + 640);
    const uint32_t base = smem_addr(smem_raw + P::HEADER);
    cplx<T> *buf0 = reinterpret_cast<cplx<T> *>(smem_raw + P::HEADER + ((1024u - (base & 1023u)) & 1023u));
    const int ncol = m1 * mk2, c0 = tile * TC;
    const int x0 = 2 * c0;
    const int y0 = (((a.slot0 + slot) * 2 + fld) * 2) * m0;
    const int npass = both ? 2 : 1;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
        for (int p = 0; p < npass; p++) {
            mbar_expect_tx(&bars[p], NBOX * BOX_BYTES);
            for (int b = 0; b < NBOX; b++)
                tma_load_2d(buf0 + p * TILE + b * P::CPB * m0, &tmap, x0 + b * P::BOXW, y0 + p * m0, &bars[p]);
        }
    }
    const T *kf = a.kfac + (size_t)a.slot_rep[slot] * a.kf_stride;  // the replica's box
    for (int i = threadIdx.x; i < m0; i += MT) gx[i] = kf[i];
    for (int t = threadIdx.x; t < TC; t += MT) {
        const int c = c0 + t;
        const int yy = c / mk2, kz = c - yy * mk2;
        colf[t] = c < ncol ? kf[m0 + yy] * kf[m0 + m1 + kz] : (T)0;
    }
    const int s = threadIdx.x & 7, oct = threadIdx.x >> 3;
    cplx<T> w[8];
    octet_twiddles(w, a.tw, s);
    __syncthreads();
    const T invM = a.invM, Mreal = a.Mreal;
    const int nlines = npass * TC;
    int stored = 0;  // spectra whose tiles have been stored
#pragma unroll 1
    for (int l0 = 0; l0 < nlines; l0 += NO) {
        const int line = l0 + oct;
        if (line < nlines) {  // whole warps: nlines and NO are multiples of 4 octets
            const int pass = line / TC, t = line - pass * TC;
            cplx<T> *buf = buf0 + pass * TILE;
            mbar_wait(&bars[pass], 0, a.err);
            cplx<T> v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = buf[P::at(s + 8 * j, t, m0)];
            octet_fft64_fwd(v, w, s);
            // bin s + 8 j of column t: pass 0: K2 = g/M ; pass 1: K1 = g^2/M
            // (Prepare_dev_expKsq2_expKsq, GPU_kernels.h:207-213)
            const T ct = colf[t];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const T k2 = gx[s + 8 * j] * ct;
                const T f = pass == 0 ? k2 * invM : (k2 * invM) * (k2 * invM) * Mreal;
                v[j].x *= f;
                v[j].y *= f;
            }
            octet_fft64_inv(v, w, s);
#pragma unroll
            for (int j = 0; j < 8; j++) buf[P::at(s + 8 * j, t, m0)] = v[j];
        }
        // spectra completed by this round of lines leave through tile stores
        const int done = min(npass, (l0 + NO) / TC);
        if (done > stored) {
            fence_proxy_async_smem();
            __syncthreads();
            if (threadIdx.x == 0)
                for (int p = stored; p < done; p++)
                    for (int b = 0; b < NBOX; b++)
                        tma_store_2d(&tmap, x0 + b * P::BOXW, y0 + p * m0, buf0 + p * TILE + b * P::CPB * m0);
            stored = done;
        }
    }
    if (threadIdx.x == 0) tma_store_wait_read();
}

template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 3 : 2) : 1)
    k_pencil_sh(const __grid_constant__ CUtensorMap tmap, PropsArgs<T> a, int both)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    pencil_sh_body<T, MT, FM0, FM1, FM2, TC>(tmap, a, both, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 4 : 2) : 1) k_mid_pf(PropsArgs<T> a, int s)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    mid_pf_body<T, MT, FM0, FM1, FM2>(a, s, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 4 : 2) : 1) k_combine_pf(PropsArgs<T> a, int s, int mode)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    combine_pf_body<T, MT, FM0, FM1, FM2>(a, s, mode, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ---------------------------------------------------------------- one launch per contour step
// The persistent form of the four launches above for the compile-time
// shapes: CTAs claim work items from a counter in a fixed order -- every
// pencil(both) tile, then every mid slab, every pencil(A) tile, every combine
// slab, each phase ordered by (slot, field) -- and an item waits only for the
// items of the previous phase of its own (slot, field).  Items are claimed in
// order by running CTAs, so whatever an item waits for is held by a CTA that
// is running or done: no residency assumption is needed.  Completion
// counters are cumulative over the steps of a props round (n_p (s+1) items of
// phase p are done after step s) and zeroed with the claim counters when the
// round starts.  Every wait is bounded (2^22 polls of ~32 ns) and records
// error 3 when it gives up, which ends the kernel.
//
// The items move data between CTAs of one launch through both proxies: tile
// stores (async proxy) feed the slab kernels' bulk loads, and the slab
// kernels' generic stores feed the next pencil's tile loads.  A producer waits
// for its bulk stores to complete, fences the async proxy against the generic
// one and releases its counter; a consumer acquires the counter and fences the
// generic proxy against the async one before it issues bulk loads.  Shared
// memory is reused across items, so every item starts with an async-proxy
// fence over the previous item's generic shared accesses, and the mbarriers
// of an item are invalidated before the next one initialises them.
constexpr uint32_t kStepSpinPF = 1u << 22;

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_all()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// The three roles out of line: each is then register-allocated as in its own
// kernel; inlined together they spilled kilobytes per thread.
template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__device__ __noinline__ void pencil_tma_call(const CUtensorMap *tmap, const PropsArgs<T> *a, int both, int tile,
                                             int fld, int slot, unsigned char *smem_raw)
{
    pencil_tma_body<T, MT, FM0, FM1, FM2, TC>(*tmap, *a, both, tile, fld, slot, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__device__ __noinline__ void pencil_sh_call(const CUtensorMap *tmap, const PropsArgs<T> *a, int both, int tile,
                                            int fld, int slot, unsigned char *smem_raw)
{
    if constexpr (FM0 == 64) pencil_sh_body<T, MT, FM0, FM1, FM2, TC>(*tmap, *a, both, tile, fld, slot, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2>
__device__ __noinline__ void mid_pf_call(const PropsArgs<T> *a, int s, int x, int fld, int slot, unsigned char *smem_raw)
{
    mid_pf_body<T, MT, FM0, FM1, FM2>(*a, s, x, fld, slot, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2>
__device__ __noinline__ void combine_pf_call(const PropsArgs<T> *a, int s, int x, int fld, int slot,
                                             unsigned char *smem_raw)
{
    combine_pf_body<T, MT, FM0, FM1, FM2>(*a, s, 0, x, fld, slot, smem_raw);
}

template <typename T, int MT, int FM0, int FM1, int FM2, int TC>
__global__ void __launch_bounds__(MT, MT == 256 ? (sizeof(T) == 4 ? 4 : 2) : 1)
    k_step_pf(const __grid_constant__ CUtensorMap tmap, PropsArgs<T> a, int s, int nslots, int sh)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int item_sh[3], ok_sh;
    constexpr int ntiles = (FM1 * (FM2 / 2 + 1) + TC - 1) / TC;
    const int G = 2 * nslots;  // (slot, field) groups
    const int per[4] = {ntiles, FM0, ntiles, FM0};
    int *claim = a.sync + s;      // this step's claim counter
    int *done = a.sync + a.g.Ns;  // [phase][group] completion counters
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    for (;;) {
        fence_proxy_async_smem();
        if (threadIdx.x == 0) {
            int ph = -1, gr = 0, un = 0;
            if (!step_item(atomicAdd(claim, 1), G, per, ph, gr, un)) ph = -1;
            item_sh[0] = ph;
            item_sh[1] = gr;
            item_sh[2] = un;
        }
        __syncthreads();
        const int phase = item_sh[0], group = item_sh[1], unit = item_sh[2];
        if (phase < 0) break;
        const int slot = group >> 1, fld = group & 1;
        if (phase > 0) {
            if (threadIdx.x == 0) {
                const int need = per[phase - 1] * (s + 1);
                const int *cnt = done + (phase - 1) * G + group;
                uint32_t i = 0;
                while (ld_acquire_gpu(cnt) < need && i < kStepSpinPF) {
                    __nanosleep(32);
                    i++;
                }
                ok_sh = i < kStepSpinPF;
                if (!ok_sh) *a.err = 3;
                fence_proxy_async_global();
            }
            __syncthreads();
            if (!ok_sh) return;
        }
        int nbar;
        if (phase == 0 || phase == 2) {
            if (sh)
                pencil_sh_call<T, MT, FM0, FM1, FM2, TC>(&tmap, &a, phase == 0, unit, fld, slot, smem_raw);
            else
                pencil_tma_call<T, MT, FM0, FM1, FM2, TC>(&tmap, &a, phase == 0, unit, fld, slot, smem_raw);
            nbar = 2;
            if (threadIdx.x == 0) {
                bulk_wait_all();  // the tile stores have reached global memory
                fence_proxy_async_global();
            }
        } else if (phase == 1) {
            mid_pf_call<T, MT, FM0, FM1, FM2>(&a, s, unit, fld, slot, smem_raw);
            nbar = 3;
        } else {
            combine_pf_call<T, MT, FM0, FM1, FM2>(&a, s, unit, fld, slot, smem_raw);
            nbar = 3;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int i = 0; i < nbar; i++) mbar_inval(&bars[i]);
            __threadfence();
            atomicAdd(done + phase * G + group, 1);
        }
    }
}

// ---------------------------------------------------------------- bounded-wait self-test
// One CTA waits on an mbarrier that expects 16 transaction bytes no copy will
// deliver (none is issued), so every thread's wait runs out after `polls`
// polls, records error 3 in the error word and returns: the path a lost bulk
// copy takes, exercised without any copy in flight.
__global__ void k_wait_selftest(int *err, uint32_t polls)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
        mbar_expect_tx(&bar, 16);
    }
    __syncthreads();
    mbar_wait(&bar, 0, err, polls);
    __syncthreads();
    if (threadIdx.x == 0) mbar_inval(&bar);
}

int launch_wait_selftest(int *err, unsigned polls, cudaStream_t st)
{
    k_wait_selftest<<<1, 32, 0, st>>>(err, polls);
    return 1;
}

// ---------------------------------------------------------------- Q and densities
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
    return t;  // valid in thread 0
}

// partial sums of q^dagger(Nh) and q(Ns) (reduction_sum, GPU_kernels.h:58-90)
template <typename T>
__global__ void k_qsum(PropsArgs<T> a)
{
    __shared__ double sh[32];
    const Geo &g = a.g;
    const int slot = blockIdx.y;
    const T *q2 = a.hist + hist_off<T>(g, slot, g.Nh, 1);
    const T *q1 = a.hist + hist_off<T>(g, slot, g.Ns, 0);
    double s2 = 0, s1 = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < g.M; r += gridDim.x * blockDim.x) {
        s2 += (double)q2[r];
        s1 += (double)q1[r];
    }
    double t2 = block_sum(s2, sh);
    double t1 = block_sum(s1, sh);
    if (threadIdx.x == 0) {
        double *pp = a.partials + (size_t)slot * a.npart_stride;
        pp[0 * gridDim.x + blockIdx.x] = t2;
        pp[1 * gridDim.x + blockIdx.x] = t1;
    }
}

// Q2, QC, lnQ and the ensemble weights (density.h:376-399); one block per slot
template <typename T>
__global__ void k_qfinal(PropsArgs<T> a, int nblk)
{
    const int slot = blockIdx.x;
    if (threadIdx.x != 0) return;
    const double *pp = a.partials + (size_t)slot * a.npart_stride;
    double Q2 = 0, QC = 0;
    for (int i = 0; i < nblk; i++) Q2 += pp[i];
    for (int i = 0; i < nblk; i++) QC += pp[nblk + i];
    const double M = (double)a.g.M;
    Q2 /= M;
    QC /= M;
    const int rep = a.slot_rep[slot];
    double *rs = a.rs + (size_t)rep * kRsStride;
    const double phic = a.phic, alpha = a.alpha;
    double zB, zC, lnQ;
    if (a.ens == 1) {
        lnQ = phic * log(QC) + ((1.0 - phic) / alpha) * log(Q2);
        zB = (1.0 - phic) / (Q2 * alpha);
        zC = phic / QC;
    } else {
        zB = 1.0;
        zC = phic;
        lnQ = zB * Q2 + zC * QC;  // zA*Q1 = 0
    }
    rs[kRsQ2] = Q2;
    rs[kRsQC] = QC;
    rs[kRsLnQ] = lnQ;
    rs[kRsZB] = zB;
    rs[kRsZC] = zC;
}

__device__ __forceinline__ void kahan_add(double &sum, double &c, double term)
{
    const double y = term - c;
    const double t = sum + y;
    c = (t - sum) - y;
    sum = t;
}

// sum += w_s u(s) v(t - s) for s in [s0, s1) with Simpson interior weights
// 4, 2, 4, ... from s0 (the reference's loops, density.h:404-422), Kahan
// compensated, in the reference's order.  u, v are fields fu, fv of the
// propagator store at point r.  The loads of four consecutive terms are
// issued before their additions, so each thread keeps eight loads in flight
// instead of two.
template <typename T>
__device__ __forceinline__ void simpson_run(const T *h, size_t M, int r, int s0, int s1, int fu, int fv, int t,
                                            double &sum, double &c)
{
    int s = s0;
    for (; s + 3 < s1; s += 4) {
        double u[4], v[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            u[k] = (double)h[((size_t)(s + k) * 2 + fu) * M + r];
            v[k] = (double)h[((size_t)(t - s - k) * 2 + fv) * M + r];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) kahan_add(sum, c, (((s + k - s0) & 1) ? 2 : 4) * u[k] * v[k]);
    }
    for (; s < s1; s++)
        kahan_add(sum, c, (((s - s0) & 1) ? 2 : 4) * (double)h[((size_t)s * 2 + fu) * M + r] *
                              (double)h[((size_t)(t - s) * 2 + fv) * M + r]);
}

// Composite-Simpson densities (rA_rB_init_Ns_homo, rA_rB_mid_segments,
// scale_concentrations, sumconcs2: GPU_kernels.h:92-139; loops density.h:402-430).
// Weights 1, 4, 2, 4, ... restart at 4 for each block with no odd-count
// correction, as in the reference.  Products are formed and summed in FP64
// with Kahan compensation.  Also emits per-block partial sums of
// rC, rA, rB, rhA, rhB and (chi*(phiA+phiB-1))^2.
template <typename T>
__global__ void k_density(PropsArgs<T> a)
{
    __shared__ double sh[32];
    const Geo &g = a.g;
    const int slot = blockIdx.y;
    const int rep = a.slot_rep[slot];
    const double *rs = a.rs + (size_t)rep * kRsStride;
    const double zB = rs[kRsZB], zC = rs[kRsZC];
    const double ds = 1.0 / g.Ns;
    const int Ns = g.Ns, n1 = g.n1, n2 = g.n2, Nh = g.Nh;
    const size_t M = g.M;
    const T *h = a.hist + hist_off<T>(g, slot, 0, 0);
    double *conc = a.conc + (size_t)rep * 4 * M;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < (int)M; r += gridDim.x * blockDim.x) {
#define Q1(s) ((double)h[((size_t)(s) * 2 + 0) * M + r])
#define Q2(s) ((double)h[((size_t)(s) * 2 + 1) * M + r])
        double rhB = 2.0 * Q2(Nh), chB = 0;
        const double q12 = Q1(n1) * Q2(n2);
        double rCA = Q2(Ns) + q12, cA = 0;
        double rCB = Q1(Ns) + q12, cB = 0;
        simpson_run(h, M, r, 1, Nh, 1, 1, Nh, rhB, chB);     // Q2(s) Q2(Nh - s)
        simpson_run(h, M, r, 1, n1, 0, 1, Ns, rCA, cA);      // Q1(s) Q2(Ns - s)
        simpson_run(h, M, r, n1 + 1, Ns, 0, 1, Ns, rCB, cB); // Q1(s) Q2(Ns - s)
        if (g.jon) {
            // continuous A fraction: theta of the junction step's trapezoid
            // weight moves from the B block to the A block (3/2 here: the sums
            // are scaled by ds/3 below)
            const double tj = 1.5 * g.theta * (Q1(n1) * Q2(Ns - n1) + Q1(n1 + 1) * Q2(Ns - n1 - 1));
            rCA += tj;
            rCB -= tj;
        }
#undef Q1
#undef Q2
        const double rhA = 0.0;  // the A-homopolymer density is scaled by zA = 0
        rhB = rhB * zB * ds / 3.0;
        rCA = rCA * zC * ds / 3.0;
        rCB = rCB * zC * ds / 3.0;
        const double rA = rhA + rCA, rB = rhB + rCB;
        conc[r] = rA;
        conc[r + M] = rB;
        conc[r + 2 * M] = rhA + rhB;
        conc[r + 3 * M] = rCB;
        const double dv = a.chi * (rB + rA - 1.0);
        acc[0] += rCA + rCB;
        acc[1] += rA;
        acc[2] += rB;
        acc[3] += rhA;
        acc[4] += rhB;
        acc[5] += dv * dv;
    }
    double *pp = a.partials + (size_t)slot * a.npart_stride;
    for (int i = 0; i < 6; i++) {
        double t = block_sum(acc[i], sh);
        if (threadIdx.x == 0) pp[i * gridDim.x + blockIdx.x] = t;
    }
}

// phis (density.h:433-454) and the W+ residual sum of solve_field0 (scft.cu:527-535)
template <typename T>
__global__ void k_dfinal(PropsArgs<T> a, int nblk)
{
    const int slot = blockIdx.x;
    if (threadIdx.x != 0) return;
    const double *pp = a.partials + (size_t)slot * a.npart_stride;
    const int rep = a.slot_rep[slot];
    double *rs = a.rs + (size_t)rep * kRsStride;
    double v[6];
    for (int k = 0; k < 6; k++) {
        double t = 0;
        for (int i = 0; i < nblk; i++) t += pp[k * nblk + i];
        v[k] = t;
    }
    const double M = (double)a.g.M;
    for (int k = 0; k < 5; k++) rs[kRsPhis + k] = v[k] / M;
    rs[kRsDev2] = v[5];
}

// ---------------------------------------------------------------- launchers
// MT bounds the CTA size of the FFT kernels.  Shapes with compile-time
// instantiations (cubic 32..128 and 64x64x96) use MT threads exactly; the
// runtime-shaped kernels use 256 (or 1024 for slabs too large for 256).
// the 64^3 FP32 shape with L.reg set runs the register-resident kernels of reg64.cu
template <typename T, int F0, int F1, int F2>
constexpr bool kReg64 = sizeof(T) == 4 && F0 == 64 && F1 == 64 && F2 == 64;

template <typename T, int MT, int F0, int F1, int F2>
void launch_combine(const PropsArgs<T> &a, const PropsLaunch &L, dim3 gs, int s, int mode, cudaStream_t st)
{
    if constexpr (kReg64<T, F0, F1, F2>) {
        if (L.reg) {
            reg64_combine(a, gs.z, s, mode, st);
            return;
        }
    }
    if constexpr (F1 != 0) {
        if (L.pf) {
            k_combine_pf<T, MT, F0, F1, F2><<<gs, MT, L.combine_pf_smem, st>>>(a, s, mode);
            return;
        }
    }
    k_combine<T, MT, F0, F1, F2><<<gs, L.slab_threads, L.slab_smem, st>>>(a, s, mode);
}

template <typename T, int MT, int F0, int F1, int F2>
void launch_mid(const PropsArgs<T> &a, const PropsLaunch &L, dim3 gs, int s, cudaStream_t st)
{
    if constexpr (kReg64<T, F0, F1, F2>) {
        if (L.reg) {
            reg64_mid(a, gs.z, s, st);
            return;
        }
    }
    if constexpr (F1 != 0) {
        if (L.pf) {
            k_mid_pf<T, MT, F0, F1, F2><<<gs, MT, L.mid_pf_smem, st>>>(a, s);
            return;
        }
    }
    k_mid<T, MT, F0, F1, F2><<<gs, L.slab_threads, L.slab_smem, st>>>(a, s);
}

template <typename T, int MT, int F0, int F1, int F2>
void launch_pencil(const PropsArgs<T> &a, const PropsLaunch &L, dim3 gp, int both, cudaStream_t st)
{
    if constexpr (kReg64<T, F0, F1, F2>) {
        if (L.reg) {
            reg64_pencil(a, gp.z, both, st);
            return;
        }
    }
    if constexpr (F1 != 0) {
        if (L.tma_pencil) {
            // tile width: kTile columns, or twice that (two butterflies per
            // thread between barriers) when the autotuner picked it
            constexpr int TC = kTile<T>::value, ncol = F1 * (F2 / 2 + 1);
            if constexpr (F0 == 64) {
                if (L.pencil_sh) {
                    if (L.ptile_wide)
                        k_pencil_sh<T, MT, F0, F1, F2, 2 * TC><<<dim3((ncol + 2 * TC - 1) / (2 * TC), gp.y, gp.z), MT,
                                                                 L.pencil_tma_smem_wide, st>>>(*L.tmap_wide, a, both);
                    else
                        k_pencil_sh<T, MT, F0, F1, F2, TC><<<dim3((ncol + TC - 1) / TC, gp.y, gp.z), MT,
                                                             L.pencil_tma_smem, st>>>(*L.tmap, a, both);
                    return;
                }
            }
            if (L.ptile_wide)
                k_pencil_tma<T, MT, F0, F1, F2, 2 * TC><<<dim3((ncol + 2 * TC - 1) / (2 * TC), gp.y, gp.z), MT,
                                                          L.pencil_tma_smem_wide, st>>>(*L.tmap_wide, a, both);
            else
                k_pencil_tma<T, MT, F0, F1, F2, TC><<<dim3((ncol + TC - 1) / TC, gp.y, gp.z), MT, L.pencil_tma_smem,
                                                      st>>>(*L.tmap, a, both);
            return;
        }
    }
    k_pencil<T, MT, F0, F1, F2><<<gp, L.pencil_threads, L.pencil_smem, st>>>(a, both);
}

template <typename T, int MT, int F0, int F1, int F2>
int launch_props_mt(const PropsArgs<T> &a, const PropsLaunch &L, int nslots, cudaStream_t st)
{
    const Geo &g = a.g;
    dim3 gs(g.m0, 2, nslots), gp(g.ncol_tiles, 2, nslots);
    k_prepare<T><<<dim3(L.ew_blocks, nslots), 256, 0, st>>>(a);
    int n = 6;
    if constexpr (kReg64<T, F0, F1, F2>) {
        if (L.reg && L.persist) {
            // one persistent launch per contour step (reg64.cu); its counters start at zero
            cudaMemsetAsync(a.sync, 0, sizeof(int) * reg64_sync_ints(g.Ns, nslots), st);
            launch_combine<T, MT, F0, F1, F2>(a, L, gs, -1, 1, st);
            for (int s = 0; s < g.Ns; s++) reg64_step(a, nslots, s, L.step_grid, st);
            n += g.Ns;
        }
    }
    if constexpr (F1 != 0) {
        if (n == 6 && !L.reg && L.persist && L.pf && L.tma_pencil && a.sync) {
            // one persistent launch per contour step on the shared-memory kernels
            constexpr int TC = kTile<T>::value;
            cudaMemsetAsync(a.sync, 0, sizeof(int) * reg64_sync_ints(g.Ns, nslots), st);
            launch_combine<T, MT, F0, F1, F2>(a, L, gs, -1, 1, st);
            for (int s = 0; s < g.Ns; s++) {
                if (L.ptile_wide)
                    k_step_pf<T, MT, F0, F1, F2, 2 * TC><<<L.step_grid_pf, MT, L.step_pf_smem, st>>>(
                        *L.tmap_wide, a, s, nslots, L.pencil_sh);
                else
                    k_step_pf<T, MT, F0, F1, F2, TC><<<L.step_grid_pf, MT, L.step_pf_smem, st>>>(*L.tmap, a, s, nslots,
                                                                                                L.pencil_sh);
            }
            n += g.Ns;
        }
    }
    if (n == 6) {
        launch_combine<T, MT, F0, F1, F2>(a, L, gs, -1, 1, st);
        for (int s = 0; s < g.Ns; s++) {
            launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 1, st);
            launch_mid<T, MT, F0, F1, F2>(a, L, gs, s, st);
            launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 0, st);
            launch_combine<T, MT, F0, F1, F2>(a, L, gs, s, 0, st);
        }
        n += 4 * g.Ns;
    }
    k_qsum<T><<<dim3(L.red_blocks, nslots), 256, 0, st>>>(a);
    k_qfinal<T><<<nslots, 32, 0, st>>>(a, L.red_blocks);
    k_density<T><<<dim3(L.red_blocks, nslots), 256, 0, st>>>(a);
    k_dfinal<T><<<nslots, 32, 0, st>>>(a, L.red_blocks);
    return n;
}

// one contour step s of slot 0 starting from the propagator store slice s
template <typename T, int MT, int F0, int F1, int F2>
int launch_single_step_mt(const PropsArgs<T> &a, const PropsLaunch &L, int s, cudaStream_t st)
{
    const Geo &g = a.g;
    dim3 gs(g.m0, 2, 1), gp(g.ncol_tiles, 2, 1);
    k_prepare<T><<<dim3(L.ew_blocks, 1), 256, 0, st>>>(a);
    launch_combine<T, MT, F0, F1, F2>(a, L, gs, s - 1, 2, st);
    launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 1, st);
    launch_mid<T, MT, F0, F1, F2>(a, L, gs, s, st);
    launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 0, st);
    launch_combine<T, MT, F0, F1, F2>(a, L, gs, s, 0, st);
    return 6;
}

// A chain segment of slot 0 (checkpointed adjoint): q and q^dagger advanced
// g.Ns steps from store slice 0 (first_mode 2) or from q = 1 (first_mode 1).
// The segment's Geo carries n1 and n2 minus the segment's first contour index,
// so every step picks the E table of its absolute index.
template <typename T, int MT, int F0, int F1, int F2>
int launch_chain_mt(const PropsArgs<T> &a, const PropsLaunch &L, int first_mode, cudaStream_t st)
{
    const Geo &g = a.g;
    dim3 gs(g.m0, 2, 1), gp(g.ncol_tiles, 2, 1);
    launch_combine<T, MT, F0, F1, F2>(a, L, gs, -1, first_mode, st);
    for (int s = 0; s < g.Ns; s++) {
        launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 1, st);
        launch_mid<T, MT, F0, F1, F2>(a, L, gs, s, st);
        launch_pencil<T, MT, F0, F1, F2>(a, L, gp, 0, st);
        launch_combine<T, MT, F0, F1, F2>(a, L, gs, s, 0, st);
    }
    return 1 + 4 * g.Ns;
}

template <typename T, int MT, int F0, int F1, int F2>
int set_smem_mt(const PropsLaunch &L)
{
    cudaError_t e1 = raise_dyn_smem(k_combine<T, MT, F0, F1, F2>, L.slab_smem);
    cudaError_t e2 = raise_dyn_smem(k_mid<T, MT, F0, F1, F2>, L.slab_smem);
    cudaError_t e3 = raise_dyn_smem(k_pencil<T, MT, F0, F1, F2>, L.pencil_smem);
    cudaError_t e4 = cudaSuccess, e5 = cudaSuccess;
    if constexpr (F1 != 0) {
        if (L.tma_pencil) {
            e4 = raise_dyn_smem(k_pencil_tma<T, MT, F0, F1, F2, kTile<T>::value>, L.pencil_tma_smem);
            if (e4 == cudaSuccess && L.tmap_wide)
                e4 = raise_dyn_smem(k_pencil_tma<T, MT, F0, F1, F2, 2 * kTile<T>::value>, L.pencil_tma_smem_wide);
            if constexpr (F0 == 64) {
                if (e4 == cudaSuccess && L.pencil_sh) {
                    e4 = raise_dyn_smem(k_pencil_sh<T, MT, F0, F1, F2, kTile<T>::value>, L.pencil_tma_smem);
                    if (e4 == cudaSuccess && L.tmap_wide)
                        e4 = raise_dyn_smem(k_pencil_sh<T, MT, F0, F1, F2, 2 * kTile<T>::value>,
                                            L.pencil_tma_smem_wide);
                }
            }
        }
        if (e4 == cudaSuccess && L.pf) {
            e4 = raise_dyn_smem(k_combine_pf<T, MT, F0, F1, F2>, L.combine_pf_smem);
            e5 = raise_dyn_smem(k_mid_pf<T, MT, F0, F1, F2>, L.mid_pf_smem);
        }
    }
    int e6 = 0;
    if constexpr (kReg64<T, F0, F1, F2>) e6 = reg64_set_smem();
    if constexpr (F1 != 0) {
        if (L.pf && L.tma_pencil && L.step_pf_smem > 0) {
            constexpr int TC = kTile<T>::value;
            if (raise_dyn_smem(k_step_pf<T, MT, F0, F1, F2, TC>, L.step_pf_smem) != cudaSuccess) e6 = 1;
            if (L.tmap_wide && raise_dyn_smem(k_step_pf<T, MT, F0, F1, F2, 2 * TC>, L.step_pf_smem) != cudaSuccess)
                e6 = 1;
        }
    }
    return (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess && e4 == cudaSuccess && e5 == cudaSuccess &&
            e6 == 0)
               ? 0
               : -1;
}

// shared-memory bytes of the prefetching slab kernels for a fixed shape
template <typename T>
void pf_smem(int id, int &mid, int &comb)
{
    switch (id) {
        case 32: mid = SlabSmem<T, 32, 32>::mid_bytes(); comb = SlabSmem<T, 32, 32>::combine_bytes(); return;
        case 48: mid = SlabSmem<T, 48, 48>::mid_bytes(); comb = SlabSmem<T, 48, 48>::combine_bytes(); return;
        case 64: mid = SlabSmem<T, 64, 64>::mid_bytes(); comb = SlabSmem<T, 64, 64>::combine_bytes(); return;
        case 96: mid = SlabSmem<T, 96, 96>::mid_bytes(); comb = SlabSmem<T, 96, 96>::combine_bytes(); return;
        case 128: mid = SlabSmem<T, 128, 128>::mid_bytes(); comb = SlabSmem<T, 128, 128>::combine_bytes(); return;
        case 6496: mid = SlabSmem<T, 64, 96>::mid_bytes(); comb = SlabSmem<T, 64, 96>::combine_bytes(); return;
        default: mid = comb = 0;
    }
}

void pf_smem_bytes(int id, int fp32, int &mid, int &comb)
{
    if (fp32)
        pf_smem<float>(id, mid, comb);
    else
        pf_smem<double>(id, mid, comb);
}

int pencil_sh_smem_bytes(int fp32, int tc, int m0)
{
    return fp32 ? PencilSh<float>::smem(tc, m0) : PencilSh<double>::smem(tc, m0);
}

// op 0: props, 1: single step, 2: shared-memory attributes, 3: chain segment, 4: CTAs of the
// persistent step kernel
template <typename T, int MT, int F0, int F1, int F2>
int run_op(int op, const PropsArgs<T> *a, const PropsLaunch &L, int n, cudaStream_t st)
{
    if (op == 0) return launch_props_mt<T, MT, F0, F1, F2>(*a, L, n, st);
    if (op == 1) return launch_single_step_mt<T, MT, F0, F1, F2>(*a, L, n, st);
    if (op == 4) {
        // CTAs of the persistent step kernel: the occupancy of its larger (wide) form times the SMs
        if constexpr (F1 != 0) {
            constexpr int TC = kTile<T>::value;
            int dev = 0, sms = 148, per_sm = 0;
            if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaError_t e = L.tmap_wide
                                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_pf<T, MT, F0, F1, F2, 2 * TC>,
                                                                                MT, L.step_pf_smem)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_pf<T, MT, F0, F1, F2, TC>, MT,
                                                                                L.step_pf_smem);
            return (e == cudaSuccess && per_sm > 0) ? sms * per_sm : 0;
        }
        return 0;
    }
    if (op == 3) return launch_chain_mt<T, MT, F0, F1, F2>(*a, L, n, st);
    return set_smem_mt<T, MT, F0, F1, F2>(L);
}

template <typename T>
int dispatch(int op, const PropsArgs<T> *a, const PropsLaunch &L, int n, cudaStream_t st)
{
    switch (L.fixed) {
        case 32: return run_op<T, 256, 32, 32, 32>(op, a, L, n, st);
        case 48: return run_op<T, 256, 48, 48, 48>(op, a, L, n, st);
        case 64: return run_op<T, 256, 64, 64, 64>(op, a, L, n, st);
        case 96: return run_op<T, 256, 96, 96, 96>(op, a, L, n, st);
        case 128: return run_op<T, 512, 128, 128, 128>(op, a, L, n, st);
        case 6496: return run_op<T, 256, 64, 64, 96>(op, a, L, n, st);
        default: break;
    }
    return L.big ? run_op<T, 1024, 0, 0, 0>(op, a, L, n, st) : run_op<T, 256, 0, 0, 0>(op, a, L, n, st);
}

// compile-time shape id for a grid (0: runtime-shaped kernels)
int fixed_shape_id(int m0, int m1, int m2)
{
    if (m0 == m1 && m1 == m2 && (m0 == 32 || m0 == 48 || m0 == 64 || m0 == 96 || m0 == 128)) return m0;
    if (m0 == 64 && m1 == 64 && m2 == 96) return 6496;
    return 0;
}

int fixed_shape_threads(int id) { return id == 128 ? 512 : 256; }

template <typename T>
int launch_props(const PropsArgs<T> &a, const PropsLaunch &L, int nslots, cudaStream_t st)
{
    return dispatch<T>(0, &a, L, nslots, st);
}

template <typename T>
int launch_single_step(const PropsArgs<T> &a, const PropsLaunch &L, int s, cudaStream_t st)
{
    return dispatch<T>(1, &a, L, s, st);
}

template <typename T>
int props_step_grid(const PropsLaunch &L)
{
    return dispatch<T>(4, nullptr, L, 0, nullptr);
}
template int props_step_grid<float>(const PropsLaunch &);
template int props_step_grid<double>(const PropsLaunch &);

template <typename T>
int set_props_smem(const PropsLaunch &L)
{
    return dispatch<T>(2, nullptr, L, 0, nullptr);
}

template <typename T>
int launch_chain(const PropsArgs<T> &a, const PropsLaunch &L, int first_mode, cudaStream_t st)
{
    return dispatch<T>(3, &a, L, first_mode, st);
}

template <typename T>
int launch_prepare(const PropsArgs<T> &a, const PropsLaunch &L, cudaStream_t st)
{
    k_prepare<T><<<dim3(L.ew_blocks, 1), 256, 0, st>>>(a);
    return 1;
}

template <typename T>
int launch_qsums(const PropsArgs<T> &a, const PropsLaunch &L, cudaStream_t st)
{
    k_qsum<T><<<dim3(L.red_blocks, 1), 256, 0, st>>>(a);
    k_qfinal<T><<<1, 32, 0, st>>>(a, L.red_blocks);
    return 2;
}

template int launch_props<float>(const PropsArgs<float> &, const PropsLaunch &, int, cudaStream_t);
template int launch_props<double>(const PropsArgs<double> &, const PropsLaunch &, int, cudaStream_t);
template int launch_single_step<float>(const PropsArgs<float> &, const PropsLaunch &, int, cudaStream_t);
template int launch_single_step<double>(const PropsArgs<double> &, const PropsLaunch &, int, cudaStream_t);
template int set_props_smem<float>(const PropsLaunch &);
template int set_props_smem<double>(const PropsLaunch &);
template int launch_chain<float>(const PropsArgs<float> &, const PropsLaunch &, int, cudaStream_t);
template int launch_chain<double>(const PropsArgs<double> &, const PropsLaunch &, int, cudaStream_t);
template int launch_prepare<float>(const PropsArgs<float> &, const PropsLaunch &, cudaStream_t);
template int launch_prepare<double>(const PropsArgs<double> &, const PropsLaunch &, cudaStream_t);
template int launch_qsums<float>(const PropsArgs<float> &, const PropsLaunch &, cudaStream_t);
template int launch_qsums<double>(const PropsArgs<double> &, const PropsLaunch &, cudaStream_t);

}  // namespace scft
