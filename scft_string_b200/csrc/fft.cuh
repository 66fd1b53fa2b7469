// fft.cuh -- CTA-wide mixed-radix FFTs on shared memory for sm_100a.
//
// This replaces the cuFFT D2Z/Z2D plans of the reference (density.h:67-74,
// 149-205).  A 3-D real transform of one field is split into
//   * an x-slab pass (one CTA per x index): the real m1 x m2 slab is packed as
//     ceil(m1/2) complex rows (y-line pairs), z-transformed, unpacked into the
//     m1 x (m2/2+1) half spectrum and y-transformed -- all in shared memory;
//   * an x-pencil pass (one CTA per tile of consecutive (ky, kz) columns) that
//     transforms along x, applies the diffusion factor and transforms back.
// The inverse runs the slab pass backwards.
//
// Each 1-D FFT is a Stockham autosort transform: stage (radix R, accumulated
// size Ns) reads element j + r*n/R of a line, multiplies by
// exp(sign*2*pi*i*r*(j%Ns)/(Ns*R)), does an R-point DFT in registers and
// writes element (j/Ns)*Ns*R + j%Ns + r*Ns.  Stages run in place: every thread
// stages its butterflies in registers across one __syncthreads.
// Twiddles come from a table exp(-2*pi*i*t/n) computed on the host in FP64.
#pragma once
#include "common.cuh"

namespace scft {

// multiply by sign*i
template <typename T>
__device__ __forceinline__ cplx<T> mul_si(cplx<T> a, int sign)
{
    return sign > 0 ? cplx<T>{-a.y, a.x} : cplx<T>{a.y, -a.x};
}

// R-point DFTs in registers: V[q] = sum_r v[r] exp(sign*2*pi*i*r*q/R).
template <typename T, int R>
struct Dft;

template <typename T>
struct Dft<T, 2> {
    static __device__ __forceinline__ void run(cplx<T> *v, int, const cplx<T> *, int)
    {
        cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <typename T>
struct Dft<T, 4> {
    static __device__ __forceinline__ void run(cplx<T> *v, int sign, const cplx<T> *, int)
    {
        cplx<T> a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        cplx<T> c = cadd(v[1], v[3]), d = mul_si(csub(v[1], v[3]), sign);
        v[0] = cadd(a, c);
        v[1] = cadd(b, d);
        v[2] = csub(a, c);
        v[3] = csub(b, d);
    }
};

template <typename T>
struct Dft<T, 8> {
    static __device__ __forceinline__ void run(cplx<T> *v, int sign, const cplx<T> *, int)
    {
        const T c = (T)0.70710678118654752440;  // sqrt(1/2)
        const T s = (T)sign;
        cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
        cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
        Dft<T, 4>::run(e, sign, nullptr, 0);
        Dft<T, 4>::run(o, sign, nullptr, 0);
        // o[k] *= exp(sign*2*pi*i*k/8)
        cplx<T> o1 = {c * (o[1].x - s * o[1].y), c * (o[1].y + s * o[1].x)};
        cplx<T> o2 = mul_si(o[2], sign);
        cplx<T> o3 = {c * (-o[3].x - s * o[3].y), c * (-o[3].y + s * o[3].x)};
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

template <typename T>
struct Dft<T, 3> {
    static __device__ __forceinline__ void run(cplx<T> *v, int sign, const cplx<T> *, int)
    {
        const T h = (T)0.86602540378443864676;  // sqrt(3)/2
        cplx<T> t1 = cadd(v[1], v[2]);
        cplx<T> m = {v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y};
        cplx<T> d = mul_si(csub(v[1], v[2]), sign);
        d.x *= h;
        d.y *= h;
        v[0] = cadd(v[0], t1);
        v[1] = cadd(m, d);
        v[2] = csub(m, d);
    }
};

template <typename T>
struct Dft<T, 5> {
    static __device__ __forceinline__ void run(cplx<T> *v, int sign, const cplx<T> *, int)
    {
        const T c1 = (T)0.30901699437494742410;   // cos(2 pi/5) = (sqrt5 - 1)/4
        const T c2 = (T)-0.80901699437494742410;  // cos(4 pi/5) = -(sqrt5 + 1)/4
        const T s1 = (T)0.95105651629515357212;   // sin(2 pi/5)
        const T s2 = (T)0.58778525229247312917;   // sin(4 pi/5)
        cplx<T> a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
        cplx<T> b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
        cplx<T> r1 = {v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y};
        cplx<T> r2 = {v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y};
        cplx<T> i1 = mul_si(cplx<T>{s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y}, sign);
        cplx<T> i2 = mul_si(cplx<T>{s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y}, sign);
        v[0] = {v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y};
        v[1] = cadd(r1, i1);
        v[4] = csub(r1, i1);
        v[2] = cadd(r2, i2);
        v[3] = csub(r2, i2);
    }
};

// direct DFT for radix 7 with roots taken from the length-n table
template <typename T>
struct Dft<T, 7> {
    static __device__ __forceinline__ void run(cplx<T> *v, int sign, const cplx<T> *tw, int n)
    {
        const int step = n / 7;
        cplx<T> out[7];
#pragma unroll
        for (int q = 0; q < 7; q++) {
            cplx<T> acc = v[0];
#pragma unroll
            for (int r = 1; r < 7; r++) {
                cplx<T> w = tw[((r * q) % 7) * step];
                acc = cadd(acc, sign < 0 ? cmul(v[r], w) : cmulc(v[r], w));
            }
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < 7; q++) v[q] = out[q];
    }
};

// Elements a thread stages in registers per stage (complex values).
constexpr int kStageBudget = 16;

template <int R>
struct Slots {
    static constexpr int value = kStageBudget / R;
};

// One Stockham stage over `nlines` lines of length n.  Element i of line l is
// buf[l*ls + i*es].  line_fast selects the butterfly->thread order: consecutive
// threads walk lines (good when ls == 1) or butterflies (good when es == 1).
template <typename T, int R>
__device__ __noinline__ void fft_stage(cplx<T> *__restrict__ buf, int n, int nlines, int es,
                                     int ls, bool line_fast, int Ns,
                                     const cplx<T> *__restrict__ tw, int sign, int *err)
{
    constexpr int SL = Slots<R>::value;
    const int nR = n / R;
    const int nb = nlines * nR;
    const int tstep = n / (Ns * R);
    const int nthr = blockDim.x;
    cplx<T> v[SL][R];
#pragma unroll
    for (int sl = 0; sl < SL; sl++) {
        const int b = threadIdx.x + sl * nthr;
        if (b < nb) {
            int line, j;
            if (line_fast) {
                line = b % nlines;
                j = b / nlines;
            } else {
                j = b % nR;
                line = b / nR;
            }
            const int k = j % Ns;
            const cplx<T> *src = buf + line * ls + j * es;
#pragma unroll
            for (int r = 0; r < R; r++) {
                cplx<T> a = src[r * nR * es];
                if (r > 0 && k > 0) {
                    const cplx<T> w = tw[r * k * tstep];
                    a = sign < 0 ? cmul(a, w) : cmulc(a, w);
                }
                v[sl][r] = a;
            }
            Dft<T, R>::run(v[sl], sign, tw, n);
        }
    }
    if (threadIdx.x + SL * nthr < nb) *err = 1;  // launch geometry too small: host bug
    __syncthreads();
#pragma unroll
    for (int sl = 0; sl < SL; sl++) {
        const int b = threadIdx.x + sl * nthr;
        if (b < nb) {
            int line, j;
            if (line_fast) {
                line = b % nlines;
                j = b / nlines;
            } else {
                j = b % nR;
                line = b / nR;
            }
            const int k = j % Ns;
            cplx<T> *dst = buf + line * ls + ((j - k) * R + k) * es;
#pragma unroll
            for (int r = 0; r < R; r++) dst[r * Ns * es] = v[sl][r];
        }
    }
    __syncthreads();
}

template <typename T>
__device__ void cta_fft(cplx<T> *buf, const Plan1D &p, int nlines, int es, int ls, bool line_fast,
                        const cplx<T> *tw, int sign, int *err)
{
    int Ns = 1;
    for (int st = 0; st < p.nst; st++) {
        const int R = p.radix[st];
        switch (R) {
            case 8: fft_stage<T, 8>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            case 4: fft_stage<T, 4>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            case 2: fft_stage<T, 2>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            case 3: fft_stage<T, 3>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            case 5: fft_stage<T, 5>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            case 7: fft_stage<T, 7>(buf, p.n, nlines, es, ls, line_fast, Ns, tw, sign, err); break;
            default: *err = 2; return;
        }
        Ns *= R;
    }
}

// After the forward z-transform of packed rows C = FFT(a[2p] + i a[2p+1]):
// A[k] = (C[k] + conj C[-k])/2 and B[k] = (C[k] - conj C[-k])/(2i) are the half
// spectra of the two real lines; they go to rows 2p and 2p+1 of the slab.
// One warp per pair; reads and writes stay inside the pair's own rows.
template <typename T>
__device__ void slab_unpack(cplx<T> *buf, const Geo &g)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int m2 = g.m2, mk2 = g.mk2;
    for (int p = warp; p < g.npair; p += nw) {
        cplx<T> *row = buf + 2 * p * mk2;
        const bool has_b = (2 * p + 1 < g.m1);
        cplx<T> A[kPairLanes], B[kPairLanes];
#pragma unroll
        for (int t = 0; t < kPairLanes; t++) {
            const int kz = lane + 32 * t;
            if (kz < mk2) {
                const cplx<T> ck = row[kz];
                const cplx<T> cm = row[kz == 0 ? 0 : m2 - kz];
                A[t] = {(ck.x + cm.x) * (T)0.5, (ck.y - cm.y) * (T)0.5};
                B[t] = {(ck.y + cm.y) * (T)0.5, (cm.x - ck.x) * (T)0.5};
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kPairLanes; t++) {
            const int kz = lane + 32 * t;
            if (kz < mk2) {
                row[kz] = A[t];
                if (has_b) row[mk2 + kz] = B[t];
            }
        }
        __syncwarp();
    }
}

// Inverse of slab_unpack with half-complex-to-real semantics: the imaginary
// parts of the self-conjugate bins (kz = 0 and kz = m2/2) are dropped, and
// C[k] = A[k] + i B[k], C[-k] = conj A[k] + i conj B[k].
template <typename T>
__device__ void slab_pack(cplx<T> *buf, const Geo &g)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int m2 = g.m2, mk2 = g.mk2;
    for (int p = warp; p < g.npair; p += nw) {
        cplx<T> *row = buf + 2 * p * mk2;
        const bool has_b = (2 * p + 1 < g.m1);
        cplx<T> A[kPairLanes], B[kPairLanes];
#pragma unroll
        for (int t = 0; t < kPairLanes; t++) {
            const int kz = lane + 32 * t;
            if (kz < mk2) {
                A[t] = row[kz];
                B[t] = has_b ? row[mk2 + kz] : cplx<T>{(T)0, (T)0};
                if (kz == 0 || 2 * kz == m2) {
                    A[t].y = (T)0;
                    B[t].y = (T)0;
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kPairLanes; t++) {
            const int kz = lane + 32 * t;
            if (kz < mk2) {
                row[kz] = {A[t].x - B[t].y, A[t].y + B[t].x};
                if (kz > 0 && 2 * kz < m2) row[m2 - kz] = {A[t].x + B[t].y, B[t].x - A[t].y};
            }
        }
        __syncwarp();
    }
}

// packed real rows -> half spectrum [y][kz]
template <typename T>
__device__ void slab_forward(cplx<T> *buf, const Geo &g, const cplx<T> *twy, const cplx<T> *twz,
                             int *err)
{
    cta_fft(buf, g.pz, g.npair, 1, 2 * g.mk2, false, twz, -1, err);
    slab_unpack(buf, g);
    __syncthreads();
    cta_fft(buf, g.py, g.mk2, g.mk2, 1, true, twy, -1, err);
}

// half spectrum [y][kz] -> packed real rows (unnormalised)
template <typename T>
__device__ void slab_inverse(cplx<T> *buf, const Geo &g, const cplx<T> *twy, const cplx<T> *twz,
                             int *err)
{
    cta_fft(buf, g.py, g.mk2, g.mk2, 1, true, twy, +1, err);
    slab_pack(buf, g);
    __syncthreads();
    cta_fft(buf, g.pz, g.npair, 1, 2 * g.mk2, false, twz, +1, err);
}

}  // namespace scft

// ===================================================================== fixed shapes
// The same Stockham transforms with every length, line count, stride and
// thread count known at compile time: index arithmetic folds to shifts and
// multiplies and each thread's butterflies are fully unrolled.  Used for the
// grid sizes the host has instantiations for; other sizes take the runtime
// path above.
namespace scft {

__host__ __device__ constexpr int pick_radix(int rem)
{
    return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5 : 7;
}

template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, int R, int NS>
__device__ __forceinline__ void fft_stage_fixed(cplx<T> *__restrict__ buf, const cplx<T> *__restrict__ tw,
                                                int sign)
{
    constexpr int NR = N / R;
    constexpr int NB = NLINES * NR;
    constexpr int PER = (NB + NT - 1) / NT;
    constexpr int TSTEP = N / (NS * R);
    cplx<T> v[PER][R];
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
            const int k = j % NS;
            const cplx<T> *src = buf + line * LS + j * ES;
#pragma unroll
            for (int r = 0; r < R; r++) {
                cplx<T> a = src[r * NR * ES];
                if (NS > 1 && r > 0) {
                    const cplx<T> w = tw[r * k * TSTEP];
                    a = sign < 0 ? cmul(a, w) : cmulc(a, w);
                }
                v[i][r] = a;
            }
            Dft<T, R>::run(v[i], sign, tw, N);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
            const int k = j % NS;
            cplx<T> *dst = buf + line * LS + ((j - k) * R + k) * ES;
#pragma unroll
            for (int r = 0; r < R; r++) dst[r * NS * ES] = v[i][r];
        }
    }
    __syncthreads();
}

template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, int NS = 1>
__device__ __forceinline__ void fft_fixed(cplx<T> *buf, const cplx<T> *tw, int sign)
{
    if constexpr (NS < N) {
        constexpr int R = pick_radix(N / NS);
        fft_stage_fixed<T, N, NLINES, ES, LS, LF, NT, R, NS>(buf, tw, sign);
        fft_fixed<T, N, NLINES, ES, LS, LF, NT, NS * R>(buf, tw, sign);
    }
}

// Radix schedule of the fixed transforms: greedy 8, 4, 2, 3, 5, 7.
template <int N>
struct RadixPlan {
    __host__ __device__ static constexpr int stages()
    {
        int s = 0, ns = 1;
        while (ns < N) {
            ns *= pick_radix(N / ns);
            s++;
        }
        return s;
    }
    __host__ __device__ static constexpr int radix(int i)
    {
        int ns = 1;
        for (int k = 0; k < i; k++) ns *= pick_radix(N / ns);
        return pick_radix(N / ns);
    }
    __host__ __device__ static constexpr int rradix(int i) { return radix(stages() - 1 - i); }  // reversed schedule
};

template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, int SIGN, int I, int NS>
__device__ __forceinline__ void stages_but_last(cplx<T> *buf, const cplx<T> *tw)
{
    if constexpr (I < RadixPlan<N>::stages() - 1) {
        constexpr int R = RadixPlan<N>::radix(I);
        fft_stage_fixed<T, N, NLINES, ES, LS, LF, NT, R, NS>(buf, tw, SIGN);
        stages_but_last<T, N, NLINES, ES, LS, LF, NT, SIGN, I + 1, NS * R>(buf, tw);
    }
}

template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, int SIGN, int I, int NS>
__device__ __forceinline__ void stages_reversed(cplx<T> *buf, const cplx<T> *tw)
{
    if constexpr (I < RadixPlan<N>::stages()) {
        constexpr int R = RadixPlan<N>::rradix(I);
        fft_stage_fixed<T, N, NLINES, ES, LS, LF, NT, R, NS>(buf, tw, SIGN);
        stages_reversed<T, N, NLINES, ES, LS, LF, NT, SIGN, I + 1, NS * R>(buf, tw);
    }
}

// Transform (sign SIGN), pointwise multiply, transform back (sign -SIGN) of
// NLINES lines in place.  Butterfly j of the first transform's last stage
// (radix R) holds the outputs j + r N/R, which are exactly the inputs of
// butterfly j of the first stage of a transform that runs the radices in
// reverse order; so those two stages and the multiply run in registers with
// one shared-memory round trip instead of three.  mul(v, line, k) scales
// element k of line `line`.
template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, int SIGN, class Mul>
__device__ __forceinline__ void fft_pair_fused(cplx<T> *__restrict__ buf, const cplx<T> *__restrict__ tw, Mul mul)
{
    stages_but_last<T, N, NLINES, ES, LS, LF, NT, SIGN, 0, 1>(buf, tw);
    constexpr int R = RadixPlan<N>::radix(RadixPlan<N>::stages() - 1);
    constexpr int NR = N / R;  // also the stride NS of the first transform's last stage
    constexpr int NB = NLINES * NR;
    constexpr int PER = (NB + NT - 1) / NT;
    cplx<T> v[PER][R];
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
            const cplx<T> *src = buf + line * LS + j * ES;
#pragma unroll
            for (int r = 0; r < R; r++) {
                cplx<T> a = src[r * NR * ES];
                if (NR > 1 && r > 0) a = SIGN < 0 ? cmul(a, tw[r * j]) : cmulc(a, tw[r * j]);
                v[i][r] = a;
            }
            Dft<T, R>::run(v[i], SIGN, tw, N);
#pragma unroll
            for (int r = 0; r < R; r++) mul(v[i][r], line, j + r * NR);
            Dft<T, R>::run(v[i], -SIGN, tw, N);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
            cplx<T> *dst = buf + line * LS + j * R * ES;
#pragma unroll
            for (int r = 0; r < R; r++) dst[r * ES] = v[i][r];
        }
    }
    __syncthreads();
    stages_reversed<T, N, NLINES, ES, LS, LF, NT, -SIGN, 1, RadixPlan<N>::rradix(0)>(buf, tw);
}

// forward transform, multiply, inverse transform
template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, class Mul>
__device__ __forceinline__ void fft_fwd_mul_inv(cplx<T> *buf, const cplx<T> *tw, Mul mul)
{
    fft_pair_fused<T, N, NLINES, ES, LS, LF, NT, -1>(buf, tw, mul);
}

// Packed z-rows of the fixed shapes sit at an odd stride of M2 + 1 complex
// elements, so that a warp transforming 32 rows at once (lines fastest) reads
// and writes 32 different banks; the half spectra [y][kz] keep their natural
// stride MK2.  The two layouts overlap in the same buffer: the unpack happens
// inside the loads of the first y stage of the forward transform, whose
// barrier separates all reads from all writes; the pack before the inverse z
// pass is a pass of its own (slab_pack_fixed).
template <int M2>
struct PackedRows {
    static constexpr int LSF = M2 + 1;
};

// First Stockham stage (NS = 1, no twiddles) whose inputs come from a
// functor: ld(line, k) returns element k of line `line`.  The outputs go to
// buf in the stage's usual layout after a barrier, so the functor may read
// any part of buf (a different layout of the same data) in place.
template <typename T, int N, int NLINES, int ES, int LS, bool LF, int NT, class Load>
__device__ __forceinline__ void fft_first_stage_ld(cplx<T> *__restrict__ buf, const cplx<T> *__restrict__ tw,
                                                   int sign, Load ld)
{
    constexpr int R = pick_radix(N);
    constexpr int NR = N / R, NB = NLINES * NR, PER = (NB + NT - 1) / NT;
    cplx<T> v[PER][R];
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = ld(line, j + r * NR);
            Dft<T, R>::run(v[i], sign, tw, N);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int b = threadIdx.x + i * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = LF ? b % NLINES : b / NR;
            const int j = LF ? b / NLINES : b % NR;
            cplx<T> *dst = buf + line * LS + j * R * ES;
#pragma unroll
            for (int r = 0; r < R; r++) dst[r * ES] = v[i][r];
        }
    }
    __syncthreads();
}

// The kz = 0 and kz = M2/2 columns of a slab's half spectrum are real
// sequences along y before the forward y pass and Hermitian ones before the
// inverse y pass, so the two travel as one complex column c0 + i cH in column
// 0: the y passes then cover M2/2 columns (M2/2 x M1/R butterflies per stage,
// e.g. exactly 256 at 64^3) instead of M2/2 + 1.  slab_ysplit_fixed recovers
// the two spectra after the forward pass: X0(k) = (C(k) + conj C(-k))/2,
// XH(k) = (C(k) - conj C(-k))/(2i).
// column 0 after the forward y pass holds C = FFT_y(c0 + i cH): split it
template <typename T, int M1, int M2, int NT>
__device__ __forceinline__ void slab_ysplit_fixed(cplx<T> *buf)
{
    constexpr int MK2 = M2 / 2 + 1, H = M2 / 2;
    cplx<T> X0, XH;
    const int k = threadIdx.x;
    static_assert(M1 <= NT, "one thread per ky");
    if (k < M1) {
        const cplx<T> c = buf[k * MK2], cm = buf[((M1 - k) % M1) * MK2];
        X0 = {(c.x + cm.x) * (T)0.5, (c.y - cm.y) * (T)0.5};
        XH = {(c.y + cm.y) * (T)0.5, (cm.x - c.x) * (T)0.5};
    }
    __syncthreads();
    if (k < M1) {
        buf[k * MK2] = X0;
        buf[k * MK2 + H] = XH;
    }
    __syncthreads();
}

// column 0 before the inverse y pass: S(ky, 0) + i S(ky, H)
template <typename T, int M1, int M2, int NT>
__device__ __forceinline__ void slab_yjoin_fixed(cplx<T> *buf)
{
    constexpr int MK2 = M2 / 2 + 1, H = M2 / 2;
    static_assert(M1 <= NT, "one thread per ky");
    const int k = threadIdx.x;
    if (k < M1) {
        const cplx<T> c0 = buf[k * MK2], ch = buf[k * MK2 + H];
        buf[k * MK2] = {c0.x - ch.y, c0.y + ch.x};
    }
    __syncthreads();
}

// Half spectra [y][kz] -> packed z-rows (the inverse of the unpack in
// slab_forward_fixed, with half-complex-to-real semantics: the imaginary
// parts of the self-conjugate bins are dropped); column 0 holds the kz = 0
// values in .x and the kz = M2/2 values in .y.  Reads all items into
// registers, then writes, with a barrier in between (the layouts overlap).
template <typename T, int M1, int M2, int NT>
__device__ __forceinline__ void slab_pack_fixed(cplx<T> *buf)
{
    constexpr int MK2 = M2 / 2 + 1, H = M2 / 2, NPAIR = (M1 + 1) / 2, LS = PackedRows<M2>::LSF;
    constexpr int ITEMS = NPAIR * MK2, PER = (ITEMS + NT - 1) / NT;
    cplx<T> A[PER], B[PER];
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int e = threadIdx.x + i * NT;
        if (ITEMS % NT == 0 || e < ITEMS) {
            const int p = e / MK2, kz = e - p * MK2;
            const bool hb = 2 * p + 1 < M1;
            if (kz == 0 || kz == H) {
                const cplx<T> a = buf[2 * p * MK2];
                const cplx<T> b = hb ? buf[(2 * p + 1) * MK2] : cplx<T>{(T)0, (T)0};
                A[i] = {kz == 0 ? a.x : a.y, (T)0};
                B[i] = {kz == 0 ? b.x : b.y, (T)0};
            } else {
                A[i] = buf[2 * p * MK2 + kz];
                B[i] = hb ? buf[(2 * p + 1) * MK2 + kz] : cplx<T>{(T)0, (T)0};
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int e = threadIdx.x + i * NT;
        if (ITEMS % NT == 0 || e < ITEMS) {
            const int p = e / MK2, kz = e - p * MK2;
            buf[p * LS + kz] = {A[i].x - B[i].y, A[i].y + B[i].x};
            if (kz > 0 && 2 * kz < M2) buf[p * LS + M2 - kz] = {A[i].x + B[i].y, B[i].x - A[i].y};
        }
    }
    __syncthreads();
}


// ===================================================================== warp-shuffle 64-point lines
// A 64-point line held by an octet of lanes (lane bits 0-2 = sub-lane s):
// lane s holds x[s + 8 j], j = 0..7.  With n = s + 8 n2 and k = k1 + 8 k2,
//   X[k1 + 8 k2] = sum_s w8^(s k2) [w64^(s k1) sum_n2 x[s + 8 n2] w8^(n2 k1)],
// so each lane runs an 8-point DFT, multiplies by w64^(s k1), the octet
// transposes its 8 x 8 block (lane k1 receives element k1 of every lane), and
// each lane runs a second 8-point DFT: lane k1 then holds X[k1 + 8 k2] in
// slot k2.  The inverse has the same shape, so a transform, a pointwise
// multiply and the inverse transform end with lane s holding x'[s + 8 j]
// again: no shared-memory round trip and no CTA barrier inside.

// 8 x 8 transpose across the lanes of an octet by three xor exchanges: at
// mask m, the lane without bit m swaps its element j|m with element j of the
// lane with bit m (for every j without bit m).  Afterwards lane i holds, in
// slot j, what lane j held in slot i.
template <typename T>
__device__ __forceinline__ void octet_transpose(cplx<T> (&a)[8], int s)
{
#pragma unroll
    for (int m = 1; m < 8; m <<= 1) {
        const bool up = (s & m) != 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j & m) continue;
            const cplx<T> send = up ? a[j] : a[j | m];
            cplx<T> r;
            r.x = __shfl_xor_sync(0xffffffffu, send.x, m);
            r.y = __shfl_xor_sync(0xffffffffu, send.y, m);
            if (up)
                a[j] = r;
            else
                a[j | m] = r;
        }
    }
}

// w[k] = exp(-2 pi i s k / 64), k = 1..7 (w[0] unused), from the length-64
// table tw[t] = exp(-2 pi i t / 64)
template <typename T>
__device__ __forceinline__ void octet_twiddles(cplx<T> (&w)[8], const cplx<T> *__restrict__ tw, int s)
{
    w[0] = {(T)1, (T)0};
#pragma unroll
    for (int k = 1; k < 8; k++) w[k] = tw[s * k];
}

// forward 64-point transform of the octet's line (sign -1): in, lane s slot j
// = x[s + 8 j]; out, lane s slot j = X[s + 8 j]
template <typename T>
__device__ __forceinline__ void octet_fft64_fwd(cplx<T> (&v)[8], const cplx<T> (&w)[8], int s)
{
    Dft<T, 8>::run(v, -1, nullptr, 0);
#pragma unroll
    for (int k = 1; k < 8; k++) v[k] = cmul(v[k], w[k]);
    octet_transpose(v, s);
    Dft<T, 8>::run(v, -1, nullptr, 0);
}

// inverse (sign +1, unnormalised) of the same layout: in, lane s slot j =
// X[s + 8 j]; out, lane s slot j = x[s + 8 j]
template <typename T>
__device__ __forceinline__ void octet_fft64_inv(cplx<T> (&v)[8], const cplx<T> (&w)[8], int s)
{
    Dft<T, 8>::run(v, +1, nullptr, 0);
#pragma unroll
    for (int k = 1; k < 8; k++) v[k] = cmulc(v[k], w[k]);
    octet_transpose(v, s);
    Dft<T, 8>::run(v, +1, nullptr, 0);
}


// packed real rows (stride M2 + 1) -> half spectrum [y][kz]
template <typename T, int M1, int M2, int NT>
__device__ __forceinline__ void slab_forward_fixed(cplx<T> *buf, const cplx<T> *twy, const cplx<T> *twz)
{
    constexpr int MK2 = M2 / 2 + 1, NPAIR = (M1 + 1) / 2;
    constexpr int H = M2 / 2, LSP = PackedRows<M2>::LSF;
    fft_fixed<T, M2, NPAIR, 1, LSP, true, NT>(buf, twz, -1);
    // first y stage reads the packed z spectra directly, unpacking per
    // element: row y = 2p (A) or 2p+1 (B) of column kz
    fft_first_stage_ld<T, M1, H, MK2, 1, true, NT>(buf, twy, -1, [&](int kz, int y) -> cplx<T> {
        const cplx<T> *row = buf + (y >> 1) * LSP;
        const bool odd = y & 1;
        if (kz == 0) {
            const cplx<T> c0 = row[0], ch = row[H];
            return odd ? cplx<T>{c0.y, ch.y} : cplx<T>{c0.x, ch.x};
        }
        const cplx<T> ck = row[kz], cm = row[M2 - kz];
        return odd ? cplx<T>{(ck.y + cm.y) * (T)0.5, (cm.x - ck.x) * (T)0.5}
                   : cplx<T>{(ck.x + cm.x) * (T)0.5, (ck.y - cm.y) * (T)0.5};
    });
    fft_fixed<T, M1, H, MK2, 1, true, NT, pick_radix(M1)>(buf, twy, -1);
    slab_ysplit_fixed<T, M1, M2, NT>(buf);
}

// half spectrum [y][kz] -> packed real rows (stride M2 + 1, unnormalised)
template <typename T, int M1, int M2, int NT>
__device__ __forceinline__ void slab_inverse_fixed(cplx<T> *buf, const cplx<T> *twy, const cplx<T> *twz)
{
    constexpr int MK2 = M2 / 2 + 1, NPAIR = (M1 + 1) / 2;
    __syncthreads();
    slab_yjoin_fixed<T, M1, M2, NT>(buf);
    constexpr int H = M2 / 2, LSP = PackedRows<M2>::LSF;
    fft_fixed<T, M1, H, MK2, 1, true, NT>(buf, twy, +1);
    // the pack runs as its own pass: read inside the first z stage (lanes
    // across packed rows) the half spectra would be 2-way bank conflicts
    slab_pack_fixed<T, M1, M2, NT>(buf);
    fft_fixed<T, M2, NPAIR, 1, LSP, true, NT>(buf, twz, +1);
}

}  // namespace scft

