// reg64.cuh -- register-resident transforms of the 64^3 FP32 contour step.
//
// A 64-point complex FFT lives entirely in one thread's registers: two
// radix-8 passes with the 64th-root twiddles between them (64 = 8 x 8).
// Writing n = j + 8r and k = q + 8s,
//   X[q + 8s] = sum_j w64^{jq} w8^{js} sum_r x[j + 8r] w8^{rq},
// so pass 1 runs eight 8-point DFTs over r (stride 8), the twiddles scale
// element (j, q), and pass 2 runs eight 8-point DFTs over j.  The result is
// left in the transposed order X[k] -> v[perm(k)], perm(k) = (k >> 3) +
// 8 (k & 7): every index is a compile-time constant after unrolling, so the
// permutation costs nothing (it renames registers).
//
// A 64 x 64 real slab (rows y, columns z) is transformed by one warp:
//   z pass: lane p holds rows p and p+32 packed as one complex line
//           a_p + i a_{p+32}; its FFT gives both rows' half spectra
//           (two-for-one: A = (C(k) + conj C(-k))/2, B = (C(k) - conj C(-k))/2i)
//   y pass: lane kz holds column kz (64 values along y) of the half spectrum;
//           the kz = 0 and kz = 32 columns are real along y before the forward
//           pass (Hermitian before the inverse one) and travel together in
//           lane 0 as one complex column c0 + i c32.
// Between the two passes the data crosses once through a per-warp
// shared-memory tile; the only synchronisation is __syncwarp.
//
// The helpers are __host__ __device__ so that the same code is checked on the
// CPU against numpy (tests/test_reg64_host.py drives a host build of it).
#pragma once
#include <cuda_runtime.h>

#ifndef SCFT_HD
#define SCFT_HD __host__ __device__ __forceinline__
#endif

namespace scft {
namespace reg64 {

constexpr int kN = 64;
constexpr int kMK = 33;                 // half-spectrum length along z
constexpr int kRowPitch = 68;           // floats per real row in the slab tile (bank-conflict free float4)
constexpr int kColPitch = 65;           // complex per spectrum column in the slab tile
constexpr int kTileFloats = 64 * kRowPitch;  // 17408 bytes; the complex view needs 33*65*2 = 4290 floats
static_assert(33 * kColPitch * 2 <= kTileFloats, "the complex view of the tile fits the real view");
constexpr int kPlane = 64 * kMK;        // complex elements of one x-plane of the half spectrum (2112)

// exp(2 pi i t / 64) from a Taylor series of the reduced angle (|phi| <= pi/4)
struct Tw {
    float c, s;  // cos(2 pi t/64), sin(2 pi t/64)
};
constexpr double taylor_sin(double x)
{
    double term = x, sum = x;
    for (int n = 1; n < 14; n++) {
        term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double taylor_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int n = 1; n < 14; n++) {
        term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}
constexpr Tw make_tw(int t)
{
    // t = 16 k + u, u in [-8, 8]: angle = k pi/2 + 2 pi u/64
    t &= 63;
    int k = (t + 8) / 16;
    int u = t - 16 * k;
    const double phi = 2.0 * 3.14159265358979323846264338327950288 * u / 64.0;
    const double c = taylor_cos(phi), s = taylor_sin(phi);
    k &= 3;
    if (k == 0) return {(float)c, (float)s};
    if (k == 1) return {(float)-s, (float)c};
    if (k == 2) return {(float)-c, (float)-s};
    return {(float)s, (float)-c};
}
struct TwTable {
    Tw v[64];
};
constexpr TwTable make_table()
{
    TwTable t{};
    for (int i = 0; i < 64; i++) t.v[i] = make_tw(i);
    return t;
}

#ifdef __CUDA_ARCH__
__constant__ constexpr TwTable kTw = make_table();
#else
constexpr TwTable kTw = make_table();
#endif

SCFT_HD constexpr int perm(int k) { return (k >> 3) + 8 * (k & 7); }

// load of data that other CTAs of the same launch may have written (the
// persistent step kernel): served from L2, never from a stale L1 line
SCFT_HD float2 ld_shared_gm(const float2 *p)
{
#ifdef __CUDA_ARCH__
    return __ldcg(p);
#else
    return *p;
#endif
}

SCFT_HD float2 cadd2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
SCFT_HD float2 csub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a * exp(SIGN 2 pi i t/64)
template <int SIGN>
SCFT_HD float2 twmul(float2 a, int t)
{
    const Tw w = kTw.v[t & 63];
    const float s = SIGN > 0 ? w.s : -w.s;
    return make_float2(a.x * w.c - a.y * s, a.x * s + a.y * w.c);
}
// a * SIGN i
template <int SIGN>
SCFT_HD float2 muli(float2 a)
{
    return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// 8-point DFT (sign SIGN) of v[b], v[b+st], ..., v[b+7st] in place, natural
// order in and out: V[q] = sum_r v[r] exp(SIGN 2 pi i r q / 8)
template <int SIGN>
SCFT_HD void dft8(float2 *v, int b, int st)
{
    const float h = 0.70710678118654752440f;
    float2 x0 = v[b], x1 = v[b + st], x2 = v[b + 2 * st], x3 = v[b + 3 * st];
    float2 x4 = v[b + 4 * st], x5 = v[b + 5 * st], x6 = v[b + 6 * st], x7 = v[b + 7 * st];
    // even / odd 4-point DFTs
    float2 a = cadd2(x0, x4), bb = csub2(x0, x4), c = cadd2(x2, x6), d = muli<SIGN>(csub2(x2, x6));
    const float2 e0 = cadd2(a, c), e1 = cadd2(bb, d), e2 = csub2(a, c), e3 = csub2(bb, d);
    a = cadd2(x1, x5);
    bb = csub2(x1, x5);
    c = cadd2(x3, x7);
    d = muli<SIGN>(csub2(x3, x7));
    float2 o0 = cadd2(a, c), o1 = cadd2(bb, d), o2 = csub2(a, c), o3 = csub2(bb, d);
    // o[k] *= exp(SIGN 2 pi i k/8)
    const float s = (float)SIGN;
    o1 = make_float2(h * (o1.x - s * o1.y), h * (o1.y + s * o1.x));
    o2 = muli<SIGN>(o2);
    o3 = make_float2(h * (-o3.x - s * o3.y), h * (-o3.y + s * o3.x));
    v[b] = cadd2(e0, o0);
    v[b + 4 * st] = csub2(e0, o0);
    v[b + st] = cadd2(e1, o1);
    v[b + 5 * st] = csub2(e1, o1);
    v[b + 2 * st] = cadd2(e2, o2);
    v[b + 6 * st] = csub2(e2, o2);
    v[b + 3 * st] = cadd2(e3, o3);
    v[b + 7 * st] = csub2(e3, o3);
}

// 64-point FFT of v (natural order in), X[k] = sum_n v[n] exp(SIGN 2 pi i n k/64),
// unnormalised; X[k] ends in v[perm(k)].
template <int SIGN>
SCFT_HD void fft64(float2 *v)
{
#pragma unroll
    for (int j = 0; j < 8; j++) dft8<SIGN>(v, j, 8);  // v[j + 8q] = Y[j][q]
#pragma unroll
    for (int j = 1; j < 8; j++)
#pragma unroll
        for (int q = 1; q < 8; q++) v[j + 8 * q] = twmul<SIGN>(v[j + 8 * q], j * q);
#pragma unroll
    for (int q = 0; q < 8; q++) dft8<SIGN>(v, 8 * q, 1);  // v[s + 8q] = X[q + 8s]
}

// The same transform with the input in the permuted order fft64 leaves its
// output in (x[n] in v[perm(n)]), and the output in natural order (X[k] in
// v[k]): with x[j + 8r] at v[r + 8j], pass 1 runs over contiguous blocks and
// pass 2 over stride-8 sets.  A forward fft64, a pointwise scale and an
// inverse fft64_pin need no reordering in between.
template <int SIGN>
SCFT_HD void fft64_pin(float2 *v)
{
#pragma unroll
    for (int j = 0; j < 8; j++) dft8<SIGN>(v, 8 * j, 1);  // v[q + 8j] = Y[j][q]
#pragma unroll
    for (int j = 1; j < 8; j++)
#pragma unroll
        for (int q = 1; q < 8; q++) v[q + 8 * j] = twmul<SIGN>(v[q + 8 * j], j * q);
#pragma unroll
    for (int q = 0; q < 8; q++) dft8<SIGN>(v, q, 8);  // v[q + 8s] = X[q + 8s]
}

// ---------------------------------------------------------------- slab phases
// R: real tile [64 rows y][kRowPitch] (z in 0..63); T: complex tile viewed as
// [33 columns kz][kColPitch] (y in 0..63) aliasing R.  Each phase is what
// one lane does between two __syncwarp of the warp owning the slab.

// forward z pass, load half: lane p packs rows p and p+32 into v (natural z order)
SCFT_HD void fz_load(const float *R, int p, float2 *v)
{
    const float *ra = R + p * kRowPitch, *rb = R + (p + 32) * kRowPitch;
#pragma unroll
    for (int z = 0; z < 64; z += 4) {
        const float4 a = *reinterpret_cast<const float4 *>(ra + z);
        const float4 b = *reinterpret_cast<const float4 *>(rb + z);
        v[z] = make_float2(a.x, b.x);
        v[z + 1] = make_float2(a.y, b.y);
        v[z + 2] = make_float2(a.z, b.z);
        v[z + 3] = make_float2(a.w, b.w);
    }
}

// forward z pass, transform and store half: the two rows' half spectra into
// column kz of T at rows p and p+32; column 0 holds (X(0), X(32)) of each row
SCFT_HD void fz_fft_store(float2 *T, int p, float2 *v)
{
    fft64<-1>(v);
    const float2 c0 = v[perm(0)], c32 = v[perm(32)];
    T[p] = make_float2(c0.x, c32.x);       // row p:    real X(0), real X(32)
    T[p + 32] = make_float2(c0.y, c32.y);  // row p+32
#pragma unroll
    for (int k = 1; k < 32; k++) {
        const float2 ck = v[perm(k)], cm = v[perm(64 - k)];
        T[k * kColPitch + p] = make_float2(0.5f * (ck.x + cm.x), 0.5f * (ck.y - cm.y));
        T[k * kColPitch + p + 32] = make_float2(0.5f * (ck.y + cm.y), 0.5f * (cm.x - ck.x));
    }
}

// forward y pass: lane kz transforms column kz (lane 0: the joined column
// c0 + i c32, split after the transform) and stores it to the spectrum plane
// out[ky * 33 + kz] (global memory, coalesced across lanes)
SCFT_HD void fy(const float2 *T, int kz, float2 *v, float2 *out)
{
#pragma unroll
    for (int y = 0; y < 64; y++) v[y] = T[kz * kColPitch + y];
    fft64<-1>(v);
    if (kz == 0) {
#pragma unroll
        for (int k = 0; k < 64; k++) {
            const float2 c = v[perm(k)], cm = v[perm((64 - k) & 63)];
            out[k * kMK] = make_float2(0.5f * (c.x + cm.x), 0.5f * (c.y - cm.y));
            out[k * kMK + 32] = make_float2(0.5f * (c.y + cm.y), 0.5f * (cm.x - c.x));
        }
    } else {
#pragma unroll
        for (int k = 0; k < 64; k++) out[k * kMK + kz] = v[perm(k)];
    }
}

// inverse y pass: lane kz loads column kz of the spectrum plane (lane 0 joins
// kz = 0 and 32 as X0 + i X32), transforms it and writes column kz of T
SCFT_HD void iy(const float2 *in, int kz, float2 *v, float2 *T)
{
    if (kz == 0) {
#pragma unroll
        for (int k = 0; k < 64; k++) {
            const float2 a = ld_shared_gm(in + k * kMK), h = ld_shared_gm(in + k * kMK + 32);
            v[k] = make_float2(a.x - h.y, a.y + h.x);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 64; k++) v[k] = ld_shared_gm(in + k * kMK + kz);
    }
    fft64<+1>(v);
#pragma unroll
    for (int y = 0; y < 64; y++) T[kz * kColPitch + y] = v[perm(y)];
}

// inverse z pass, load half: lane p gathers the half spectra of rows p and
// p+32 from T and forms the packed line C(k) = A(k) + i B(k), with
// C(64-k) = conj A(k) + i conj B(k); the imaginary parts of the
// self-conjugate bins kz = 0, 32 are dropped (half-complex-to-real semantics)
SCFT_HD void iz_load(const float2 *T, int p, float2 *v)
{
    const float2 j0 = T[p], j1 = T[p + 32];  // (A0, A32) of row p, (B0, B32) of row p+32 (real parts)
    v[0] = make_float2(j0.x, j1.x);
    v[32] = make_float2(j0.y, j1.y);
#pragma unroll
    for (int k = 1; k < 32; k++) {
        const float2 A = T[k * kColPitch + p], B = T[k * kColPitch + p + 32];
        v[k] = make_float2(A.x - B.y, A.y + B.x);
        v[64 - k] = make_float2(A.x + B.y, B.x - A.y);
    }
}

// inverse z pass, transform and store half: rows p and p+32 of R
SCFT_HD void iz_fft_store(float *R, int p, float2 *v)
{
    fft64<+1>(v);
    float *ra = R + p * kRowPitch, *rb = R + (p + 32) * kRowPitch;
#pragma unroll
    for (int z = 0; z < 64; z += 4) {
        const float2 c0 = v[perm(z)], c1 = v[perm(z + 1)], c2 = v[perm(z + 2)], c3 = v[perm(z + 3)];
        *reinterpret_cast<float4 *>(ra + z) = make_float4(c0.x, c1.x, c2.x, c3.x);
        *reinterpret_cast<float4 *>(rb + z) = make_float4(c0.y, c1.y, c2.y, c3.y);
    }
}

}  // namespace reg64
}  // namespace scft
