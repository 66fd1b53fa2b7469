// stress_kernels.cu -- box-size derivative of lnQ by the adjoint of the
// Richardson propagator (no reference code; checked against central finite
// differences of the reference's own discretisation).
//
// One contour step of q is S = (4 E4 D2 E2 D2 E4 - E2 D1 E2)/3 with real
// diagonal E and symmetric circulant D = F^-1 diag(K/M) F (density.h:129-220),
// so S is symmetric and q^dagger's step t is q's step N-1-t.  Hence the
// adjoint of q's chain is the stored q^dagger:
//   dQC/dL = (1/M) sum_s < q^dagger(N-1-s), dS_s/dL q(s) >
//   dQ2/dL = (1/M) sum_j < q^dagger(Nh-1-j), dS_B/dL q^dagger(j) >
// and by Parseval, with X = FFT, u4 = E4 x, u2 = E2 x, w = E2 D2 E4 x (same for y):
//   < y, dS/dL x > = (1/M) [ 4/3 sum dK2 Re(X(w_x) conj X(u4_y) + X(u4_x) conj X(w_y))
//                           - 1/3 sum dK1 Re(X(u2_x) conj X(u2_y)) ]
// over the full spectrum (half spectrum with weight 2 off the kz = 0, m2/2
// planes), dK2/dL_i = K2 (ds/12) 8 pi^2 n_i^2 / L_i^3, dK1/dL_i = K1 (ds/6) 8 pi^2 n_i^2 / L_i^3.
//
// Pairs are processed in chunks; per chunk four launches: slab forward (u4,
// u2 of x and y), pencil 1 (x forward; dK1 sums; K2, x inverse of u4),
// slab mid (E2 D2 E4), pencil 2 (x forward; dK2 sums).
#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"

namespace scft {

namespace {

template <typename T>
__device__ __forceinline__ const T *slice(const StressArgs<T> &a, int s, int fld)
{
    return a.hist + (((size_t)a.slot * (a.g.Ns + 1) + s) * 2 + fld) * (size_t)a.g.M;
}

// E4 table `sel` (0 A, 1 B, 2 junction step) of the slot
template <typename T>
__device__ __forceinline__ const T *etab_of(const StressArgs<T> &a, int sel)
{
    return sel == 2 ? a.jtab + (size_t)a.slot * a.g.M : a.etab + ((size_t)a.slot * 2 + sel) * a.g.M;
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

// u4 = E4 x and u2 = E2 x (and the same for y), forward slab transforms
template <typename T>
__global__ void k_stress_slab_fwd(StressArgs<T> a, StressPairs P)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twy = buf + g.slab_c;
    cplx<T> *twz = twy + g.m1;
    for (int i = threadIdx.x; i < g.m1; i += blockDim.x) twy[i] = a.tw[g.m0 + i];
    for (int i = threadIdx.x; i < g.m2; i += blockDim.x) twz[i] = a.tw[g.m0 + g.m1 + i];
    const int x = blockIdx.x, xy = blockIdx.y, p = blockIdx.z;
    const int m1 = g.m1, m2 = g.m2, mk2 = g.mk2;
    const size_t slab_r = (size_t)x * m1 * m2, slab_k = (size_t)x * m1 * mk2;
    const T *src = slice(a, xy ? P.ys[p] : P.xs[p], xy ? P.yf[p] : P.xf[p]) + slab_r;
    const T *E4 = etab_of(a, P.sel[p]) + slab_r;
    const int npz = g.npair * m2;
    for (int pass = 0; pass < 2; pass++) {
        __syncthreads();
        for (int e = threadIdx.x; e < npz; e += blockDim.x) {
            const int pp = e / m2, z = e - pp * m2;
            const int r0 = 2 * pp * m2 + z;
            T e0 = E4[r0], v1 = (T)0;
            if (pass) e0 *= e0;
            if (2 * pp + 1 < m1) {
                T e1 = E4[r0 + m2];
                if (pass) e1 *= e1;
                v1 = src[r0 + m2] * e1;
            }
            buf[2 * pp * mk2 + z] = {src[r0] * e0, v1};
        }
        __syncthreads();
        slab_forward(buf, g, twy, twz, a.err);
        cplx<T> *dst = (pass ? a.S2 : a.S4) + ((size_t)p * 2 + xy) * g.Mk + slab_k;
        for (int i = threadIdx.x; i < m1 * mk2; i += blockDim.x) dst[i] = buf[i];
    }
}

// per-element weights of dK/dL_i: n_i^2 * 8 pi^2 / L_i^3 (the ds/12 and K factors are applied by the caller)
template <typename T>
__device__ __forceinline__ void dk_weights(const StressArgs<T> &a, int xk, int c, double wi[3], double &K2,
                                           double &hw)
{
    const Geo &g = a.g;
    const int yk = c / g.mk2, kz = c - yk * g.mk2;
    const int n0 = xk <= g.m0 / 2 ? xk : xk - g.m0;
    const int n1 = yk <= g.m1 / 2 ? yk : yk - g.m1;
    const double PI = 3.14159265358979323846;
    wi[0] = 8.0 * PI * PI * (double)n0 * n0 / (a.L[0] * a.L[0] * a.L[0]);
    wi[1] = 8.0 * PI * PI * (double)n1 * n1 / (a.L[1] * a.L[1] * a.L[1]);
    wi[2] = 8.0 * PI * PI * (double)kz * kz / (a.L[2] * a.L[2] * a.L[2]);
    K2 = (double)a.kfac[xk] * (double)a.kfac[g.m0 + yk] * (double)a.kfac[g.m0 + g.m1 + kz];
    hw = (kz == 0 || 2 * kz == g.m2) ? 1.0 : 2.0;
}

// x forward of u4 (x, y) and u2 (x, y); dK1 sums of u2; K2/M and x inverse of u4
template <typename T>
__global__ void k_stress_pencil1(StressArgs<T> a)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ double sh[32];
    const Geo &g = a.g;
    const int tc = g.tc, m0 = g.m0, ncol = g.m1 * g.mk2;
    cplx<T> *bx = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *by = bx + tc * m0;
    cplx<T> *twx = by + tc * m0;
    for (int i = threadIdx.x; i < m0; i += blockDim.x) twx[i] = a.tw[i];
    const int tile = blockIdx.x, p = blockIdx.y, c0 = tile * tc;
    const double ds = 1.0 / g.Ns;
    // dK1 sums over the full-step spectra
    {
        const cplx<T> *sx = a.S2 + ((size_t)p * 2 + 0) * g.Mk, *sy = a.S2 + ((size_t)p * 2 + 1) * g.Mk;
        __syncthreads();
        for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
            const int xx = e / tc, t = e - xx * tc, c = c0 + t;
            bx[e] = c < ncol ? sx[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
            by[e] = c < ncol ? sy[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
        }
        __syncthreads();
        cta_fft(bx, g.px, tc, tc, 1, true, twx, -1, a.err);
        cta_fft(by, g.px, tc, tc, 1, true, twx, -1, a.err);
        double acc[3] = {0, 0, 0};
        for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
            const int xx = e / tc, t = e - xx * tc, c = c0 + t;
            if (c >= ncol) continue;
            double wi[3], K2, hw;
            dk_weights(a, xx, c, wi, K2, hw);
            const double re = (double)bx[e].x * by[e].x + (double)bx[e].y * by[e].y;
            const double k1 = K2 * K2 * (ds / 6.0) * hw * re;
            for (int i = 0; i < 3; i++) acc[i] += k1 * wi[i];
        }
        for (int i = 0; i < 3; i++) {
            const double t = bsum(acc[i], sh);
            if (threadIdx.x == 0) a.part[((size_t)p * 9 + 6 + i) * gridDim.x + tile] = t;
        }
    }
    // u4: forward x (kept for pencil 2), then K2/M and inverse x into S4p
    for (int xy = 0; xy < 2; xy++) {
        cplx<T> *s4 = a.S4 + ((size_t)p * 2 + xy) * g.Mk, *s4p = a.S4p + ((size_t)p * 2 + xy) * g.Mk;
        __syncthreads();
        for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
            const int xx = e / tc, t = e - xx * tc, c = c0 + t;
            bx[e] = c < ncol ? s4[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
        }
        __syncthreads();
        cta_fft(bx, g.px, tc, tc, 1, true, twx, -1, a.err);
        for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
            const int xx = e / tc, t = e - xx * tc, c = c0 + t;
            if (c < ncol) s4[(size_t)xx * ncol + c] = bx[e];
            const int yk = c / g.mk2, kz = c - yk * g.mk2;
            const T f = c < ncol ? a.kfac[xx] * a.kfac[m0 + yk] * a.kfac[m0 + g.m1 + kz] * a.invM : (T)0;
            bx[e].x *= f;
            bx[e].y *= f;
        }
        __syncthreads();
        cta_fft(bx, g.px, tc, tc, 1, true, twx, +1, a.err);
        for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
            const int xx = e / tc, t = e - xx * tc, c = c0 + t;
            if (c < ncol) s4p[(size_t)xx * ncol + c] = bx[e];
        }
    }
}

// w = E2 D2 E4 x: inverse slab, times E2, forward slab
template <typename T>
__global__ void k_stress_slab_mid(StressArgs<T> a, StressPairs P)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twy = buf + g.slab_c;
    cplx<T> *twz = twy + g.m1;
    for (int i = threadIdx.x; i < g.m1; i += blockDim.x) twy[i] = a.tw[g.m0 + i];
    for (int i = threadIdx.x; i < g.m2; i += blockDim.x) twz[i] = a.tw[g.m0 + g.m1 + i];
    const int x = blockIdx.x, xy = blockIdx.y, p = blockIdx.z;
    const int m1 = g.m1, m2 = g.m2, mk2 = g.mk2;
    const size_t slab_r = (size_t)x * m1 * m2, slab_k = (size_t)x * m1 * mk2;
    const T *E4 = etab_of(a, P.sel[p]) + slab_r;
    cplx<T> *sp = a.S4p + ((size_t)p * 2 + xy) * g.Mk + slab_k;
    for (int i = threadIdx.x; i < m1 * mk2; i += blockDim.x) buf[i] = sp[i];
    __syncthreads();
    slab_inverse(buf, g, twy, twz, a.err);
    const int npz = g.npair * m2;
    for (int e = threadIdx.x; e < npz; e += blockDim.x) {
        const int pp = e / m2, z = e - pp * m2;
        cplx<T> &c = buf[2 * pp * mk2 + z];
        const int r0 = 2 * pp * m2 + z;
        const T e0 = E4[r0];
        c.x *= e0 * e0;
        if (2 * pp + 1 < m1) {
            const T e1 = E4[r0 + m2];
            c.y *= e1 * e1;
        } else {
            c.y = (T)0;
        }
    }
    __syncthreads();
    slab_forward(buf, g, twy, twz, a.err);
    for (int i = threadIdx.x; i < m1 * mk2; i += blockDim.x) sp[i] = buf[i];
}

// x forward of w (x, y); dK2 sums  Re(W_x conj U4_y + U4_x conj W_y)
template <typename T>
__global__ void k_stress_pencil2(StressArgs<T> a)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ double sh[32];
    const Geo &g = a.g;
    const int tc = g.tc, m0 = g.m0, ncol = g.m1 * g.mk2;
    cplx<T> *bx = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *by = bx + tc * m0;
    cplx<T> *twx = by + tc * m0;
    for (int i = threadIdx.x; i < m0; i += blockDim.x) twx[i] = a.tw[i];
    const int tile = blockIdx.x, p = blockIdx.y, c0 = tile * tc;
    const double ds = 1.0 / g.Ns;
    const cplx<T> *wx = a.S4p + ((size_t)p * 2 + 0) * g.Mk, *wy = a.S4p + ((size_t)p * 2 + 1) * g.Mk;
    const cplx<T> *ux = a.S4 + ((size_t)p * 2 + 0) * g.Mk, *uy = a.S4 + ((size_t)p * 2 + 1) * g.Mk;
    __syncthreads();
    for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
        const int xx = e / tc, t = e - xx * tc, c = c0 + t;
        bx[e] = c < ncol ? wx[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
        by[e] = c < ncol ? wy[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
    }
    __syncthreads();
    cta_fft(bx, g.px, tc, tc, 1, true, twx, -1, a.err);
    cta_fft(by, g.px, tc, tc, 1, true, twx, -1, a.err);
    double acc[3] = {0, 0, 0};
    for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
        const int xx = e / tc, t = e - xx * tc, c = c0 + t;
        if (c >= ncol) continue;
        double wi[3], K2, hw;
        dk_weights(a, xx, c, wi, K2, hw);
        const cplx<T> Ux = ux[(size_t)xx * ncol + c], Uy = uy[(size_t)xx * ncol + c];
        const double re = ((double)bx[e].x * Uy.x + (double)bx[e].y * Uy.y) +
                          ((double)Ux.x * by[e].x + (double)Ux.y * by[e].y);
        const double k2 = K2 * (ds / 12.0) * hw * re;
        for (int i = 0; i < 3; i++) acc[i] += k2 * wi[i];
    }
    for (int i = 0; i < 3; i++) {
        const double t = bsum(acc[i], sh);
        if (threadIdx.x == 0) a.part[((size_t)p * 9 + i) * gridDim.x + tile] = t;
    }
}

// < y, dS/dL_i x > for every pair of the chunk
__global__ void k_stress_final(const double *part, int ntiles, int npairs, double invM, double *out)
{
    const int p = blockIdx.x;
    if (p >= npairs || threadIdx.x >= 3) return;
    const int i = threadIdx.x;
    double t12 = 0, t3 = 0;
    for (int t = 0; t < ntiles; t++) {
        t12 += part[((size_t)p * 9 + i) * ntiles + t];
        t3 += part[((size_t)p * 9 + 6 + i) * ntiles + t];
    }
    out[p * 3 + i] = invM * (4.0 / 3.0 * t12 - 1.0 / 3.0 * t3);
}

// ---------------------------------------------------------------- junction step
// d/dtheta of q's junction step with a continuous A fraction.  The step is
// S = (4 E4 D2 E2 D2 E4 - E2 D1 E2)/3 with the field theta wA + (1-theta) wB,
// so dE4/dtheta = -(ds/4) delta E4, dE2/dtheta = -(ds/2) delta E2 with
// delta = wA - wB = 2 W-.  With b = D2 E4 v, d = D2 E2 b, g = D1 E2 v
// (v = x, y; D symmetric, E diagonal):
//   <y, dS/dtheta x> = -(ds/3) sum delta (y E4 d_x + d_y E4 x)
//                      -(2 ds/3) sum delta b_y E2 b_x
//                      +(ds/6) sum delta (y E2 g_x + g_y E2 x)
// Launches: k_stress_slab_fwd (spectra of E4 v, E2 v), pencil pass 0 (K2 on
// the first, K1 on the second), slab pass 0 (b, g real; spectrum of E2 b),
// pencil pass 1 (K2), slab pass 1 (d real), reduction.
// rbuf rows: 0 b_x, 1 b_y, 2 g_x, 3 g_y, 4 d_x, 5 d_y.

// x transform of a column tile, times K2/M (k1 = 0) or K1/M (k1 = 1), back
template <typename T>
__device__ void jn_pencil_tile(const StressArgs<T> &a, cplx<T> *bx, const cplx<T> *twx, const cplx<T> *src,
                               cplx<T> *dst, int c0, int k1)
{
    const Geo &g = a.g;
    const int tc = g.tc, m0 = g.m0, ncol = g.m1 * g.mk2;
    __syncthreads();
    for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
        const int xx = e / tc, t = e - xx * tc, c = c0 + t;
        bx[e] = c < ncol ? src[(size_t)xx * ncol + c] : cplx<T>{(T)0, (T)0};
    }
    __syncthreads();
    cta_fft(bx, g.px, tc, tc, 1, true, twx, -1, a.err);
    for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
        const int xx = e / tc, t = e - xx * tc, c = c0 + t;
        const int yk = c / g.mk2, kz = c - yk * g.mk2;
        T f = (T)0;
        if (c < ncol) {
            const T k = a.kfac[xx] * a.kfac[m0 + yk] * a.kfac[m0 + g.m1 + kz];
            f = (k1 ? k * k : k) * a.invM;
        }
        bx[e].x *= f;
        bx[e].y *= f;
    }
    __syncthreads();
    cta_fft(bx, g.px, tc, tc, 1, true, twx, +1, a.err);
    for (int e = threadIdx.x; e < tc * m0; e += blockDim.x) {
        const int xx = e / tc, t = e - xx * tc, c = c0 + t;
        if (c < ncol) dst[(size_t)xx * ncol + c] = bx[e];
    }
}

template <typename T>
__global__ void k_jn_pencil(StressArgs<T> a, int pass)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    cplx<T> *bx = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twx = bx + g.tc * g.m0;
    for (int i = threadIdx.x; i < g.m0; i += blockDim.x) twx[i] = a.tw[i];
    const int tile = blockIdx.x, xy = blockIdx.y, c0 = tile * g.tc;
    cplx<T> *s4 = a.S4 + (size_t)xy * g.Mk, *s4p = a.S4p + (size_t)xy * g.Mk, *s2 = a.S2 + (size_t)xy * g.Mk;
    jn_pencil_tile(a, bx, twx, s4, s4p, c0, 0);
    if (pass == 0) jn_pencil_tile(a, bx, twx, s2, s2, c0, 1);
}

// inverse slab transform of `src` into the real slab `dst` (slab_r offset applied)
template <typename T>
__device__ void jn_slab_to_real(const StressArgs<T> &a, cplx<T> *buf, const cplx<T> *twy, const cplx<T> *twz,
                                const cplx<T> *src, T *dst)
{
    const Geo &g = a.g;
    const int m1 = g.m1, m2 = g.m2, mk2 = g.mk2;
    __syncthreads();
    for (int i = threadIdx.x; i < m1 * mk2; i += blockDim.x) buf[i] = src[i];
    __syncthreads();
    slab_inverse(buf, g, twy, twz, a.err);
    for (int e = threadIdx.x; e < g.npair * m2; e += blockDim.x) {
        const int pp = e / m2, z = e - pp * m2;
        const cplx<T> c = buf[2 * pp * mk2 + z];
        const int r0 = 2 * pp * m2 + z;
        dst[r0] = c.x;
        if (2 * pp + 1 < m1) dst[r0 + m2] = c.y;
    }
}

template <typename T>
__global__ void k_jn_slab(StressArgs<T> a, int pass)
{
    extern __shared__ unsigned char smem_raw[];
    const Geo &g = a.g;
    cplx<T> *buf = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *twy = buf + g.slab_c;
    cplx<T> *twz = twy + g.m1;
    for (int i = threadIdx.x; i < g.m1; i += blockDim.x) twy[i] = a.tw[g.m0 + i];
    for (int i = threadIdx.x; i < g.m2; i += blockDim.x) twz[i] = a.tw[g.m0 + g.m1 + i];
    const int x = blockIdx.x, xy = blockIdx.y;
    const int m1 = g.m1, m2 = g.m2, mk2 = g.mk2;
    const size_t M = g.M, slab_r = (size_t)x * m1 * m2, slab_k = (size_t)x * m1 * mk2;
    cplx<T> *s4 = a.S4 + (size_t)xy * g.Mk + slab_k, *s4p = a.S4p + (size_t)xy * g.Mk + slab_k;
    cplx<T> *s2 = a.S2 + (size_t)xy * g.Mk + slab_k;
    if (pass == 1) {
        jn_slab_to_real(a, buf, twy, twz, s4p, a.rbuf + (4 + xy) * M + slab_r);  // d
        return;
    }
    T *b = a.rbuf + (0 + xy) * M + slab_r;
    jn_slab_to_real(a, buf, twy, twz, s4p, b);                                  // b = D2 E4 v
    const T *E4 = etab_of(a, 2) + slab_r;
    __syncthreads();
    for (int e = threadIdx.x; e < g.npair * m2; e += blockDim.x) {
        const int pp = e / m2, z = e - pp * m2;
        const int r0 = 2 * pp * m2 + z;
        const T e0 = E4[r0];
        T v1 = (T)0;
        if (2 * pp + 1 < m1) {
            const T e1 = E4[r0 + m2];
            v1 = b[r0 + m2] * (e1 * e1);
        }
        buf[2 * pp * mk2 + z] = {b[r0] * (e0 * e0), v1};
    }
    __syncthreads();
    slab_forward(buf, g, twy, twz, a.err);                                      // spectrum of E2 b
    for (int i = threadIdx.x; i < m1 * mk2; i += blockDim.x) s4[i] = buf[i];
    jn_slab_to_real(a, buf, twy, twz, s2, a.rbuf + (2 + xy) * M + slab_r);      // g = D1 E2 v
}

template <typename T>
__global__ void k_jn_reduce(StressArgs<T> a, StressPairs P, double *part)
{
    __shared__ double sh[32];
    const Geo &g = a.g;
    const size_t M = g.M;
    const T *x = slice(a, P.xs[0], P.xf[0]), *y = slice(a, P.ys[0], P.yf[0]);
    const T *E4 = etab_of(a, 2);
    const T *bx = a.rbuf, *by = a.rbuf + M, *gx = a.rbuf + 2 * M, *gy = a.rbuf + 3 * M;
    const T *dx = a.rbuf + 4 * M, *dy = a.rbuf + 5 * M;
    const double ds = 1.0 / g.Ns;
    double acc = 0;
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += (size_t)gridDim.x * blockDim.x) {
        const double del = 2.0 * a.wminus[r];
        const double e4 = (double)E4[r], e2 = e4 * e4;
        const double X = x[r], Y = y[r];
        const double t1 = Y * e4 * (double)dx[r] + (double)dy[r] * e4 * X;
        const double t2 = (double)by[r] * e2 * (double)bx[r];
        const double t3 = Y * e2 * (double)gx[r] + (double)gy[r] * e2 * X;
        acc += del * (-(ds / 3.0) * t1 - (2.0 * ds / 3.0) * t2 + (ds / 6.0) * t3);
    }
    const double t = bsum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_jn_final(const double *part, int nblk, double *out)
{
    if (threadIdx.x != 0) return;
    double t = 0;
    for (int i = 0; i < nblk; i++) t += part[i];
    out[0] = t;
}

}  // namespace

template <typename T>
int launch_junction_dtheta(const StressArgs<T> &a, const StressPairs &P, int slab_threads, int slab_smem,
                           int pencil_threads, int pencil_smem, double *part, int nblk, double *out,
                           cudaStream_t st)
{
    const Geo &g = a.g;
    k_stress_slab_fwd<T><<<dim3(g.m0, 2, 1), slab_threads, slab_smem, st>>>(a, P);
    k_jn_pencil<T><<<dim3(g.ncol_tiles, 2), pencil_threads, pencil_smem, st>>>(a, 0);
    k_jn_slab<T><<<dim3(g.m0, 2), slab_threads, slab_smem, st>>>(a, 0);
    k_jn_pencil<T><<<dim3(g.ncol_tiles, 2), pencil_threads, pencil_smem, st>>>(a, 1);
    k_jn_slab<T><<<dim3(g.m0, 2), slab_threads, slab_smem, st>>>(a, 1);
    k_jn_reduce<T><<<nblk, 256, 0, st>>>(a, P, part);
    k_jn_final<<<1, 32, 0, st>>>(part, nblk, out);
    return 7;
}

template <typename T>
int launch_stress_chunk(const StressArgs<T> &a, const StressPairs &P, int slab_threads, int slab_smem,
                        int pencil_threads, int pencil_smem, double *out, cudaStream_t st)
{
    const Geo &g = a.g;
    k_stress_slab_fwd<T><<<dim3(g.m0, 2, P.n), slab_threads, slab_smem, st>>>(a, P);
    k_stress_pencil1<T><<<dim3(g.ncol_tiles, P.n), pencil_threads, pencil_smem, st>>>(a);
    k_stress_slab_mid<T><<<dim3(g.m0, 2, P.n), slab_threads, slab_smem, st>>>(a, P);
    k_stress_pencil2<T><<<dim3(g.ncol_tiles, P.n), pencil_threads, pencil_smem, st>>>(a);
    k_stress_final<<<P.n, 32, 0, st>>>(a.part, g.ncol_tiles, P.n, 1.0 / g.M, out);
    return 5;
}

template <typename T>
int set_stress_smem(int slab_smem, int pencil_smem)
{
    cudaError_t e1 = raise_dyn_smem(k_stress_slab_fwd<T>, slab_smem);
    cudaError_t e2 = raise_dyn_smem(k_stress_slab_mid<T>, slab_smem);
    cudaError_t e3 = raise_dyn_smem(k_stress_pencil1<T>, pencil_smem);
    cudaError_t e4 = raise_dyn_smem(k_stress_pencil2<T>, pencil_smem);
    cudaError_t e5 = raise_dyn_smem(k_jn_slab<T>, slab_smem);
    cudaError_t e6 = raise_dyn_smem(k_jn_pencil<T>, pencil_smem);
    return (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess && e4 == cudaSuccess &&
            e5 == cudaSuccess && e6 == cudaSuccess) ? 0 : -1;
}

template int launch_stress_chunk<float>(const StressArgs<float> &, const StressPairs &, int, int, int, int, double *, cudaStream_t);
template int launch_stress_chunk<double>(const StressArgs<double> &, const StressPairs &, int, int, int, int, double *, cudaStream_t);
template int launch_junction_dtheta<float>(const StressArgs<float> &, const StressPairs &, int, int, int, int,
                                           double *, int, double *, cudaStream_t);
template int launch_junction_dtheta<double>(const StressArgs<double> &, const StressPairs &, int, int, int, int,
                                            double *, int, double *, cudaStream_t);
template int set_stress_smem<float>(int, int);
template int set_stress_smem<double>(int, int);

}  // namespace scft
