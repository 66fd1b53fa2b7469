// reg64.cu -- the 64^3 FP32 contour step on register-resident transforms.
//
// Same four roles per Richardson step as the shared-memory kernels of
// props_kernels.cu (density.h:129-220, GPU_kernels.h:175-203), same buffers
// and layouts (reference order r = z + 64 (y + 64 x), half spectra
// [x][ky][kz] with 33 kz), so the two paths are interchangeable per launch:
//   pencil  one thread per (ky, kz) column: the 64 x values are loaded
//           (coalesced across the warp), transformed, scaled by the diffusion
//           factor and transformed back without leaving registers;
//   mid     one warp per x-slab: inverse slab of the full step -> P = E2 qs1;
//           inverse slab of the half step, times E2, forward slab;
//   combine one warp per x-slab: inverse slab -> q' = (4 E4 qs0 - P)/3 ->
//           propagator store; forward slabs of E4' q' and E2' q'.
// A slab transform is two passes of 64-point register FFTs (z, then y) with
// one trip through a per-warp shared tile in between (reg64.cuh); the
// elementwise epilogues read and write the tile with lanes across z, so every
// global access is a coalesced row.
#include "common.cuh"
#include "kernels.h"
#include "reg64.cuh"

namespace scft {
namespace {

using namespace reg64;
constexpr int kM = 64 * 64 * 64;
constexpr int kMk = 64 * kPlane;
constexpr int kWPB = 4;  // warps (slabs) per CTA of the slab kernels
constexpr int kPencilThreads = 128;

__device__ __forceinline__ size_t hoff(const Geo &g, int slot, int s, int fld)
{
    return (((size_t)slot * (g.Ns + 1) + s) * 2 + fld) * (size_t)kM;
}

__device__ __forceinline__ int esel(const Geo &g, int fld, int s)
{
    if (g.jon && s == (fld == 0 ? g.jq : g.jqd)) return 2;
    return fld == 0 ? (s < g.n1 ? 0 : 1) : (s < g.n2 ? 1 : 0);
}

__device__ __forceinline__ const float *eptr(const PropsArgs<float> &a, int slot, int sel)
{
    return sel == 2 ? a.jtab + (size_t)slot * kM : a.etab + ((size_t)slot * 2 + sel) * kM;
}

// inverse slab transform of the spectrum plane `in` into the real tile R.
// The slab transforms are kept out of line: every kernel calls them two or
// three times, and inlined copies of their unrolled 64-point transforms
// overflow the instruction cache.
__device__ __noinline__ void slab_inverse(const float2 *in, float *R, int lane)
{
    float2 v[64];
    float2 *T = reinterpret_cast<float2 *>(R);
    __syncwarp();
    iy(in, lane, v, T);
    __syncwarp();
    iz_load(T, lane, v);
    __syncwarp();
    iz_fft_store(R, lane, v);
    __syncwarp();
}

// forward slab transform of the real tile R into the spectrum plane `out`
__device__ __noinline__ void slab_forward(float *R, float2 *out, int lane)
{
    float2 v[64];
    float2 *T = reinterpret_cast<float2 *>(R);
    __syncwarp();
    fz_load(R, lane, v);
    __syncwarp();
    fz_fft_store(T, lane, v);
    __syncwarp();
    fy(T, lane, v, out);
    __syncwarp();
}

// ---------------------------------------------------------------- pencil
// Column c of spectrum A (times K2) and, when both != 0, of spectrum B (times
// K1) of (slot, fld) (Mult_self, GPU_kernels.h:175-181; factors
// Prepare_dev_expKsq2_expKsq, GPU_kernels.h:207-213, from the replica's
// separable per-axis table).
__device__ __forceinline__ void pencil_column(const PropsArgs<float> &a, int both, int slot, int fld, int c)
{
    const int ky = c / kMK, kz = c - ky * kMK;
    const float *kf = a.kfac + (size_t)a.slot_rep[slot] * a.kf_stride;  // x (64) | y (64) | z (33)
    const float colf = kf[64 + ky] * kf[128 + kz];
    const float invM = a.invM, Mreal = a.Mreal;
    float2 *spec = reinterpret_cast<float2 *>(a.spec) + ((size_t)slot * 2 + fld) * 2 * kMk;
    const int npass = both ? 2 : 1;
    for (int pass = 0; pass < npass; pass++) {
        float2 *sp = spec + (size_t)pass * kMk + c;
        float2 v[64];
#pragma unroll
        for (int x = 0; x < 64; x++) v[x] = ld_shared_gm(sp + (size_t)x * kPlane);
        fft64<-1>(v);  // bin kx in v[perm(kx)]
#pragma unroll
        for (int kx = 0; kx < 64; kx++) {
            const float k2 = __ldg(kf + kx) * colf;
            const float f = pass == 0 ? k2 * invM : (k2 * invM) * (k2 * invM) * Mreal;
            float2 &t = v[perm(kx)];
            t = make_float2(t.x * f, t.y * f);
        }
        fft64_pin<+1>(v);  // x in v[x]
#pragma unroll
        for (int x = 0; x < 64; x++) sp[(size_t)x * kPlane] = v[x];
    }
}

// ---------------------------------------------------------------- mid
// slab x of (slot, fld) by one warp with tile R: inverse slab of the full step
// -> P = E2 qs1; inverse slab of the half step, times E2, forward slab
__device__ __forceinline__ void mid_slab(const PropsArgs<float> &a, int s, int slot, int fld, int x, float *R,
                                         int lane)
{
    const Geo &g = a.g;
    const size_t slab_r = (size_t)x * 4096;
    const float *E = eptr(a, slot, esel(g, fld, s)) + slab_r;
    float2 *specA = reinterpret_cast<float2 *>(a.spec) + ((size_t)slot * 2 + fld) * 2 * kMk;
    float2 *specB = specA + kMk;
    float *P = a.pbuf + ((size_t)slot * 2 + fld) * kM + slab_r;
    const int z = 2 * lane;
    // full step: P = E2 * qs1
    slab_inverse(specB + (size_t)x * kPlane, R, lane);
#pragma unroll 4
    for (int y = 0; y < 64; y++) {
        const float2 c = *reinterpret_cast<const float2 *>(R + y * kRowPitch + z);
        const float2 e = *reinterpret_cast<const float2 *>(E + y * 64 + z);
        *reinterpret_cast<float2 *>(P + y * 64 + z) = make_float2(c.x * (e.x * e.x), c.y * (e.y * e.y));
    }
    // second half step input: E2 * (first half step)
    slab_inverse(specA + (size_t)x * kPlane, R, lane);
#pragma unroll 4
    for (int y = 0; y < 64; y++) {
        float2 *cp = reinterpret_cast<float2 *>(R + y * kRowPitch + z);
        const float2 c = *cp;
        const float2 e = *reinterpret_cast<const float2 *>(E + y * 64 + z);
        *cp = make_float2(c.x * (e.x * e.x), c.y * (e.y * e.y));
    }
    slab_forward(R, specA + (size_t)x * kPlane, lane);
}

// ---------------------------------------------------------------- combine
// mode 0: finishes step s (q(s+1) = Richardson combination, GPU_kernels.h:199-203);
// mode 1: q(s+1) = 1 (Array_set_value, density.h:368-369; called with s = -1);
// mode 2: q(s+1) is taken from the propagator store.
// Then starts step s+1 when s+1 < Ns.
__device__ __forceinline__ void combine_slab(const PropsArgs<float> &a, int s, int mode, int slot, int fld, int x,
                                             float *R, int lane)
{
    const Geo &g = a.g;
    const size_t slab_r = (size_t)x * 4096;
    float2 *specA = reinterpret_cast<float2 *>(a.spec) + ((size_t)slot * 2 + fld) * 2 * kMk;
    float2 *specB = specA + kMk;
    const int sn = s + 1;
    float *qn = a.hist + hoff(g, slot, sn, fld) + slab_r;
    const int z = 2 * lane;
    if (mode == 0) {
        slab_inverse(specA + (size_t)x * kPlane, R, lane);
        const float *E = eptr(a, slot, esel(g, fld, s)) + slab_r;
        const float *P = a.pbuf + ((size_t)slot * 2 + fld) * kM + slab_r;
#pragma unroll 4
        for (int y = 0; y < 64; y++) {
            float2 *cp = reinterpret_cast<float2 *>(R + y * kRowPitch + z);
            const float2 c = *cp;
            const float2 e = *reinterpret_cast<const float2 *>(E + y * 64 + z);
            const float2 p = ld_shared_gm(reinterpret_cast<const float2 *>(P + y * 64 + z));
            const float2 q = make_float2((c.x * e.x * 4.0f - p.x) / 3.0f, (c.y * e.y * 4.0f - p.y) / 3.0f);
            *reinterpret_cast<float2 *>(qn + y * 64 + z) = q;
            *cp = q;
        }
    } else {
        __syncwarp();
#pragma unroll 4
        for (int y = 0; y < 64; y++) {
            float2 q = make_float2(1.0f, 1.0f);
            if (mode == 1)
                *reinterpret_cast<float2 *>(qn + y * 64 + z) = q;
            else
                q = *reinterpret_cast<const float2 *>(qn + y * 64 + z);
            *reinterpret_cast<float2 *>(R + y * kRowPitch + z) = q;
        }
    }
    if (sn >= g.Ns) return;
    const float *En = eptr(a, slot, esel(g, fld, sn)) + slab_r;
    // half step input E4' q'
#pragma unroll 4
    for (int y = 0; y < 64; y++) {
        float2 *cp = reinterpret_cast<float2 *>(R + y * kRowPitch + z);
        const float2 c = *cp;
        const float2 e = *reinterpret_cast<const float2 *>(En + y * 64 + z);
        *cp = make_float2(c.x * e.x, c.y * e.y);
    }
    slab_forward(R, specA + (size_t)x * kPlane, lane);
    // full step input E2' q' (q' re-read from the propagator store: this lane wrote it above)
#pragma unroll 4
    for (int y = 0; y < 64; y++) {
        const float2 q = *reinterpret_cast<const float2 *>(qn + y * 64 + z);
        const float2 e = *reinterpret_cast<const float2 *>(En + y * 64 + z);
        *reinterpret_cast<float2 *>(R + y * kRowPitch + z) = make_float2(q.x * (e.x * e.x), q.y * (e.y * e.y));
    }
    slab_forward(R, specB + (size_t)x * kPlane, lane);
}

__global__ void __launch_bounds__(kPencilThreads) k_pencil_r(PropsArgs<float> a, int both)
{
    const int c = blockIdx.x * kPencilThreads + threadIdx.x;
    if (c < kPlane) pencil_column(a, both, blockIdx.z, blockIdx.y, c);
}

__global__ void __launch_bounds__(32 * kWPB) k_mid_r(PropsArgs<float> a, int s)
{
    extern __shared__ __align__(16) float smem_r[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    mid_slab(a, s, blockIdx.z, blockIdx.y, blockIdx.x * kWPB + warp, smem_r + warp * kTileFloats, lane);
}

__global__ void __launch_bounds__(32 * kWPB) k_combine_r(PropsArgs<float> a, int s, int mode)
{
    extern __shared__ __align__(16) float smem_r[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    combine_slab(a, s, mode, blockIdx.z, blockIdx.y, blockIdx.x * kWPB + warp, smem_r + warp * kTileFloats, lane);
}

// ---------------------------------------------------------------- one launch per contour step
// A persistent kernel runs the whole step s of every slot: CTAs claim work
// items from a counter in a fixed order -- all pencil(both) column blocks,
// then all mid slab quads, all pencil(A) column blocks, all combine slab
// quads, each phase ordered by (slot, field) -- and an item waits only for
// the items of the previous phase of its own (slot, field).  Items are
// claimed in order by running CTAs, so whatever an item waits for has been
// claimed by a CTA that is running or done: no residency assumption is
// needed.  Completion counters are cumulative over the steps of a props
// round (phase p of (slot, field) has n_p (s+1) items done after step s) and
// are zeroed with the claim counters when the round starts.  Every wait is
// bounded (kStepSpin polls); one that gives up records error 3 and ends the
// kernel, so a lost item cannot hang the GPU.  Data another CTA of the same
// launch wrote (spectra, P) is read through L2 (ld_shared_gm).
constexpr int kColBlocks = (kPlane + kPencilThreads - 1) / kPencilThreads;  // 17
constexpr int kSlabQuads = 64 / kWPB;                                       // 16
constexpr uint32_t kStepSpin = 1u << 22;

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__global__ void __launch_bounds__(32 * kWPB) k_step_r(PropsArgs<float> a, int s, int nslots)
{
    extern __shared__ __align__(16) float smem_r[];
    __shared__ int item_sh, ok_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = 2 * nslots;  // (slot, field) groups
    const int per[4] = {kColBlocks, kSlabQuads, kColBlocks, kSlabQuads};
    const int total = G * (2 * kColBlocks + 2 * kSlabQuads);
    int *claim = a.sync + s;           // this step's claim counter
    int *done = a.sync + a.g.Ns;       // [phase][group] completion counters
    for (;;) {
        if (threadIdx.x == 0) item_sh = atomicAdd(claim, 1);
        __syncthreads();
        int it = item_sh;
        if (it >= total) break;
        int phase = 0;
        while (it >= G * per[phase]) {
            it -= G * per[phase];
            phase++;
        }
        const int group = it / per[phase], unit = it - group * per[phase];
        const int slot = group >> 1, fld = group & 1;
        if (phase > 0) {
            if (threadIdx.x == 0) {
                const int need = per[phase - 1] * (s + 1);
                const int *cnt = done + (phase - 1) * G + group;
                uint32_t i = 0;
                while (ld_acquire(cnt) < need && i < kStepSpin) {
                    __nanosleep(32);
                    i++;
                }
                ok_sh = i < kStepSpin;
                if (!ok_sh) *a.err = 3;
            }
            __syncthreads();
            if (!ok_sh) return;
        }
        if (phase == 0 || phase == 2) {
            const int c = unit * kPencilThreads + threadIdx.x;
            if (c < kPlane) pencil_column(a, phase == 0, slot, fld, c);
        } else if (phase == 1) {
            mid_slab(a, s, slot, fld, unit * kWPB + warp, smem_r + warp * kTileFloats, lane);
        } else {
            combine_slab(a, s, 0, slot, fld, unit * kWPB + warp, smem_r + warp * kTileFloats, lane);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + phase * G + group, 1);
        }
    }
}

constexpr int kSlabSmem = kWPB * kTileFloats * (int)sizeof(float);

}  // namespace

bool reg64_applicable(int m0, int m1, int m2) { return m0 == 64 && m1 == 64 && m2 == 64; }

int reg64_set_smem()
{
    cudaError_t e1 = raise_dyn_smem(k_mid_r, kSlabSmem);
    cudaError_t e2 = raise_dyn_smem(k_combine_r, kSlabSmem);
    cudaError_t e3 = raise_dyn_smem(k_step_r, kSlabSmem);
    return (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess) ? 0 : 1;
}

int reg64_sync_ints(int Ns, int nslots) { return Ns + 4 * 2 * nslots; }

int reg64_step_grid()
{
    int dev = 0, sms = 148, per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_r, 32 * kWPB, kSlabSmem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    return sms * per_sm;
}

void reg64_step(const PropsArgs<float> &a, int nslots, int s, int grid, cudaStream_t st)
{
    k_step_r<<<grid, 32 * kWPB, kSlabSmem, st>>>(a, s, nslots);
}

void reg64_combine(const PropsArgs<float> &a, int nslots, int s, int mode, cudaStream_t st)
{
    k_combine_r<<<dim3(64 / kWPB, 2, nslots), 32 * kWPB, kSlabSmem, st>>>(a, s, mode);
}

void reg64_mid(const PropsArgs<float> &a, int nslots, int s, cudaStream_t st)
{
    k_mid_r<<<dim3(64 / kWPB, 2, nslots), 32 * kWPB, kSlabSmem, st>>>(a, s);
}

void reg64_pencil(const PropsArgs<float> &a, int nslots, int both, cudaStream_t st)
{
    k_pencil_r<<<dim3((kPlane + kPencilThreads - 1) / kPencilThreads, 2, nslots), kPencilThreads, 0, st>>>(a, both);
}

}  // namespace scft
