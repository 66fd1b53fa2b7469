// noalloc.cu -- one Richardson contour step that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they need a propagator
// step: a real-time loop that must not stall on the allocator (cudaMalloc
// can synchronise the whole device), or an embedding framework that owns
// every device allocation through its own pool and forbids foreign ones.
// For them, scft_do_step_noalloc runs the same runtime-shaped kernels as
// scft_do_step (k_prepare, k_combine, k_pencil, k_mid) with all of their
// working buffers -- spectra, E tables, the full-step partial, the two
// propagator slices, FFT twiddles, diffusion factors and the error word --
// in one file-scope __device__ array of kNoAllocBytes.  The caller passes
// only its own device buffers for the fields, the input slice and the
// output slice.
//
// Limits and sharing: FP64, M = m0*m1*m2 <= 32768 and every m_i <= 64 with
// prime factors <= 7.  The array lives on every GPU that loads this library
// until the process exits.  All calls share it and it keeps the last call's
// contents, so calls that overlap on the GPU (different streams or threads
// without ordering) race; serialise them.  The call waits for its stream
// before it returns (it reads the kernels' error word).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/scft_b200.h"
#include "kernels.h"

namespace scft {
namespace {

constexpr int kNoAllocMaxM = 32768;
constexpr int kNoAllocMaxAxis = 64;
constexpr int kNoAllocMaxDevices = 64;
// doubles: spectra 8M + pbuf 2M + etab 2M + two propagator slices 4M + tables
constexpr size_t kNoAllocDoubles = 16 * (size_t)kNoAllocMaxM + 9 * kNoAllocMaxAxis + 64;
constexpr size_t kNoAllocBytes = kNoAllocDoubles * sizeof(double);

__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];
static_assert(sizeof(g_noalloc_scratch) == kNoAllocBytes, "scratch size");

// device address of g_noalloc_scratch per device, from cudaGetSymbolAddress;
// each entry is filled once, under its own once-flag, by the first call on
// that device (host threads racing on a first call wait for the winner)
void *g_scratch_addr[kNoAllocMaxDevices];
cudaError_t g_scratch_rc[kNoAllocMaxDevices];
std::once_flag g_scratch_once[kNoAllocMaxDevices];

bool factor7(int n, Plan1D &p)
{
    if (n < 1) return false;
    p.n = n;
    p.nst = 0;
    int rem = n;
    const int pref[] = {8, 4, 2, 3, 5, 7};
    for (int R : pref)
        while (rem % R == 0 && p.nst < kMaxStages) {
            p.radix[p.nst++] = R;
            rem /= R;
        }
    return rem == 1;
}

int threads_needed(const Plan1D &p, int nlines)
{
    int need = 32;
    for (int i = 0; i < p.nst; i++) {
        const int R = p.radix[i];
        const long nb = (long)nlines * (p.n / R);
        const int sl = 16 / R;
        need = (int)std::max<long>(need, (nb + sl - 1) / sl);
    }
    return need;
}

// twiddles exp(-2 pi i t/n) per axis and the per-axis diffusion factors
// exp(-4 pi^2 k^2 ds / (12 D^2)) (setup_k_sq, density.h:79-95)
__global__ void k_noalloc_tables(cplx<double> *tw, double *kfac, int m0, int m1, int m2, double D0, double D1,
                                 double D2, double ds)
{
    const int ns[3] = {m0, m1, m2};
    const double Ds[3] = {D0, D1, D2};
    const double PI = 3.14159265358979323846;
    int off = 0, koff = 0;
    for (int a = 0; a < 3; a++) {
        const int n = ns[a];
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            double sv, cv;
            sincospi(2.0 * t / n, &sv, &cv);
            tw[off + t] = {cv, -sv};
        }
        const int cnt = a == 2 ? n / 2 + 1 : n;
        for (int K = threadIdx.x; K < cnt; K += blockDim.x) {
            const int k = (a == 2) ? K : (K <= n / 2 ? K : K - n);
            const double A = (double)k * k / (Ds[a] * Ds[a]);
            kfac[koff + K] = exp(-4 * PI * PI * A * ds / 12);
        }
        off += n;
        koff += cnt;
    }
}

}  // namespace
}  // namespace scft

using namespace scft;

extern "C" scft_status scft_do_step_noalloc(const int *m, const double *D, int N, double f, const double *w2M,
                                            const double *in2M, double *out2M, int s, void *stream)
{
    if (!m || !D || !w2M || !in2M || !out2M || N < 1 || s < 0 || s >= N) return SCFT_BAD_INPUT;
    if (!(f >= 0.0 && f <= 1.0)) return SCFT_BAD_INPUT;  // as scft_create
    for (int i = 0; i < 3; i++)
        if (m[i] < 1 || m[i] > kNoAllocMaxAxis || !(D[i] > 0)) return SCFT_BAD_INPUT;
    const long Ml = (long)m[0] * m[1] * m[2];
    if (Ml > kNoAllocMaxM) return SCFT_BAD_INPUT;
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.m0 = m[0];
    g.m1 = m[1];
    g.m2 = m[2];
    if (!factor7(g.m0, g.px) || !factor7(g.m1, g.py) || !factor7(g.m2, g.pz)) return SCFT_BAD_INPUT;
    g.mk2 = g.m2 / 2 + 1;
    g.M = (int)Ml;
    g.Mk = g.m0 * g.m1 * g.mk2;
    g.npair = (g.m1 + 1) / 2;
    g.slab_c = g.m1 * g.mk2 + g.m2 + 32;
    const double fr = std::round(N * f) / N;  // scft.cu:1008
    g.Ns = N;
    g.n1 = (int)std::round(N * fr);           // density.h:346
    g.n2 = N - g.n1;
    g.Nh = 0;
    g.tc = 16;
    g.ncol_tiles = (g.m1 * g.mk2 + g.tc - 1) / g.tc;
    PropsLaunch L;
    std::memset(&L, 0, sizeof(L));
    const int st_need = std::max(threads_needed(g.pz, g.npair), threads_needed(g.py, g.mk2));
    const int pt_need = threads_needed(g.px, g.tc);
    if (st_need > 1024 || pt_need > 1024) return SCFT_BAD_INPUT;
    L.slab_threads = std::min(1024, std::max(256, (st_need + 31) / 32 * 32));
    L.pencil_threads = std::min(1024, std::max(128, (pt_need + 31) / 32 * 32));
    L.big = (L.slab_threads > 256 || L.pencil_threads > 256) ? 1 : 0;
    L.slab_smem = (g.slab_c + g.m1 + g.m2) * 16;
    L.pencil_smem = (g.tc * g.m0 + g.m0) * 16 + (g.tc + g.m0) * 8;
    L.ew_blocks = std::max(1, std::min(1024, (g.M + 255) / 256));
    L.red_blocks = 148;
    if (L.slab_smem > 48 * 1024 || L.pencil_smem > 48 * 1024) return SCFT_BAD_INPUT;

    // set-up on first use on this device: the array's device address
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return SCFT_CUDA_ERROR;
    std::call_once(g_scratch_once[dev], [dev] {
        void *p = nullptr;
        g_scratch_rc[dev] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        g_scratch_addr[dev] = p;
    });
    if (g_scratch_rc[dev] != cudaSuccess || !g_scratch_addr[dev]) return SCFT_CUDA_ERROR;
    double *base = static_cast<double *>(g_scratch_addr[dev]);
    const size_t M = g.M;
    int *err = reinterpret_cast<int *>(base);     // first 64 doubles: error word and slot map
    int *slot_rep = err + 1;
    double *spec = base + 64;                     // 2 fields x 2 spectra x Mk complex
    double *pbuf = spec + 8 * M;
    double *etab = pbuf + 2 * M;
    double *hist = etab + 2 * M;                  // slices s and s+1, each [q, q^dagger]
    cplx<double> *tw = reinterpret_cast<cplx<double> *>(hist + 4 * M);
    double *kfac = reinterpret_cast<double *>(tw + 3 * kNoAllocMaxAxis);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // state that must start at zero every call: the error word and the slot map
    if (cudaMemsetAsync(base, 0, 64 * sizeof(double), st) != cudaSuccess) return SCFT_CUDA_ERROR;
    k_noalloc_tables<<<1, 128, 0, st>>>(tw, kfac, g.m0, g.m1, g.m2, D[0], D[1], D[2], 1.0 / N);
    if (cudaMemcpyAsync(hist, in2M, sizeof(double) * 2 * M, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return SCFT_CUDA_ERROR;
    PropsArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.g = g;
    a.slot_rep = slot_rep;  // slot 0 -> replica 0, the caller's fields
    a.W = w2M;
    a.etab = etab;
    a.hist = hist;
    a.spec = reinterpret_cast<cplx<double> *>(spec);
    a.pbuf = pbuf;
    a.tw = tw;
    a.kfac = kfac;
    a.invM = 1.0 / g.M;
    a.Mreal = (double)g.M;
    a.err = err;
    // E tables of the whole chain (ds = 1/N), then a one-step chain segment
    // whose store holds only slices s and s+1: its geometry counts contour
    // steps from s, so n1 and n2 shrink by s and each step still picks the E
    // table of its absolute index
    // the runtime-shaped kernels' shared-memory limits are raised to this
    // grid's need if they are below it (host-side attribute, no allocation)
    if (set_props_smem<double>(L) != 0) return SCFT_CUDA_ERROR;
    launch_prepare<double>(a, L, st);
    PropsArgs<double> seg = a;
    seg.g.Ns = 1;
    seg.g.n1 = g.n1 - s;
    seg.g.n2 = g.n2 - s;
    launch_chain<double>(seg, L, 2, st);
    if (cudaGetLastError() != cudaSuccess) return SCFT_CUDA_ERROR;
    if (cudaMemcpyAsync(out2M, hist + 2 * M, sizeof(double) * 2 * M, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return SCFT_CUDA_ERROR;
    int e = 0;
    if (cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SCFT_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SCFT_CUDA_ERROR;
    return e ? (e == 3 ? SCFT_TIMEOUT : SCFT_CUDA_ERROR) : SCFT_OK;
}
