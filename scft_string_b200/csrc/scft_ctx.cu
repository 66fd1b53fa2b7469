// scft_ctx.cu -- host side of the C ABI (include/scft_b200.h): the device
// context and the solver control flow of solve_field0 / solve_field / FreeE
// (scft.cu:516-853) driving the sm_100a kernels.
//
// The heavy work (propagators, densities, residuals, spline, projection,
// mixing) runs on the device; the host keeps only the per-replica scalars
// the reference keeps (errors, mixing parameters, arc-length knots) and
// evaluates them in FP64 in the reference's order.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/scft_b200.h"
#include "kernels.h"

using namespace scft;

// schedules scft_autotune_ex times: slot groups (1, 2, 4) x tile width x launch form
constexpr int kTuneCandidates = 12;

namespace {

constexpr int kRedBlocks = 148;  // reduction grid: one block per SM

bool factor(int n, Plan1D &p)
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
    // a radix-2 stage after radix 8/4 stages is better merged: 8*2 -> 4*4
    return rem == 1;
}

int slots_for(int R) { return 16 / R; }

int threads_for(const Plan1D &p, int nlines)
{
    int need = 32;
    for (int i = 0; i < p.nst; i++) {
        const int R = p.radix[i];
        const long nb = (long)nlines * (p.n / R);
        const int t = (int)((nb + slots_for(R) - 1) / slots_for(R));
        need = std::max(need, t);
    }
    return need;
}

int round32(int v) { return (v + 31) / 32 * 32; }

}  // namespace

struct scft_ctx {
    scft_problem p;
    Geo g;
    int M, Mk, strn, nrep_alloc, nslots, prec;
    double f;  // rounded A fraction
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr, join = nullptr;
    int ngroups = 2;
    cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
    PropsLaunch L;
    std::string lasterr;

    // device memory
    double *W = nullptr, *conc = nullptr, *DEV = nullptr, *dWda = nullptr, *rs = nullptr;
    double *partials = nullptr, *redout = nullptr;
    int npart_stride = 0, nred_rows = 0;
    int *rep_dev = nullptr, *err = nullptr;
    int *sync = nullptr;     // counters of the persistent step kernel, one block per slot group
    int sync_stride = 0;
    bool persist_ok = false; // a persistent step launch exists for this context
    std::vector<double> Dr;  // box of every replica (3 per replica); p.D is the last common box
    int kf_n = 0;            // diffusion factors per replica (m0 + m1 + mk2)
    void *jtab = nullptr;  // junction-step E table per slot (continuous A fraction)
    void *etab = nullptr, *hist = nullptr, *spec = nullptr, *pbuf = nullptr, *tw = nullptr,
         *kfac = nullptr;
    SplineKnots *knots = nullptr;
    CUtensorMap tmap;       // spectra as a 2-D array for the x-pencil tiles
    CUtensorMap tmap_wide;  // the same with tiles of twice the width
    // adjoint (stress) scratch, allocated on first use
    void *st_S4 = nullptr, *st_S2 = nullptr, *st_S4p = nullptr;
    double *and_X = nullptr, *and_D = nullptr;  // Anderson histories
    int and_H = 0;
    double *st_part = nullptr, *st_out = nullptr;
    void *jd_rbuf = nullptr;  // junction derivative: six real work arrays
    bool nostore = false;    // props from checkpoints, no full propagator store
    int ckK = 0;             // checkpoint interval of the nostore props
    void *ck_mem = nullptr;  // checkpointed adjoint: checkpoints, two segments, Q slices
    size_t ck_bytes = 0;
    int rt_slab_threads = 0, rt_slab_smem = 0, rt_pencil_threads = 0, rt_pencil_smem = 0;

    // one captured CUDA graph per (chunk offset, batch size) of a props round
    std::vector<cudaGraphExec_t> graphs;
    bool use_graphs = true;

    // host state
    std::vector<int> doiis;
    std::vector<int> slot_of;   // replica -> slot of its last props (-1 unknown)
    std::vector<double> rs_h;   // [rep][kRsStride]
    std::vector<double> red_h;
    scft_stats stats{};
    bool timing_pending = false;

    // solve_field loop state (scft.cu:561-590)
    struct {
        bool active = false;
        int doii = -1, maxIter = 0, k = 0;
        double errTol = 1e-3, lambda = 0.05, err = 1, errt = 1, FE = 0;
        int dospring = 1, doredist = 0, doperp = 0;
        bool skip_freee = false;  // cell relaxation runs the loop without FreeE
        std::vector<double> x, xref, alf, errs, errs3, FEs, FEs0, FEs1, phctot;
        std::vector<int> steps;
    } sf;
};

namespace {

scft_status cuda_fail(scft_ctx *c, cudaError_t e, const char *what)
{
    c->lasterr = std::string(what) + ": " + cudaGetErrorString(e);
    return SCFT_CUDA_ERROR;
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call);   \
    } while (0)

template <typename T>
PropsArgs<T> props_args(scft_ctx *ctx, const int *slot_rep)
{
    PropsArgs<T> a;
    a.g = ctx->g;
    a.slot_rep = slot_rep;
    a.W = ctx->W;
    a.conc = ctx->conc;
    a.rs = ctx->rs;
    a.etab = (T *)ctx->etab;
    a.hist = (T *)ctx->hist;
    a.spec = (cplx<T> *)ctx->spec;
    a.pbuf = (T *)ctx->pbuf;
    a.tw = (const cplx<T> *)ctx->tw;
    a.kfac = (const T *)ctx->kfac;
    a.kf_stride = ctx->kf_n;
    a.partials = ctx->partials;
    a.npart_stride = ctx->npart_stride;
    a.invM = (T)(1.0 / ctx->M);
    a.Mreal = (T)ctx->M;
    a.chi = ctx->p.chi;
    a.phic = ctx->p.phidb;
    a.alpha = ctx->p.alpha;
    a.ens = ctx->p.ens;
    a.err = ctx->err;
    a.sync = ctx->sync;
    a.slot0 = 0;
    a.jtab = (T *)ctx->jtab;
    return a;
}

// the same arguments for the slots [s0, s0 + n) of a round: every per-slot
// base pointer moves by s0 slots
template <typename T>
PropsArgs<T> props_args_from(scft_ctx *ctx, const int *slot_rep, int s0, int lane = 0)
{
    PropsArgs<T> a = props_args<T>(ctx, slot_rep + s0);
    const size_t M = ctx->M, Mk = ctx->Mk;
    a.etab += (size_t)s0 * 2 * M;
    a.hist += (size_t)s0 * (ctx->g.Ns + 1) * 2 * M;
    a.spec += (size_t)s0 * 2 * 2 * Mk;
    a.pbuf += (size_t)s0 * 2 * M;
    a.partials += (size_t)s0 * ctx->npart_stride;
    a.slot0 = s0;
    if (a.jtab) a.jtab += (size_t)s0 * M;
    if (a.sync && lane) a.sync += ctx->sync_stride;  // counters of the groups on the second stream
    return a;
}

FieldArgs field_args(scft_ctx *ctx, const int *rep_list)
{
    FieldArgs a;
    a.M = ctx->M;
    a.strn = ctx->strn;
    a.rep_list = rep_list;
    a.W = ctx->W;
    a.conc = ctx->conc;
    a.DEV = ctx->DEV;
    a.dWda = ctx->dWda;
    a.partials = ctx->partials;
    a.chi = ctx->p.chi;
    return a;
}

// the kernels' error word: 1, 2 launch geometry (a host bug), 3 a bounded
// bulk-copy wait gave up (tma.cuh).  It is cleared once reported, so the
// context stays usable.
scft_status check_device_err(scft_ctx *ctx)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, ctx->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (e == 0) return SCFT_OK;
    CK(cudaMemsetAsync(ctx->err, 0, sizeof(int), ctx->st));
    if (e == 3) {
        ctx->lasterr = "a bounded device wait for a bulk copy gave up";
        return SCFT_TIMEOUT;
    }
    ctx->lasterr = "device kernel reported a launch-geometry error " + std::to_string(e);
    return SCFT_CUDA_ERROR;
}

// uploads a replica list to the device (pageable copy: staged before return)
scft_status upload_list(scft_ctx *ctx, const std::vector<int> &reps)
{
    CK(cudaMemcpyAsync(ctx->rep_dev, reps.data(), sizeof(int) * reps.size(), cudaMemcpyHostToDevice,
                       ctx->st));
    return SCFT_OK;
}

scft_status props_ckpt_impl(scft_ctx *ctx, int ii, int K, double *lnQ_out, double *phis_out, double *bytes_out);

// Slot groups of a batch of nb replicas: the configured count, halved while a
// group of more than two would get fewer than 4 replicas (a launch of 2 or 3
// replicas leaves most SMs idle: the W+ relaxation runs many such partial
// batches), and 1 when there are fewer than 2 replicas per group.
int effective_groups(int ngroups, int nb)
{
    int ng = ngroups;
    while (ng > 2 && nb < 4 * ng) ng /= 2;
    return (ng > 1 && nb >= 2 * ng) ? ng : 1;
}

// density::props for a list of replicas; scalars land in ctx->rs_h.  Without a
// full store (nostore) each replica runs from checkpoints.
scft_status props_list(scft_ctx *ctx, const std::vector<int> &reps)
{
    if (reps.empty()) return SCFT_OK;
    if (ctx->nostore) {
        CK(cudaEventRecord(ctx->ev0, ctx->st));
        for (int r : reps) {
            scft_status s = props_ckpt_impl(ctx, r, ctx->ckK, nullptr, nullptr, nullptr);
            if (s != SCFT_OK) return s;
            ctx->slot_of[r] = -1;
        }
        CK(cudaEventRecord(ctx->ev1, ctx->st));
        CK(cudaMemcpyAsync(ctx->rs_h.data(), ctx->rs, sizeof(double) * ctx->rs_h.size(), cudaMemcpyDeviceToHost,
                           ctx->st));
        scft_status s = check_device_err(ctx);
        if (s != SCFT_OK) return s;
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        ctx->stats.props_seconds += ms * 1e-3;
        ctx->stats.props_calls += (long long)reps.size();
        ctx->stats.contour_steps += (long long)reps.size() * ctx->g.Ns;
        return SCFT_OK;
    }
    scft_status s = upload_list(ctx, reps);
    if (s != SCFT_OK) return s;
    CK(cudaEventRecord(ctx->ev0, ctx->st));
    int launches = 0;
    for (size_t c0 = 0; c0 < reps.size(); c0 += ctx->nslots) {
        const int nb = (int)std::min<size_t>(ctx->nslots, reps.size() - c0);
        // groups of slots run as independent chains on two streams, so the
        // last wave of one group's launch overlaps the other group's work;
        // with more than two groups each stream runs its groups one after
        // another (fewer spectra live at once)
        const int ng = effective_groups(ctx->ngroups, nb);
        auto launch = [&]() {
            int n = 0;
            if (ng > 1) {
                cudaEventRecord(ctx->fork, ctx->st);
                cudaStreamWaitEvent(ctx->st2, ctx->fork, 0);
            }
            for (int gi = 0; gi < ng; gi++) {
                const int s0 = nb * gi / ng, s1 = nb * (gi + 1) / ng;
                cudaStream_t sg = (gi % 2 == 0) ? ctx->st : ctx->st2;
                if (ctx->prec == SCFT_FP32)
                    n += launch_props<float>(props_args_from<float>(ctx, ctx->rep_dev + c0, s0, gi % 2), ctx->L,
                                             s1 - s0, sg);
                else
                    n += launch_props<double>(props_args_from<double>(ctx, ctx->rep_dev + c0, s0, gi % 2), ctx->L,
                                              s1 - s0, sg);
            }
            if (ng > 1) {
                cudaEventRecord(ctx->join, ctx->st2);
                cudaStreamWaitEvent(ctx->st, ctx->join, 0);
            }
            return n;
        };
        const size_t key = (c0 <= (size_t)ctx->nrep_alloc) ? c0 * (ctx->nslots + 1) + nb : (size_t)-1;
        if (ctx->use_graphs && key < ctx->graphs.size()) {
            // the whole props round (4 Ns + 6 launches) replays as one graph
            if (!ctx->graphs[key]) {
                cudaGraph_t gr;
                CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
                launch();
                CK(cudaStreamEndCapture(ctx->st, &gr));
                cudaError_t e = cudaGraphInstantiate(&ctx->graphs[key], gr, 0);
                cudaGraphDestroy(gr);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
            }
            CK(cudaGraphLaunch(ctx->graphs[key], ctx->st));
            launches += ((ctx->L.persist ? 1 : 4) * ctx->g.Ns + 6) * ng;
        } else {
            launches += launch();
        }
        for (int j = 0; j < nb; j++) {
            for (auto &so : ctx->slot_of)
                if (so == j) so = -1;
            ctx->slot_of[reps[c0 + j]] = j;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->st));
    CK(cudaMemcpyAsync(ctx->rs_h.data(), ctx->rs, sizeof(double) * ctx->rs_h.size(),
                       cudaMemcpyDeviceToHost, ctx->st));
    s = check_device_err(ctx);
    if (s != SCFT_OK) return s;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->stats.props_seconds += ms * 1e-3;
    ctx->stats.props_calls += (long long)reps.size();
    ctx->stats.contour_steps += (long long)reps.size() * ctx->g.Ns;
    ctx->stats.kernel_launches += launches;
    return SCFT_OK;
}

double rsv(const scft_ctx *ctx, int rep, int k) { return ctx->rs_h[(size_t)rep * kRsStride + k]; }

// final reduction of `rows` partial rows into ctx->red_h
scft_status reduce_rows(scft_ctx *ctx, int rows, int nblk)
{
    launch_reduce_final(ctx->partials, rows, nblk, ctx->redout, ctx->st);
    ctx->stats.kernel_launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->red_h.data(), ctx->redout, sizeof(double) * rows,
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCFT_OK;
}

// solve_field0 (scft.cu:516-554) over a set of replicas.  Replicas are
// independent, so the batched form (all together, props per round) gives the
// same per-replica results as the reference's one-after-another order.
scft_status field0_set(scft_ctx *ctx, const std::vector<int> &set, int maxIter, double errTol,
                       std::vector<int> &kout)
{
    struct St {
        double lam = 0.05, err = 1.0, errt = 1.0;
        int k = 1;
    };
    const double dlam1 = 1.09, dlam2 = 1.10;
    std::vector<St> stt(ctx->nrep_alloc);
    kout.assign(ctx->nrep_alloc, 0);
    std::vector<std::vector<int>> groups;
    if (ctx->p.batched)
        groups.push_back(set);
    else
        for (int ii : set) groups.push_back({ii});
    for (auto &grp : groups) {
        std::vector<int> cur;
        for (int ii : grp)
            if (stt[ii].k < maxIter && stt[ii].err > errTol) cur.push_back(ii);
        while (!cur.empty()) {
            scft_status s = props_list(ctx, cur);
            if (s != SCFT_OK) return s;
            std::vector<double> lam(cur.size());
            for (size_t j = 0; j < cur.size(); j++) {
                St &q = stt[cur[j]];
                q.err = std::pow(rsv(ctx, cur[j], kRsDev2) / ctx->M, 0.5);
                if (!(q.err == q.err)) {
                    ctx->lasterr = "solve_field0: residual is NaN for replica " + std::to_string(cur[j]);
                    return SCFT_NAN_DETECTED;
                }
                lam[j] = q.lam;
            }
            s = upload_list(ctx, cur);
            if (s != SCFT_OK) return s;
            launch_mix0(field_args(ctx, ctx->rep_dev), (int)cur.size(), lam.data(), ctx->st);
            ctx->stats.kernel_launches += 1;
            CK(cudaGetLastError());
            std::vector<int> nxt;
            for (int ii : cur) {
                St &q = stt[ii];
                if (q.err < q.errt)
                    q.lam = std::min(0.1, q.lam * dlam1);
                else
                    q.lam = std::max(0.005, q.lam / dlam2);
                q.errt = q.err;
                q.k++;
                if (q.k < maxIter && q.err > errTol) nxt.push_back(ii);
            }
            cur.swap(nxt);
        }
    }
    for (int ii : set) kout[ii] = stt[ii].k;
    return SCFT_OK;
}

// EDist between consecutive replicas (scft.cu:351-355)
scft_status edists(scft_ctx *ctx, std::vector<double> &del)
{
    const int n = ctx->strn - 1;
    del.assign(std::max(n, 0), 0.0);
    if (n <= 0) return SCFT_OK;
    launch_edist(field_args(ctx, ctx->rep_dev), kRedBlocks, ctx->st);
    ctx->stats.kernel_launches += 1;
    scft_status s = reduce_rows(ctx, n, kRedBlocks);
    if (s != SCFT_OK) return s;
    for (int i = 0; i < n; i++) del[i] = std::sqrt(ctx->red_h[i]);
    return SCFT_OK;
}

// arc-length knots x (scft.cu:612-621, 725-736)
scft_status arc_length(scft_ctx *ctx, std::vector<double> &x)
{
    std::vector<double> del;
    scft_status s = edists(ctx, del);
    if (s != SCFT_OK) return s;
    const int strn = ctx->strn;
    double Delsum = 0;
    for (int ii = 0; ii < strn - 1; ii++) Delsum += del[ii];
    for (int ii = 0; ii < strn - 1; ii++) del[ii] /= Delsum;
    x.assign(strn, 0.0);
    x[0] = 0;
    x[strn - 1] = 1;
    for (int ii = 1; ii < strn - 1; ii++) x[ii] = x[ii - 1] + del[ii - 1];
    return SCFT_OK;
}

int interval(const std::vector<double> &x, double xx)
{
    int nm = 0;
    for (size_t i = 0; i < x.size(); ++i) {
        if (x[i] < xx)
            nm = (int)i;
        else
            break;
    }
    return nm;
}

// knot-only parts of cubefit_chunk_g (GPU_kernels.h:253-267) and the interval
// searches of eval_spline_*_chunk_g (GPU_kernels.h:292-297, 314-319)
scft_status upload_knots(scft_ctx *ctx, const std::vector<double> &x, const std::vector<double> *xref,
                         const int *doiis)
{
    SplineKnots K;
    std::memset(&K, 0, sizeof(K));
    const int strn = ctx->strn, n = strn - 1;
    K.strn = strn;
    for (int i = 0; i <= n - 1; ++i) K.h[i] = x[i + 1] - x[i];
    K.l[0] = 1.0;
    K.u[0] = 0.0;
    for (int i = 1; i <= n - 1; ++i) {
        K.l[i] = 2.0 * (x[i + 1] - x[i - 1]) - K.h[i - 1] * K.u[i - 1];
        K.u[i] = K.h[i] / K.l[i];
    }
    if (n >= 0) K.l[n] = 1.0;
    for (int ev = 0; ev < strn; ev++) {
        K.nm_d[ev] = interval(x, x[ev]);
        K.dx_d[ev] = x[ev] - x[K.nm_d[ev]];
        if (xref) {
            K.nm_v[ev] = interval(x, (*xref)[ev]);
            K.dx_v[ev] = (*xref)[ev] - x[K.nm_v[ev]];
        }
        K.doiis[ev] = doiis[ev];
    }
    CK(cudaMemcpyAsync(ctx->knots, &K, sizeof(K), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));  // K lives on this stack frame
    return SCFT_OK;
}

// FreeE, scft.cu:812-853 (single process: every replica is evaluated)
scft_status free_energy(scft_ctx *ctx, double *FEout)
{
    auto &S = ctx->sf;
    const int strn = ctx->strn;
    std::vector<int> set;
    for (int ii = 0; ii < strn; ii++)
        if (ctx->doiis[ii] == 1 || ii == 0 || ii == strn - 1) set.push_back(ii);
    std::vector<int> k0;
    scft_status s = field0_set(ctx, set, 100, 1e-4, k0);
    if (s != SCFT_OK) return s;
    if (ctx->p.batched) {
        s = props_list(ctx, set);
        if (s != SCFT_OK) return s;
    }
    // plain mode: props of each replica right after its own W+ solve
    std::vector<double> lnQ(strn, 0.0);
    if (!ctx->p.batched) {
        for (int ii : set) {
            s = props_list(ctx, {ii});
            if (s != SCFT_OK) return s;
            lnQ[ii] = rsv(ctx, ii, kRsLnQ);
        }
    } else {
        for (int ii : set) lnQ[ii] = rsv(ctx, ii, kRsLnQ);
    }
    s = upload_list(ctx, set);
    if (s != SCFT_OK) return s;
    launch_freee(field_args(ctx, ctx->rep_dev), (int)set.size(), ctx->f, kRedBlocks, ctx->st);
    ctx->stats.kernel_launches += 1;
    s = reduce_rows(ctx, 2 * (int)set.size(), kRedBlocks);
    if (s != SCFT_OK) return s;
    for (size_t j = 0; j < set.size(); j++) {
        const int ii = set[j];
        S.FEs0[ii] = -lnQ[ii];
        S.FEs1[ii] = ctx->red_h[2 * j];
        S.phctot[ii] = ctx->red_h[2 * j + 1];
        S.FEs[ii] = S.FEs0[ii] + S.FEs1[ii];
    }
    std::vector<double> del;
    s = edists(ctx, del);
    if (s != SCFT_OK) return s;
    S.alf[0] = 0;
    for (int ii = 1; ii < strn; ii++) S.alf[ii] = S.alf[ii - 1] + del[ii - 1];
    double FE = 0;
    for (int ii = 0; ii < strn; ii++) FE += S.FEs[ii];
    if (FEout) *FEout = FE;
    return SCFT_OK;
}

template <typename T>
void upload_tables(scft_ctx *ctx, std::vector<unsigned char> &twb, std::vector<unsigned char> &kfb,
                   const double *Dbox = nullptr)
{
    const double *Dx = Dbox ? Dbox : ctx->p.D;
    const Geo &g = ctx->g;
    const double PI = 3.14159265358979323846264338327950288;
    const int ns[3] = {g.m0, g.m1, g.m2};
    std::vector<cplx<T>> tw;
    for (int a = 0; a < 3; a++)
        for (int t = 0; t < ns[a]; t++) {
            const double ang = 2.0 * PI * (double)t / (double)ns[a];
            tw.push_back({(T)std::cos(ang), (T)(-std::sin(ang))});
        }
    // diffusion factor per axis: exp(-4 pi^2 k^2 ds / (12 D^2)) with k in
    // [-(m-1)/2, m/2] (setup_k_sq, density.h:79-95); the last axis is halved
    const double ds = 1.0 / g.Ns;
    std::vector<T> kf;
    for (int a = 0; a < 3; a++) {
        const int m = ns[a];
        const int cnt = a == 2 ? g.mk2 : m;
        for (int K = 0; K < cnt; K++) {
            const int k = (a == 2) ? K : (K <= m / 2 ? K : K - m);
            const double A = (double)k * k / (Dx[a] * Dx[a]);
            kf.push_back((T)std::exp(-4 * PI * PI * A * ds / 12));
        }
    }
    twb.assign((unsigned char *)tw.data(), (unsigned char *)(tw.data() + tw.size()));
    kfb.assign((unsigned char *)kf.data(), (unsigned char *)(kf.data() + kf.size()));
}

template <typename T>
size_t elem() { return sizeof(T); }

}  // namespace

extern "C" {

const char *scft_status_string(scft_status s)
{
    switch (s) {
        case SCFT_OK: return "ok";
        case SCFT_CUDA_ERROR: return "CUDA error";
        case SCFT_NAN_DETECTED: return "NaN detected";
        case SCFT_BAD_INPUT: return "bad input";
        case SCFT_TIMEOUT: return "timeout";
        case SCFT_OUT_OF_MEMORY: return "out of memory";
        case SCFT_UNSUPPORTED: return "unsupported device";
    }
    return "unknown";
}

const char *scft_last_error(const scft_ctx *ctx) { return ctx ? ctx->lasterr.c_str() : "no context"; }

void scft_destroy(scft_ctx *ctx)
{
    if (!ctx) return;
    void *ptrs[] = {ctx->W, ctx->conc, ctx->DEV, ctx->dWda, ctx->rs, ctx->partials, ctx->redout,
                    ctx->rep_dev, ctx->err, ctx->etab, ctx->hist, ctx->spec, ctx->pbuf, ctx->tw,
                    ctx->kfac, ctx->knots, ctx->st_S4, ctx->st_S2, ctx->st_S4p, ctx->st_part,
                    ctx->st_out, ctx->and_X, ctx->and_D, ctx->ck_mem, ctx->jtab, ctx->jd_rbuf, ctx->sync};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (auto &e : ctx->tev)
        if (e) cudaEventDestroy(e);
    for (auto &g : ctx->graphs)
        if (g) cudaGraphExecDestroy(g);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->st2) cudaStreamDestroy(ctx->st2);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

scft_status scft_create(const scft_problem *p, scft_ctx **out)
{
    if (!p || !out) return SCFT_BAD_INPUT;
    *out = nullptr;
    if (p->strn < 1 || p->strn > kMaxStrn || p->N < 1 || (p->ens != 1 && p->ens != 2) ||
        (p->precision != SCFT_FP32 && p->precision != SCFT_FP64) || p->alpha < 0)
        return SCFT_BAD_INPUT;
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.m0 = p->m[0];
    g.m1 = p->m[1];
    g.m2 = p->m[2];
    if (!factor(g.m0, g.px) || !factor(g.m1, g.py) || !factor(g.m2, g.pz)) return SCFT_BAD_INPUT;
    g.mk2 = g.m2 / 2 + 1;
    if (g.mk2 > 32 * kPairLanes) return SCFT_BAD_INPUT;
    g.M = g.m0 * g.m1 * g.m2;
    g.Mk = g.m0 * g.m1 * g.mk2;
    g.npair = (g.m1 + 1) / 2;
    g.slab_c = g.m1 * g.mk2 + g.m2 + 32;
    if (!(p->f >= 0 && p->f <= 1) || p->N < 1) return SCFT_BAD_INPUT;
    const double f = p->fcont ? p->f : std::round(p->N * p->f) / p->N;  // scft.cu:1008
    g.Ns = p->N;
    g.n1 = p->fcont ? (int)std::floor(g.Ns * f) : (int)std::round(g.Ns * f);  // density.h:346
    g.n2 = g.Ns - g.n1;
    g.Nh = (int)(p->alpha * g.Ns);
    g.jon = 0;
    g.jq = g.jqd = -1;
    g.theta = 0;
    if (g.n1 < 0 || g.n1 > g.Ns || g.Nh > g.Ns) return SCFT_BAD_INPUT;
    if (p->fcont) {
        // junction inside q's step n1 = q^dagger's step N-1-n1; the homopolymer
        // (q^dagger's first Nh steps) must stay in the pure B block
        if (g.n1 >= g.Ns || g.Nh > g.n2 - 1) return SCFT_BAD_INPUT;
        g.jon = 1;
        g.jq = g.n1;
        g.jqd = g.n2 - 1;
        g.theta = g.Ns * f - g.n1;
    }

    int dev = p->device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return SCFT_UNSUPPORTED;
    if (prop.major != 10) return SCFT_UNSUPPORTED;
    if (cudaSetDevice(dev) != cudaSuccess) return SCFT_UNSUPPORTED;

    scft_ctx *ctx = new scft_ctx();
    ctx->p = *p;
    ctx->f = f;
    ctx->prec = p->precision;
    ctx->strn = p->strn;
    ctx->M = g.M;
    ctx->Mk = g.Mk;
    ctx->nrep_alloc = p->strn + 1;  // + one scratch replica for scft_props_host
    ctx->nostore = p->nostore != 0;
    ctx->ckK = p->ckpt_K > 0 ? p->ckpt_K : (int)std::ceil(std::sqrt((double)p->N));
    ctx->nslots = (p->batched && !ctx->nostore) ? p->strn : 1;
    const size_t T = p->precision == SCFT_FP32 ? 4 : 8;

    // launch geometry
    g.tc = T == 4 ? 32 : 16;
    g.ncol_tiles = (g.m1 * g.mk2 + g.tc - 1) / g.tc;
    PropsLaunch &L = ctx->L;
    L.slab_threads = std::min(1024, std::max(256, round32(std::max(threads_for(g.pz, g.npair),
                                                                      threads_for(g.py, g.mk2)))));
    L.pencil_threads = std::min(1024, std::max(128, round32(threads_for(g.px, g.tc))));
    L.big = (L.slab_threads > 256 || L.pencil_threads > 256) ? 1 : 0;
    const int rt_slab_threads = L.slab_threads, rt_pencil_threads = L.pencil_threads;
    L.fixed = fixed_shape_id(g.m0, g.m1, g.m2);
    if (L.fixed) L.slab_threads = L.pencil_threads = fixed_shape_threads(L.fixed);
    // 64^3 FP32: the register-resident step kernels (reg64.cu) with SCFT_REG64=1;
    // the shared-memory kernels otherwise (measured faster on a B200)
    L.reg = 0;
    if (const char *ev = getenv("SCFT_REG64"))
        L.reg = (ev[0] == '1' && T == 4 && reg64_applicable(g.m0, g.m1, g.m2)) ? 1 : 0;
    L.pf = 0;
    if (L.fixed) {
        pf_smem_bytes(L.fixed, T == 4, L.mid_pf_smem, L.combine_pf_smem);
        L.pf = (std::max(L.mid_pf_smem, L.combine_pf_smem) <= (int)prop.sharedMemPerBlockOptin) ? 1 : 0;
        if (const char *ev = getenv("SCFT_NO_PREFETCH")) L.pf = ev[0] == '1' ? 0 : L.pf;
    }
    if (threads_for(g.pz, g.npair) > 1024 || threads_for(g.py, g.mk2) > 1024 ||
        threads_for(g.px, g.tc) > 1024) {
        delete ctx;
        return SCFT_BAD_INPUT;
    }
    L.slab_smem = (int)((g.slab_c + g.m1 + g.m2) * 2 * T);
    L.pencil_smem = (int)((g.tc * g.m0 + g.m0) * 2 * T + (g.tc + g.m0) * T);
    L.ew_blocks = std::max(1, std::min(1024, (g.M + 255) / 256));
    L.red_blocks = kRedBlocks;
    if (L.slab_smem > (int)prop.sharedMemPerBlockOptin || L.pencil_smem > (int)prop.sharedMemPerBlockOptin) {
        delete ctx;
        return SCFT_BAD_INPUT;
    }
    ctx->g = g;
    ctx->rt_slab_threads = rt_slab_threads;
    ctx->rt_pencil_threads = rt_pencil_threads;
    ctx->rt_slab_smem = L.slab_smem;
    ctx->rt_pencil_smem = (int)((2 * g.tc * g.m0 + g.m0) * 2 * T);
    scft_status rc = SCFT_OK;
    auto fail = [&](cudaError_t e, const char *what) {
        ctx->lasterr = std::string(what) + ": " + cudaGetErrorString(e);
        rc = (e == cudaErrorMemoryAllocation) ? SCFT_OUT_OF_MEMORY : SCFT_CUDA_ERROR;
    };
#define CKC(call)                      \
    do {                               \
        cudaError_t _e = (call);       \
        if (_e != cudaSuccess) {       \
            fail(_e, #call);           \
            goto done;                 \
        }                              \
    } while (0)
    {
        const size_t M = g.M, R = ctx->nrep_alloc, S = ctx->nslots;
        std::vector<unsigned char> twb, kfb;
        if (T == 4)
            upload_tables<float>(ctx, twb, kfb);
        else
            upload_tables<double>(ctx, twb, kfb);
        ctx->npart_stride = 6 * kRedBlocks;
        ctx->nred_rows = 2 * kMaxStrn + 8;
        CKC(cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking));
        CKC(cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking));
        CKC(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming));
        if (const char *ev = getenv("SCFT_GROUPS")) ctx->ngroups = std::max(1, std::min(8, atoi(ev)));
        CKC(cudaEventCreate(&ctx->ev0));
        CKC(cudaEventCreate(&ctx->ev1));
        for (auto &e : ctx->tev) CKC(cudaEventCreate(&e));
        CKC(cudaMalloc(&ctx->W, sizeof(double) * 2 * M * R));
        CKC(cudaMalloc(&ctx->conc, sizeof(double) * 4 * M * R));
        CKC(cudaMalloc(&ctx->DEV, sizeof(double) * 2 * M * R));
        CKC(cudaMalloc(&ctx->dWda, sizeof(double) * M * R));
        CKC(cudaMalloc(&ctx->rs, sizeof(double) * kRsStride * R));
        CKC(cudaMalloc(&ctx->partials,
                       sizeof(double) * std::max<size_t>(ctx->npart_stride * S, (size_t)ctx->nred_rows * kRedBlocks)));
        CKC(cudaMalloc(&ctx->redout, sizeof(double) * ctx->nred_rows));
        CKC(cudaMalloc(&ctx->rep_dev, sizeof(int) * (R + 1)));
        CKC(cudaMalloc(&ctx->err, sizeof(int)));
        CKC(cudaMalloc(&ctx->etab, T * 2 * M * S));
        if (g.jon) CKC(cudaMalloc(&ctx->jtab, T * M * S));
        // the full propagator store (2 slices per step and slot); a stub without it
        CKC(cudaMalloc(&ctx->hist, ctx->nostore ? T * 2 * M : T * 2 * M * (size_t)(g.Ns + 1) * S));
        CKC(cudaMalloc(&ctx->spec, T * 2 * 4 * (size_t)g.Mk * S));
        CKC(cudaMalloc(&ctx->pbuf, T * 2 * M * S));
        if (L.reg || L.fixed) {  // counters of the persistent step launch
            ctx->sync_stride = reg64_sync_ints(g.Ns, (int)S);
            CKC(cudaMalloc(&ctx->sync, sizeof(int) * 2 * (size_t)ctx->sync_stride));
        }
        CKC(cudaMalloc(&ctx->tw, twb.size()));
        // one block of diffusion factors per replica (every replica may own its box)
        ctx->kf_n = g.m0 + g.m1 + g.mk2;
        ctx->Dr.assign(3 * R, 0.0);
        for (size_t r = 0; r < R; r++)
            for (int i = 0; i < 3; i++) ctx->Dr[3 * r + i] = p->D[i];
        CKC(cudaMalloc(&ctx->kfac, kfb.size() * R));
        CKC(cudaMalloc(&ctx->knots, sizeof(SplineKnots)));
        CKC(cudaMemcpy(ctx->tw, twb.data(), twb.size(), cudaMemcpyHostToDevice));
        for (size_t r = 0; r < R; r++)
            CKC(cudaMemcpy((unsigned char *)ctx->kfac + r * kfb.size(), kfb.data(), kfb.size(),
                           cudaMemcpyHostToDevice));
        CKC(cudaMemset(ctx->W, 0, sizeof(double) * 2 * M * R));
        CKC(cudaMemset(ctx->conc, 0, sizeof(double) * 4 * M * R));
        CKC(cudaMemset(ctx->DEV, 0, sizeof(double) * 2 * M * R));
        CKC(cudaMemset(ctx->dWda, 0, sizeof(double) * M * R));
        CKC(cudaMemset(ctx->rs, 0, sizeof(double) * kRsStride * R));
        CKC(cudaMemset(ctx->err, 0, sizeof(int)));
        // 2-D tensor map of all spectra: rows of 2*m1*mk2 reals, nslots*2*2*m0 rows
        L.tma_pencil = 0;
        if (L.fixed && !getenv("SCFT_NO_TMA_PENCIL")) {
            typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess && fn) {
                const int tc = T == 4 ? 32 : 16;  // kTile<T> of the kernels
                cuuint64_t dims[2] = {(cuuint64_t)2 * g.m1 * g.mk2, (cuuint64_t)S * 2 * 2 * g.m0};
                cuuint64_t strides[1] = {(cuuint64_t)2 * g.m1 * g.mk2 * T};
                cuuint32_t es[2] = {1, 1};
                // m0 = 64 with SCFT_PENCIL_SHUFFLE=1: the shuffle pencil, which reads 128-byte boxes
                // with 128-byte swizzling (opt-in: it measured no faster than the Stockham pencil)
                const char *shv = getenv("SCFT_PENCIL_SHUFFLE");
                L.pencil_sh = g.m0 == 64 && shv && shv[0] == '1';
                auto encode = [&](CUtensorMap *m, int w) {
                    cuuint32_t box[2] = {(cuuint32_t)(L.pencil_sh ? 128 / T : 2 * w), (cuuint32_t)g.m0};
                    return ((EncodeFn)fn)(m, T == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                                          ctx->spec, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          L.pencil_sh ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                };
                auto smem_for = [&](int w) {
                    return L.pencil_sh ? pencil_sh_smem_bytes(T == 4, w, g.m0)
                                       : (int)(128 + (2 * w * g.m0 + g.m0) * 2 * T + (w + g.m0) * T);
                };
                if (encode(&ctx->tmap, tc) == CUDA_SUCCESS && g.m0 <= 256 && (strides[0] % 16) == 0) {
                    L.tma_pencil = 1;
                    L.tmap = &ctx->tmap;
                    L.pencil_tma_smem = smem_for(tc);
                    // the wide tile (2 tc columns; box width 4 tc reals <= 256, or 4 boxes of the swizzled map)
                    if (4 * tc <= 256 && smem_for(2 * tc) <= (int)prop.sharedMemPerBlockOptin &&
                        encode(&ctx->tmap_wide, 2 * tc) == CUDA_SUCCESS) {
                        L.tmap_wide = &ctx->tmap_wide;
                        L.pencil_tma_smem_wide = smem_for(2 * tc);
                        if (const char *ev = getenv("SCFT_PENCIL_TILE_WIDE")) L.ptile_wide = ev[0] == '1';
                    }
                }
                if (!L.tma_pencil) L.pencil_sh = 0;
            }
        }
        // the persistent step kernel of the compile-time shapes runs all three
        // roles in one CTA shape: the largest of their shared-memory layouts
        L.step_pf_smem = 0;
        if (L.fixed && L.pf && L.tma_pencil) {
            int sm = std::max(L.mid_pf_smem, std::max(L.combine_pf_smem, L.pencil_tma_smem));
            if (L.tmap_wide) sm = std::max(sm, L.pencil_tma_smem_wide);
            if (sm <= (int)prop.sharedMemPerBlockOptin) L.step_pf_smem = sm;
        }
        if ((T == 4 ? set_props_smem<float>(L) : set_props_smem<double>(L)) != 0) {
            ctx->lasterr = "cudaFuncSetAttribute(max dynamic shared memory) failed";
            rc = SCFT_CUDA_ERROR;
            goto done;
        }
        // one persistent launch per contour step: the register kernels start with
        // it, the shared-memory kernels with four launches (scft_autotune compares
        // both); SCFT_PERSIST=0|1 sets the start, SCFT_NO_PERSIST=1 rules it out
        L.persist = 0;
        L.step_grid_pf = L.step_pf_smem > 0 ? (T == 4 ? props_step_grid<float>(L) : props_step_grid<double>(L)) : 0;
        if (L.reg) {
            L.step_grid = reg64_step_grid();
            L.persist = 1;
        }
        ctx->persist_ok = (L.reg || L.step_grid_pf > 0) && ctx->sync;
        if (const char *ev = getenv("SCFT_PERSIST")) L.persist = ev[0] == '1' ? 1 : 0;
        if (const char *ev = getenv("SCFT_NO_PERSIST"))
            if (ev[0] == '1') ctx->persist_ok = false;
        if (!ctx->persist_ok) L.persist = 0;
        ctx->doiis.assign(ctx->strn, 1);  // one process owns every replica (scft.cu:952-975)
        ctx->graphs.assign((size_t)(R + 1) * (S + 1) + 1, nullptr);
        if (const char *ev = getenv("SCFT_NO_GRAPHS")) ctx->use_graphs = ev[0] != '1';
        ctx->slot_of.assign(R, -1);
        ctx->rs_h.assign(kRsStride * R, 0.0);
        ctx->red_h.assign(ctx->nred_rows, 0.0);
        auto &S_ = ctx->sf;
        S_.x.assign(ctx->strn, 0.0);
        S_.xref.assign(ctx->strn, 0.0);
        S_.alf.assign(ctx->strn, 0.0);
        S_.errs.assign(ctx->strn, 0.0);
        S_.errs3.assign(ctx->strn, 0.0);
        S_.FEs.assign(ctx->strn, 0.0);
        S_.FEs0.assign(ctx->strn, 0.0);
        S_.FEs1.assign(ctx->strn, 0.0);
        S_.phctot.assign(ctx->strn, 0.0);
        S_.steps.assign(ctx->strn, 0);
    }
done:
#undef CKC
    if (rc != SCFT_OK) {
        std::string msg = ctx->lasterr;
        scft_destroy(ctx);
        fprintf(stderr, "scft_create: %s\n", msg.c_str());
        return rc;
    }
    *out = ctx;
    return SCFT_OK;
}

scft_status scft_set_fields(scft_ctx *ctx, int ii, const double *w2M)
{
    if (!ctx || !w2M || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    CK(cudaMemcpyAsync(ctx->W + (size_t)ii * 2 * ctx->M, w2M, sizeof(double) * 2 * ctx->M,
                       cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCFT_OK;
}

scft_status scft_get_fields(const scft_ctx *cctx, int ii, double *w2M)
{
    scft_ctx *ctx = const_cast<scft_ctx *>(cctx);
    if (!ctx || !w2M || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    CK(cudaMemcpyAsync(w2M, ctx->W + (size_t)ii * 2 * ctx->M, sizeof(double) * 2 * ctx->M,
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCFT_OK;
}

scft_status upload_box(scft_ctx *ctx, int r, const double *D);

scft_status scft_copy_fields(scft_ctx *ctx, const scft_ctx *src)
{
    if (!ctx || !src || ctx == src) return SCFT_BAD_INPUT;
    const Geo &a = ctx->g, &b = src->g;
    if (ctx->strn != src->strn || a.m0 != b.m0 || a.m1 != b.m1 || a.m2 != b.m2) {
        ctx->lasterr = "scft_copy_fields: the contexts differ in grid or replica count";
        return SCFT_BAD_INPUT;
    }
    CK(cudaStreamSynchronize(src->st));  // the source's pending updates of its fields
    CK(cudaMemcpyAsync(ctx->W, src->W, sizeof(double) * 2 * ctx->M * ctx->strn, cudaMemcpyDefault, ctx->st));
    for (int r = 0; r < ctx->strn; r++) {
        const double *D = &src->Dr[3 * (size_t)r];
        if (D[0] != ctx->Dr[3 * (size_t)r] || D[1] != ctx->Dr[3 * (size_t)r + 1] || D[2] != ctx->Dr[3 * (size_t)r + 2]) {
            scft_status s = upload_box(ctx, r, D);
            if (s != SCFT_OK) return s;
        }
    }
    CK(cudaStreamSynchronize(ctx->st));
    return SCFT_OK;
}

scft_status scft_get_conc(const scft_ctx *cctx, int ii, double *out4M, double *lnQ, double *phis)
{
    scft_ctx *ctx = const_cast<scft_ctx *>(cctx);
    if (!ctx || ii < 0 || ii >= ctx->nrep_alloc) return SCFT_BAD_INPUT;
    if (out4M) {
        CK(cudaMemcpyAsync(out4M, ctx->conc + (size_t)ii * 4 * ctx->M, sizeof(double) * 4 * ctx->M,
                           cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaMemcpyAsync(ctx->rs_h.data() + (size_t)ii * kRsStride, ctx->rs + (size_t)ii * kRsStride,
                       sizeof(double) * kRsStride, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (lnQ) *lnQ = rsv(ctx, ii, kRsLnQ);
    if (phis)
        for (int k = 0; k < 5; k++) phis[k] = rsv(ctx, ii, kRsPhis + k);
    return SCFT_OK;
}

scft_status scft_get_doiis(const scft_ctx *ctx, int *doiis)
{
    if (!ctx || !doiis) return SCFT_BAD_INPUT;
    for (int i = 0; i < ctx->strn; i++) doiis[i] = ctx->doiis[i];
    return SCFT_OK;
}

scft_status scft_props(scft_ctx *ctx, int ii)
{
    if (!ctx || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    return props_list(ctx, {ii});
}

scft_status scft_props_host(scft_ctx *ctx, double *w, double *lnQ, int ii, int Ns, double alpha,
                            double phic, double *phis, double f)
{
    (void)ii;
    if (!ctx || !w) return SCFT_BAD_INPUT;
    const bool f_ok = ctx->g.jon ? std::fabs(f - ctx->f) <= 1e-12 : (int)std::round(Ns * f) == ctx->g.n1;
    if (Ns != ctx->g.Ns || alpha != ctx->p.alpha || phic != ctx->p.phidb || !f_ok) {
        ctx->lasterr = "scft_props_host: Ns/alpha/phic/f differ from the context";
        return SCFT_BAD_INPUT;
    }
    const int sc = ctx->strn;  // scratch replica
    const size_t M = ctx->M;
    CK(cudaMemcpyAsync(ctx->W + (size_t)sc * 2 * M, w, sizeof(double) * 2 * M, cudaMemcpyHostToDevice,
                       ctx->st));
    scft_status s = props_list(ctx, {sc});
    if (s != SCFT_OK) return s;
    CK(cudaMemcpyAsync(w + 2 * M, ctx->conc + (size_t)sc * 4 * M, sizeof(double) * 4 * M,
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (lnQ) *lnQ = rsv(ctx, sc, kRsLnQ);
    if (phis)
        for (int k = 0; k < 5; k++) phis[k] = rsv(ctx, sc, kRsPhis + k);
    return SCFT_OK;
}

scft_status scft_do_step(scft_ctx *ctx, int ii, const double *in, double *out, int s)
{
    if (!ctx || !in || !out || ii < 0 || ii >= ctx->strn || s < 0 || s >= ctx->g.Ns)
        return SCFT_BAD_INPUT;
    if (ctx->nostore) {
        ctx->lasterr = "scft_do_step needs the full propagator store (context created with nostore)";
        return SCFT_UNSUPPORTED;
    }
    const size_t M = ctx->M;
    const size_t T = ctx->prec == SCFT_FP32 ? 4 : 8;
    const size_t slice = 2 * M;
    std::vector<unsigned char> tmp(slice * T);
    if (T == 4)
        for (size_t i = 0; i < slice; i++) ((float *)tmp.data())[i] = (float)in[i];
    else
        std::memcpy(tmp.data(), in, slice * 8);
    CK(cudaMemcpyAsync(ctx->rep_dev, &ii, sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    unsigned char *h0 = (unsigned char *)ctx->hist + (size_t)s * slice * T;
    CK(cudaMemcpyAsync(h0, tmp.data(), slice * T, cudaMemcpyHostToDevice, ctx->st));
    int nl;
    if (T == 4)
        nl = launch_single_step<float>(props_args<float>(ctx, ctx->rep_dev), ctx->L, s, ctx->st);
    else
        nl = launch_single_step<double>(props_args<double>(ctx, ctx->rep_dev), ctx->L, s, ctx->st);
    ctx->stats.kernel_launches += nl;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(tmp.data(), h0 + slice * T, slice * T, cudaMemcpyDeviceToHost, ctx->st));
    scft_status st = check_device_err(ctx);
    if (st != SCFT_OK) return st;
    for (auto &so : ctx->slot_of)
        if (so == 0) so = -1;
    if (T == 4)
        for (size_t i = 0; i < slice; i++) out[i] = ((float *)tmp.data())[i];
    else
        std::memcpy(out, tmp.data(), slice * 8);
    return SCFT_OK;
}

scft_status scft_get_propagator(const scft_ctx *cctx, int ii, int which, int s, double *outM)
{
    scft_ctx *ctx = const_cast<scft_ctx *>(cctx);
    if (!ctx || !outM || ii < 0 || ii >= ctx->nrep_alloc || s < 0 || s > ctx->g.Ns) return SCFT_BAD_INPUT;
    if (ctx->nostore) {
        ctx->lasterr = "scft_get_propagator needs the full propagator store (context created with nostore)";
        return SCFT_UNSUPPORTED;
    }
    const int slot = ctx->slot_of[ii];
    if (slot < 0) {
        ctx->lasterr = "propagators of this replica are no longer resident";
        return SCFT_BAD_INPUT;
    }
    const size_t M = ctx->M, T = ctx->prec == SCFT_FP32 ? 4 : 8;
    const size_t off = (((size_t)slot * (ctx->g.Ns + 1) + s) * 2 + (which ? 1 : 0)) * M;
    std::vector<unsigned char> tmp(M * T);
    CK(cudaMemcpyAsync(tmp.data(), (unsigned char *)ctx->hist + off * T, M * T, cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (T == 4)
        for (size_t i = 0; i < M; i++) outM[i] = ((float *)tmp.data())[i];
    else
        std::memcpy(outM, tmp.data(), M * 8);
    return SCFT_OK;
}

scft_status scft_solve_field0(scft_ctx *ctx, int ii, int maxIter, double errTol, int *k_out)
{
    if (!ctx || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    std::vector<int> k;
    scft_status s = field0_set(ctx, {ii}, maxIter, errTol, k);
    if (k_out) *k_out = k.empty() ? 0 : k[ii];
    return s;
}

scft_status scft_solve_field0_all(scft_ctx *ctx, int maxIter, double errTol, int *k_out)
{
    if (!ctx) return SCFT_BAD_INPUT;
    std::vector<int> set;
    for (int ii = 0; ii < ctx->strn; ii++)
        if (ctx->doiis[ii] == 1) set.push_back(ii);
    std::vector<int> k;
    scft_status s = field0_set(ctx, set, maxIter, errTol, k);
    if (k_out)
        for (int ii = 0; ii < ctx->strn; ii++) k_out[ii] = k.empty() ? 0 : k[ii];
    return s;
}

scft_status scft_string_begin(scft_ctx *ctx, int doii, int maxIter, double errTol)
{
    if (!ctx || doii < -1 || doii >= ctx->strn) return SCFT_BAD_INPUT;
    auto &S = ctx->sf;
    S.active = true;
    S.doii = doii;
    S.maxIter = maxIter;
    S.errTol = errTol;
    S.k = 0;
    S.lambda = 0.05;
    S.err = 1;
    S.errt = 1;
    S.dospring = 1;
    S.doredist = 0;
    S.doperp = 0;
    S.skip_freee = false;
    if (doii > -1 || ctx->p.dostring != 1) S.dospring = S.doredist = S.doperp = 0;
    if (ctx->p.fix[0] == 1) ctx->doiis[0] = 0;  // scft.cu:587-588
    if (ctx->p.fix[1] == 1) ctx->doiis[ctx->strn - 1] = 0;
    std::fill(S.steps.begin(), S.steps.end(), 0);
    return SCFT_OK;
}

scft_status scft_string_resume(scft_ctx *ctx, int doii, int maxIter, double errTol, int k0)
{
    if (!ctx || k0 < 0) return SCFT_BAD_INPUT;
    scft_status s = scft_string_begin(ctx, doii, maxIter, errTol);
    if (s != SCFT_OK) return s;
    ctx->sf.k = k0;
    return SCFT_OK;
}

scft_status scft_selftest_timeout(scft_ctx *ctx, int polls)
{
    if (!ctx || polls < 1) return SCFT_BAD_INPUT;
    launch_wait_selftest(ctx->err, (unsigned)polls, ctx->st);
    ctx->stats.kernel_launches += 1;
    CK(cudaGetLastError());
    return check_device_err(ctx);
}

// one k-pass of the solve_field loop, scft.cu:592-806
scft_status scft_string_step(scft_ctx *ctx, scft_iter_report *rep, double *errs_out,
                             double *errs3_out, int *done)
{
    if (!ctx || !ctx->sf.active) return SCFT_BAD_INPUT;
    auto &S = ctx->sf;
    const int strn = ctx->strn, doii = S.doii;
    const size_t M = ctx->M;
    const double eps = 0.5;
    const int skip = 50;
    scft_status s;
    if (!(S.k < S.maxIter && S.err > S.errTol)) {
        if (done) *done = 1;
        return SCFT_OK;
    }
    const int k = S.k;
    if (k >= ctx->p.springsteps && doii == -1 && ctx->p.dostring == 1) {
        S.dospring = 0;
        S.doredist = 1;
        S.doperp = 1;
    }
    CK(cudaMemsetAsync(ctx->DEV, 0, sizeof(double) * 2 * M * strn, ctx->st));
    std::vector<int> set;
    for (int ii = 0; ii < strn; ii++) {
        S.steps[ii] = 0;
        if ((ctx->doiis[ii] == 1 && doii == -1) || doii == ii) set.push_back(ii);
    }
    for (int ii : set) S.steps[ii]++;
    std::vector<int> k0;
    s = field0_set(ctx, set, 20, S.errTol, k0);
    if (s != SCFT_OK) return s;
    for (int ii : set) S.steps[ii] += k0[ii];
    if (ctx->p.batched) {
        s = props_list(ctx, set);
        if (s != SCFT_OK) return s;
    } else {
        for (int ii : set) {
            s = props_list(ctx, {ii});
            if (s != SCFT_OK) return s;
        }
    }
    // residuals DEV (scft.cu:604-608)
    std::vector<double> sum2(strn, 0.0), summ(strn, 0.0);
    if (!set.empty()) {
        s = upload_list(ctx, set);
        if (s != SCFT_OK) return s;
        launch_dev(field_args(ctx, ctx->rep_dev), (int)set.size(), kRedBlocks, S.dospring, eps, ctx->st);
        ctx->stats.kernel_launches += 1;
        s = reduce_rows(ctx, 2 * (int)set.size(), kRedBlocks);
        if (s != SCFT_OK) return s;
        for (size_t j = 0; j < set.size(); j++) {
            sum2[set[j]] = ctx->red_h[2 * j];
            summ[set[j]] = ctx->red_h[2 * j + 1];
        }
    }
    if (doii == -1) {
        s = arc_length(ctx, S.x);
        if (s != SCFT_OK) return s;
        for (int ii = 0; ii < strn; ii++) S.xref[ii] = (1.0 * ii) / (strn - 1.0);
        for (int ii = 0; ii < strn; ii++) S.errs[ii] = std::pow(sum2[ii] / (2 * (double)M), 0.5);
    } else {
        for (int ii = 0; ii < strn; ii++) S.errs[ii] = 0;
        S.errs[doii] = std::pow(sum2[doii] / (2 * (double)M), 0.5);
    }
    if (S.doperp == 1) {
        // spline derivative along the string and projection (scft.cu:641-683)
        s = upload_knots(ctx, S.x, nullptr, ctx->doiis.data());
        if (s != SCFT_OK) return s;
        launch_spline_deriv(field_args(ctx, ctx->rep_dev), ctx->knots, 4 * kRedBlocks, ctx->st);
        ctx->stats.kernel_launches += 1;
        std::vector<int> dset;
        for (int ii = 0; ii < strn; ii++)
            if (ctx->doiis[ii] == 1) dset.push_back(ii);
        std::vector<double> normDER(strn, 0.0), normDEV(strn, 0.0), dotWs(strn, 0.0);
        if (!dset.empty()) {
            s = upload_list(ctx, dset);
            if (s != SCFT_OK) return s;
            launch_dots(field_args(ctx, ctx->rep_dev), (int)dset.size(), kRedBlocks, ctx->st);
            ctx->stats.kernel_launches += 1;
            s = reduce_rows(ctx, 2 * (int)dset.size(), kRedBlocks);
            if (s != SCFT_OK) return s;
            for (size_t j = 0; j < dset.size(); j++) {
                const int ii = dset[j];
                normDER[ii] = std::sqrt(ctx->red_h[2 * j]);
                normDEV[ii] = std::sqrt(summ[ii]);
                dotWs[ii] = ctx->red_h[2 * j + 1] / (normDEV[ii] * normDER[ii]);
            }
        }
        for (int ii = 0; ii < strn; ii++) S.errs3[ii] = 0;
        std::vector<int> pset;
        std::vector<double> coef, ndev;
        for (int ii = 1; ii < strn - 1; ii++) {
            if (ctx->doiis[ii] == 1 && normDER[ii] > 0 && normDEV[ii] > 0) {
                pset.push_back(ii);
                coef.push_back(dotWs[ii] / normDER[ii]);
                ndev.push_back(normDEV[ii]);
            } else if (ctx->doiis[ii] == 1) {
                fprintf(stderr, "Fatal error occurred (0)... %d %d %lf %lf\n", k, ii, normDER[ii],
                        normDEV[ii]);
            }
        }
        if (!pset.empty()) {
            s = upload_list(ctx, pset);
            if (s != SCFT_OK) return s;
            launch_perp(field_args(ctx, ctx->rep_dev), (int)pset.size(), coef.data(), ndev.data(),
                        kRedBlocks, ctx->st);
            ctx->stats.kernel_launches += 1;
            s = reduce_rows(ctx, (int)pset.size(), kRedBlocks);
            if (s != SCFT_OK) return s;
            for (size_t j = 0; j < pset.size(); j++)
                S.errs3[pset[j]] = std::pow(ctx->red_h[j] / (2 * (double)M), 0.5);
        }
    } else {
        for (int ii = 0; ii < strn; ii++) S.errs3[ii] = S.errs[ii];
    }
    S.errs3[0] = S.errs[0];
    S.errs3[strn - 1] = S.errs[strn - 1];
    // simple mixing with fixed mixing parameter (scft.cu:691-693)
    launch_mix(field_args(ctx, ctx->rep_dev), S.lambda, ctx->st);
    ctx->stats.kernel_launches += 1;
    CK(cudaGetLastError());
    double stepav = 0;
    for (int ii = 0; ii < strn; ii++) stepav += S.steps[ii];
    stepav /= strn;
    double fitup = 0;
    std::vector<double> xnew = S.x;
    if (doii == -1) {
        s = arc_length(ctx, xnew);
        if (s != SCFT_OK) return s;
        for (int ii = 0; ii < strn; ii++) S.alf[ii] = xnew[ii];
        for (int ii = 1; ii < strn - 1; ii++) fitup += std::pow(xnew[ii] - S.xref[ii], 2.0);
        fitup /= strn - 2.0;
        fitup = std::sqrt(fitup);
        fitup /= strn - 1.0;
        S.x = xnew;
    }
    if (S.doredist == 1) {
        // equal-arc redistribution (scft.cu:745-757)
        s = upload_knots(ctx, S.x, &S.xref, ctx->doiis.data());
        if (s != SCFT_OK) return s;
        launch_redist(field_args(ctx, ctx->rep_dev), ctx->knots, S.lambda, 4 * kRedBlocks, ctx->st);
        ctx->stats.kernel_launches += 1;
        CK(cudaGetLastError());
    }
    double errtot = 0;
    for (int ii = 0; ii < strn; ii++) errtot += S.errs3[ii] * S.errs3[ii] / strn;
    errtot = std::sqrt(errtot);
    int did_fe = 0;
    if (!S.skip_freee && (k % skip == 0 || k == S.maxIter - 1 || !(S.err > S.errTol))) {
        s = free_energy(ctx, &S.FE);
        if (s != SCFT_OK) return s;
        did_fe = 1;
    }
    CK(cudaStreamSynchronize(ctx->st));
    if (rep) {
        rep->k = k;
        rep->lambda = S.lambda;
        rep->errtot = errtot;
        rep->fitup = fitup;
        rep->stepav = stepav;
        rep->did_freee = did_fe;
        rep->FE = did_fe ? S.FE : 0.0;
    }
    if (errs_out) std::memcpy(errs_out, S.errs.data(), sizeof(double) * strn);
    if (errs3_out) std::memcpy(errs3_out, S.errs3.data(), sizeof(double) * strn);
    // mixing-parameter update (scft.cu:793-798): err stays 1, so lambda stays 0.05
    if (S.err < S.errt)
        S.lambda = std::min(0.2, S.lambda * 1.015);
    else
        S.lambda = std::max(0.05, S.lambda / 1.016);
    S.errt = S.err;
    S.k++;
    if (done) *done = (S.k < S.maxIter && S.err > S.errTol) ? 0 : 1;
    return SCFT_OK;
}

scft_status scft_string_end(scft_ctx *ctx, int *k_out)
{
    if (!ctx) return SCFT_BAD_INPUT;
    if (k_out) *k_out = ctx->sf.k;
    ctx->sf.active = false;
    return SCFT_OK;
}

scft_status scft_solve_field(scft_ctx *ctx, int doii, int maxIter, double errTol,
                             scft_iter_report *reports, double *errs, double *errs3, int *k_out)
{
    scft_status s = scft_string_begin(ctx, doii, maxIter, errTol);
    if (s != SCFT_OK) return s;
    int done = 0;
    while (!done) {
        const int k = ctx->sf.k;
        if (!(k < maxIter && ctx->sf.err > errTol)) break;
        s = scft_string_step(ctx, reports ? reports + k : nullptr,
                             errs ? errs + (size_t)k * ctx->strn : nullptr,
                             errs3 ? errs3 + (size_t)k * ctx->strn : nullptr, &done);
        if (s != SCFT_OK) return s;
    }
    return scft_string_end(ctx, k_out);
}

scft_status scft_free_energy(scft_ctx *ctx, double *FE, double *FEs, double *FEs0, double *FEs1,
                             double *phctot, double *alf)
{
    if (!ctx) return SCFT_BAD_INPUT;
    double fe = 0;
    scft_status s = free_energy(ctx, &fe);
    if (s != SCFT_OK) return s;
    ctx->sf.FE = fe;
    const size_t n = sizeof(double) * ctx->strn;
    if (FE) *FE = fe;
    if (FEs) std::memcpy(FEs, ctx->sf.FEs.data(), n);
    if (FEs0) std::memcpy(FEs0, ctx->sf.FEs0.data(), n);
    if (FEs1) std::memcpy(FEs1, ctx->sf.FEs1.data(), n);
    if (phctot) std::memcpy(phctot, ctx->sf.phctot.data(), n);
    if (alf) std::memcpy(alf, ctx->sf.alf.data(), n);
    return SCFT_OK;
}

scft_status scft_last_free_energy(const scft_ctx *ctx, double *FE, double *FEs, double *FEs0,
                                  double *FEs1, double *phctot, double *alf)
{
    if (!ctx) return SCFT_BAD_INPUT;
    const size_t n = sizeof(double) * ctx->strn;
    if (FE) *FE = ctx->sf.FE;
    if (FEs) std::memcpy(FEs, ctx->sf.FEs.data(), n);
    if (FEs0) std::memcpy(FEs0, ctx->sf.FEs0.data(), n);
    if (FEs1) std::memcpy(FEs1, ctx->sf.FEs1.data(), n);
    if (phctot) std::memcpy(phctot, ctx->sf.phctot.data(), n);
    if (alf) std::memcpy(alf, ctx->sf.alf.data(), n);
    return SCFT_OK;
}

// density::splineDerivsChunked with host arrays (density.h:491-508).  Uses the
// device W- storage of the context as staging (replicas' fields are restored).
static scft_status spline_host(scft_ctx *ctx, const double *x, const double *xref,
                               const double *const *ww, double *const *out, double *const *wio,
                               int r0, int n, const int *doiis, double lambda)
{
    if (!ctx || !x || n < 0 || r0 < 0 || r0 + n > ctx->M) return SCFT_BAD_INPUT;
    const int strn = ctx->strn;
    const size_t M = ctx->M;
    // save W-, stage the chunk at the start of each replica's W- row
    std::vector<double> saved(2 * M * strn);
    CK(cudaMemcpyAsync(saved.data(), ctx->W, sizeof(double) * 2 * M * strn, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<double> stage(saved);
    for (int ii = 0; ii < strn; ii++) {
        const double *src = ww ? ww[ii] : wio[ii];
        std::memcpy(stage.data() + (size_t)ii * 2 * M, src + r0, sizeof(double) * n);
    }
    CK(cudaMemcpyAsync(ctx->W, stage.data(), sizeof(double) * 2 * M * strn, cudaMemcpyHostToDevice, ctx->st));
    std::vector<double> xv(x, x + strn), xr;
    if (xref) xr.assign(xref, xref + strn);
    scft_status s = upload_knots(ctx, xv, xref ? &xr : nullptr, doiis);
    if (s != SCFT_OK) return s;
    FieldArgs a = field_args(ctx, ctx->rep_dev);
    a.M = (int)M;
    if (out) {
        launch_spline_deriv(a, ctx->knots, 4 * kRedBlocks, ctx->st);
        std::vector<double> d(M * strn);
        CK(cudaMemcpyAsync(d.data(), ctx->dWda, sizeof(double) * M * strn, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int ii = 0; ii < strn; ii++)
            if (doiis[ii] == 1) std::memcpy(out[ii] + r0, d.data() + (size_t)ii * M, sizeof(double) * n);
    } else {
        launch_redist(a, ctx->knots, lambda, 4 * kRedBlocks, ctx->st);
        std::vector<double> w(2 * M * strn);
        CK(cudaMemcpyAsync(w.data(), ctx->W, sizeof(double) * 2 * M * strn, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int ii = 1; ii < strn - 1; ii++)
            if (doiis[ii] == 1) std::memcpy(wio[ii] + r0, w.data() + (size_t)ii * 2 * M, sizeof(double) * n);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->W, saved.data(), sizeof(double) * 2 * M * strn, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return SCFT_OK;
}

scft_status scft_spline_derivs(scft_ctx *ctx, const double *x, const double *const *ww, int r0, int n,
                               const int *doiis, double *const *out)
{
    if (!ww || !out || !doiis) return SCFT_BAD_INPUT;
    return spline_host(ctx, x, nullptr, ww, out, nullptr, r0, n, doiis, 0.0);
}

scft_status scft_spline_redist(scft_ctx *ctx, const double *x, const double *xref, double *const *ww,
                               int r0, int n, const int *doiis, double lambda)
{
    if (!ww || !xref || !doiis) return SCFT_BAD_INPUT;
    return spline_host(ctx, x, xref, nullptr, nullptr, ww, r0, n, doiis, lambda);
}

// box lengths: re-derive the per-axis diffusion factors (setup_k_sq, density.h:79-95)
namespace {
// uploads the diffusion factors of replica r for the box D
scft_status upload_box(scft_ctx *ctx, int r, const double *D)
{
    std::vector<unsigned char> twb, kfb;
    if (ctx->prec == SCFT_FP32)
        upload_tables<float>(ctx, twb, kfb, D);
    else
        upload_tables<double>(ctx, twb, kfb, D);
    CK(cudaMemcpyAsync((unsigned char *)ctx->kfac + (size_t)r * kfb.size(), kfb.data(), kfb.size(),
                       cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));  // kfb is pageable and goes out of scope
    for (int i = 0; i < 3; i++) ctx->Dr[3 * (size_t)r + i] = D[i];
    return SCFT_OK;
}

bool box_ok(const double *D)
{
    if (!D) return false;
    for (int i = 0; i < 3; i++)
        if (!(std::isfinite(D[i]) && D[i] > 0)) return false;
    return true;
}
}  // namespace

// the box of every replica (and the scratch replica of scft_props_host)
scft_status scft_set_box(scft_ctx *ctx, const double *D)
{
    if (!ctx || !box_ok(D)) return SCFT_BAD_INPUT;
    for (int i = 0; i < 3; i++) ctx->p.D[i] = D[i];
    std::fill(ctx->slot_of.begin(), ctx->slot_of.end(), -1);  // stored propagators are of the old box
    for (int r = 0; r < ctx->nrep_alloc; r++) {
        scft_status s = upload_box(ctx, r, D);
        if (s != SCFT_OK) return s;
    }
    return SCFT_OK;
}

scft_status scft_get_box(const scft_ctx *ctx, double *D)
{
    if (!ctx || !D) return SCFT_BAD_INPUT;
    for (int i = 0; i < 3; i++) D[i] = ctx->p.D[i];
    return SCFT_OK;
}

scft_status scft_set_box_replica(scft_ctx *ctx, int ii, const double *D)
{
    if (!ctx || ii < 0 || ii >= ctx->strn || !box_ok(D)) return SCFT_BAD_INPUT;
    ctx->slot_of[ii] = -1;  // its stored propagators no longer match its box
    return upload_box(ctx, ii, D);
}

scft_status scft_get_box_replica(const scft_ctx *ctx, int ii, double *D)
{
    if (!ctx || !D || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    for (int i = 0; i < 3; i++) D[i] = ctx->Dr[3 * (size_t)ii + i];
    return SCFT_OK;
}

// d lnQ / d L_i of replica ii at its current fields, by the adjoint of the
// propagator (stress_kernels.cu); the free energy's box derivative at the
// saddle point is dF/dL = -dlnQ/dL (the field terms carry no explicit L).
}  // extern "C"

namespace {

// one adjoint pair <y, dS/dL x>: slices (xs, xf) and (ys, yf) of the store at
// `hist` (slot `slot`), E table `sel`, homopolymer (Q2) or copolymer (QC) sum
struct StressPr {
    int xs, xf, ys, yf, sel, homo;
};

scft_status stress_alloc(scft_ctx *ctx)
{
    if (ctx->st_S4) return SCFT_OK;
    const Geo &g = ctx->g;
    const size_t T = ctx->prec == SCFT_FP32 ? 4 : 8;
    const size_t sz = T * 2 * 2 * (size_t)g.Mk * kStressPairs;
    CK(cudaMalloc(&ctx->st_S4, sz));
    CK(cudaMalloc(&ctx->st_S2, sz));
    CK(cudaMalloc(&ctx->st_S4p, sz));
    CK(cudaMalloc(&ctx->st_part, sizeof(double) * 9 * (size_t)g.ncol_tiles * kStressPairs));
    CK(cudaMalloc(&ctx->st_out, sizeof(double) * 3 * kStressPairs));
    if ((T == 4 ? set_stress_smem<float>(ctx->rt_slab_smem, ctx->rt_pencil_smem)
                : set_stress_smem<double>(ctx->rt_slab_smem, ctx->rt_pencil_smem)) != 0) {
        ctx->lasterr = "stress kernels: shared memory attribute";
        return SCFT_CUDA_ERROR;
    }
    return SCFT_OK;
}

// sums the pairs (in chunks of kStressPairs) into dQC / dQ2 (unnormalised)
scft_status stress_pairs(scft_ctx *ctx, int rep, int slot, const void *hist, const std::vector<StressPr> &pairs,
                         double *dQC, double *dQ2)
{
    const Geo &g = ctx->g;
    const double *Lr = &ctx->Dr[3 * (size_t)rep];  // the replica's box
    std::vector<double> out(3 * kStressPairs);
    for (size_t c0 = 0; c0 < pairs.size(); c0 += kStressPairs) {
        StressPairs P;
        std::memset(&P, 0, sizeof(P));
        P.n = (int)std::min<size_t>(kStressPairs, pairs.size() - c0);
        for (int p = 0; p < P.n; p++) {
            const StressPr &q = pairs[c0 + p];
            P.xs[p] = q.xs;
            P.xf[p] = q.xf;
            P.ys[p] = q.ys;
            P.yf[p] = q.yf;
            P.sel[p] = q.sel;
        }
        int nl;
        if (ctx->prec == SCFT_FP32) {
            StressArgs<float> a{g, slot, (const float *)hist, (const float *)ctx->etab,
                                (const cplx<float> *)ctx->tw, (const float *)ctx->kfac + (size_t)rep * ctx->kf_n,
                                (cplx<float> *)ctx->st_S4, (cplx<float> *)ctx->st_S2,
                                (cplx<float> *)ctx->st_S4p, ctx->st_part,
                                {Lr[0], Lr[1], Lr[2]}, (float)(1.0 / g.M), ctx->err};
            a.jtab = (const float *)ctx->jtab;
            nl = launch_stress_chunk<float>(a, P, ctx->rt_slab_threads, ctx->rt_slab_smem,
                                            ctx->rt_pencil_threads, ctx->rt_pencil_smem, ctx->st_out, ctx->st);
        } else {
            StressArgs<double> a{g, slot, (const double *)hist, (const double *)ctx->etab,
                                 (const cplx<double> *)ctx->tw, (const double *)ctx->kfac + (size_t)rep * ctx->kf_n,
                                 (cplx<double> *)ctx->st_S4, (cplx<double> *)ctx->st_S2,
                                 (cplx<double> *)ctx->st_S4p, ctx->st_part,
                                 {Lr[0], Lr[1], Lr[2]}, 1.0 / g.M, ctx->err};
            a.jtab = (const double *)ctx->jtab;
            nl = launch_stress_chunk<double>(a, P, ctx->rt_slab_threads, ctx->rt_slab_smem,
                                             ctx->rt_pencil_threads, ctx->rt_pencil_smem, ctx->st_out, ctx->st);
        }
        ctx->stats.kernel_launches += nl;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out.data(), ctx->st_out, sizeof(double) * 3 * P.n, cudaMemcpyDeviceToHost, ctx->st));
        scft_status s = check_device_err(ctx);
        if (s != SCFT_OK) return s;
        for (int p = 0; p < P.n; p++)
            for (int i = 0; i < 3; i++) (pairs[c0 + p].homo ? dQ2 : dQC)[i] += out[3 * p + i];
    }
    return SCFT_OK;
}

// d lnQ/dL from the pair sums (the ensemble's lnQ, density.h:388-399)
void stress_finish(const scft_ctx *ctx, double Q2, double QC, double *dQC, double *dQ2, double *dlnQ_dL,
                   double *dF_dL)
{
    const double invM = 1.0 / ctx->g.M, phic = ctx->p.phidb, alpha = ctx->p.alpha;
    for (int i = 0; i < 3; i++) {
        dQC[i] *= invM;
        dQ2[i] *= invM;
        double d;
        if (ctx->p.ens == 1)  // lnQ = phic ln QC + (1-phic)/alpha ln Q2 (density.h:390)
            d = phic * dQC[i] / QC + ((1.0 - phic) / alpha) * dQ2[i] / Q2;
        else                  // "lnQ" = Q2 + phic QC (density.h:398)
            d = dQ2[i] + phic * dQC[i];
        if (dlnQ_dL) dlnQ_dL[i] = d;
        if (dF_dL) dF_dL[i] = -d;
    }
}

// E table of q's step s (0 A, 1 B, 2 junction step of a continuous A fraction)
int q_table(const Geo &g, int s) { return (g.jon && s == g.jq) ? 2 : (s < g.n1 ? 0 : 1); }

// Symmetric partition of [0, n) into pieces of at most K steps: boundaries
// 0, K, 2K, ... up to the middle and their mirrors n - jK, so that the mirror
// [n-b, n-a) of every piece [a, b) is a piece too.
std::vector<int> mirror_bounds(int n, int K)
{
    std::vector<int> b;
    const int j = n / (2 * K), a = j * K, m = n - 2 * a;
    for (int x = 0; x <= a; x += K) b.push_back(x);
    if (m > K) {
        if (m % 2 == 0) {
            b.push_back(a + m / 2);
        } else {
            b.push_back(a + (m - 1) / 2);
            b.push_back(a + (m + 1) / 2);
        }
    }
    for (int x = a; x >= 0; x -= K) b.push_back(n - x);
    std::sort(b.begin(), b.end());
    b.erase(std::unique(b.begin(), b.end()), b.end());
    return b;
}

}  // namespace

extern "C" {

scft_status scft_stress(scft_ctx *ctx, int ii, double *dlnQ_dL, double *dF_dL)
{
    if (!ctx || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    if (ctx->nostore) return scft_stress_ckpt(ctx, ii, ctx->ckK, dlnQ_dL, dF_dL, nullptr);
    const Geo &g = ctx->g;
    scft_status s = stress_alloc(ctx);
    if (s != SCFT_OK) return s;
    // fresh propagators of replica ii
    s = props_list(ctx, {ii});
    if (s != SCFT_OK) return s;
    const int slot = ctx->slot_of[ii];
    const double Q2 = rsv(ctx, ii, kRsQ2), QC = rsv(ctx, ii, kRsQC);
    // pairs: copolymer (q(s), q^dagger(N-1-s)), homopolymer (q^dagger(j), q^dagger(Nh-1-j))
    std::vector<StressPr> pairs;
    for (int s2 = 0; s2 < g.Ns; s2++) pairs.push_back({s2, 0, g.Ns - 1 - s2, 1, q_table(g, s2), 0});
    for (int j = 0; j < g.Nh; j++) pairs.push_back({j, 1, g.Nh - 1 - j, 1, 1, 1});
    double dQC[3] = {0, 0, 0}, dQ2[3] = {0, 0, 0};
    s = stress_pairs(ctx, ii, slot, ctx->hist, pairs, dQC, dQ2);
    if (s != SCFT_OK) return s;
    stress_finish(ctx, Q2, QC, dQC, dQ2, dlnQ_dL, dF_dL);
    return SCFT_OK;
}

}  // extern "C"

namespace {

// Propagators of one replica held only at checkpoints (the checkpointed
// adjoint and density pass).  Positions: the starts of a mirror-symmetric
// partition of [0, N) into pieces of at most K steps, and of [0, Nh) for the
// homopolymer.  ck_mem holds, in slice pairs (q, q^dagger): the checkpoints,
// two segments of K+1 slices, [q^dagger(Nh), q(N)], then `extra` bytes.
struct CkptRun {
    int K = 0;
    std::vector<int> bc, bh, row_of, pos;
    size_t pairB = 0;
    unsigned char *ck = nullptr, *seg = nullptr, *segB = nullptr, *qb = nullptr, *extra = nullptr;
    double bytes = 0;
};

template <typename T>
PropsArgs<T> ckpt_args(scft_ctx *ctx, const Geo &gg, void *hist)
{
    PropsArgs<T> a = props_args_from<T>(ctx, ctx->rep_dev, 0);
    a.g = gg;
    a.hist = (T *)hist;
    return a;
}

// g.Ns = len steps of slot 0 from contour index p0 (segment Geo: n1, n2 and the
// junction steps shifted by p0), starting from store slice 0 (mode 2) or q = 1
void ckpt_chain(scft_ctx *ctx, int p0, int len, void *buf, int first_mode)
{
    const Geo &g = ctx->g;
    Geo gg = g;
    gg.Ns = len;
    gg.n1 = g.n1 - p0;
    gg.n2 = g.n2 - p0;
    gg.jq = g.jq - p0;
    gg.jqd = g.jqd - p0;
    ctx->stats.kernel_launches += ctx->prec == SCFT_FP32
                                      ? launch_chain<float>(ckpt_args<float>(ctx, gg, buf), ctx->L, first_mode, ctx->st)
                                      : launch_chain<double>(ckpt_args<double>(ctx, gg, buf), ctx->L, first_mode, ctx->st);
}

// allocation, forward pass (checkpoints, q^dagger(Nh), q(N)), then Q2, QC,
// lnQ and the ensemble weights of replica ii in rs (device and rs_h)
scft_status ckpt_forward(scft_ctx *ctx, int ii, int K, size_t extra_bytes, CkptRun &R)
{
    const Geo &g = ctx->g;
    const int N = g.Ns, Nh = g.Nh;
    R.K = K = std::min(K, N);
    R.bc = mirror_bounds(N, K);
    R.bh = Nh > 0 ? mirror_bounds(Nh, std::min(K, Nh)) : std::vector<int>{0};
    R.row_of.assign(N + 1, -1);
    R.pos.clear();
    for (size_t k = 0; k + 1 < R.bc.size(); k++) R.pos.push_back(R.bc[k]);
    for (size_t k = 0; k + 1 < R.bh.size(); k++) R.pos.push_back(R.bh[k]);
    R.pos.push_back(0);
    std::sort(R.pos.begin(), R.pos.end());
    R.pos.erase(std::unique(R.pos.begin(), R.pos.end()), R.pos.end());
    for (size_t r = 0; r < R.pos.size(); r++) R.row_of[R.pos[r]] = (int)r;
    const size_t T = ctx->prec == SCFT_FP32 ? 4 : 8;
    R.pairB = 2 * (size_t)g.M * T;
    const size_t nrow = R.pos.size() + 2 * (size_t)(K + 1) + 2;
    const size_t need = nrow * R.pairB + extra_bytes;
    if (ctx->ck_bytes < need) {
        if (ctx->ck_mem) cudaFree(ctx->ck_mem);
        ctx->ck_mem = nullptr;
        ctx->ck_bytes = 0;
        CK(cudaMalloc(&ctx->ck_mem, need));
        ctx->ck_bytes = need;
    }
    R.ck = (unsigned char *)ctx->ck_mem;
    R.seg = R.ck + R.pos.size() * R.pairB;
    R.segB = R.seg + (size_t)(K + 1) * R.pairB;
    R.qb = R.segB + (size_t)(K + 1) * R.pairB;
    R.extra = R.qb + 2 * R.pairB;
    R.bytes = (double)need;
    scft_status s = upload_list(ctx, {ii});
    if (s != SCFT_OK) return s;
    for (auto &so : ctx->slot_of)  // slot 0's E tables and spectra are reused below
        if (so == 0) so = -1;
    const bool f32 = ctx->prec == SCFT_FP32;
    auto cp = [&](void *dst, const void *src) {
        return cudaMemcpyAsync(dst, src, R.pairB, cudaMemcpyDeviceToDevice, ctx->st);
    };
    // E tables of replica ii in slot 0, then the chain piece by piece
    ctx->stats.kernel_launches += f32 ? launch_prepare<float>(ckpt_args<float>(ctx, g, ctx->hist), ctx->L, ctx->st)
                                      : launch_prepare<double>(ckpt_args<double>(ctx, g, ctx->hist), ctx->L, ctx->st);
    std::vector<int> stops(R.pos);
    stops.push_back(N);
    if (Nh > 0 && Nh < N) stops.push_back(Nh);
    std::sort(stops.begin(), stops.end());
    stops.erase(std::unique(stops.begin(), stops.end()), stops.end());
    int prev = 0;  // length of the previous piece: its last slice starts the next one
    unsigned char *seg = R.seg;
    for (size_t k = 0; k + 1 < stops.size(); k++) {
        const int p0 = stops[k], p1 = stops[k + 1];
        if (p0 > 0) CK(cp(seg, seg + (size_t)prev * R.pairB));
        ckpt_chain(ctx, p0, p1 - p0, seg, p0 == 0 ? 1 : 2);
        prev = p1 - p0;
        if (p0 == 0) CK(cp(R.ck + R.row_of[0] * R.pairB, seg));
        if (p0 == 0 && Nh == 0) CK(cp(R.qb, seg));
        if (p1 < N && R.row_of[p1] >= 0) CK(cp(R.ck + R.row_of[p1] * R.pairB, seg + (size_t)(p1 - p0) * R.pairB));
        if (p1 == Nh) CK(cp(R.qb, seg + (size_t)(p1 - p0) * R.pairB));
        if (p1 == N) CK(cp(R.qb + R.pairB, seg + (size_t)(p1 - p0) * R.pairB));
    }
    CK(cudaGetLastError());
    // Q2 = <q^dagger(Nh)>, QC = <q(N)>: a two-slice store with Ns = 1, Nh = 0
    Geo gq = g;
    gq.Ns = 1;
    gq.Nh = 0;
    ctx->stats.kernel_launches += f32 ? launch_qsums<float>(ckpt_args<float>(ctx, gq, R.qb), ctx->L, ctx->st)
                                      : launch_qsums<double>(ckpt_args<double>(ctx, gq, R.qb), ctx->L, ctx->st);
    CK(cudaMemcpyAsync(&ctx->rs_h[(size_t)ii * kRsStride], ctx->rs + (size_t)ii * kRsStride,
                       sizeof(double) * kRsStride, cudaMemcpyDeviceToHost, ctx->st));
    return check_device_err(ctx);
}

}  // namespace

extern "C" {

// The same adjoint with the propagators stored only at checkpoints (CkptRun).
// Each piece [a, b) is recomputed together with its mirror [N-b, N-a): the two
// segments hold q(s) and q^dagger(N-1-s) for every s of both pieces, i.e. all
// of their pairs.  Cost: two chain passes; memory: (#checkpoints + 2 (K+1) + 2)
// slice pairs instead of N+1.  The slices are the same bits as the full
// store's (same kernels, same inputs), so the result equals scft_stress up to
// the order of the final FP64 pair sums.
scft_status scft_stress_ckpt(scft_ctx *ctx, int ii, int K, double *dlnQ_dL, double *dF_dL, double *bytes_out)
{
    if (!ctx || ii < 0 || ii >= ctx->strn || K < 1) return SCFT_BAD_INPUT;
    const Geo &g = ctx->g;
    const int N = g.Ns, Nh = g.Nh;
    scft_status s = stress_alloc(ctx);
    if (s != SCFT_OK) return s;
    CkptRun R;
    s = ckpt_forward(ctx, ii, K, 0, R);
    if (s != SCFT_OK) return s;
    K = R.K;
    if (bytes_out) *bytes_out = R.bytes;
    const size_t pairB = R.pairB;
    unsigned char *ck = R.ck, *seg = R.seg, *segB = R.segB;
    const std::vector<int> &bc = R.bc, &bh = R.bh, &row_of = R.row_of;
    auto cp = [&](void *dst, const void *src) {
        return cudaMemcpyAsync(dst, src, pairB, cudaMemcpyDeviceToDevice, ctx->st);
    };
    auto chain = [&](int p0, int len, void *buf, int first_mode) { ckpt_chain(ctx, p0, len, buf, first_mode); };
    const double Q2 = rsv(ctx, ii, kRsQ2), QC = rsv(ctx, ii, kRsQC);
    double dQC[3] = {0, 0, 0}, dQ2[3] = {0, 0, 0};
    // recompute each piece with its mirror; the pairs of both pieces
    auto sweep = [&](const std::vector<int> &b, int n, bool homo) -> scft_status {
        const size_t segoff = (size_t)(K + 1);  // slice index of segment B's first slice
        for (size_t k = 0; k + 1 < b.size(); k++) {
            const int a0 = b[k], a1 = b[k + 1], m0 = n - a1, m1 = n - a0;
            if (a0 > m0) continue;  // right half: done as a mirror
            const bool self = (a0 == m0);
            std::vector<StressPr> pairs;
            cudaError_t e = cp(seg, ck + row_of[a0] * pairB);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "checkpoint copy");
            chain(a0, a1 - a0, seg, 2);
            if (!self) {
                e = cp(segB, ck + row_of[m0] * pairB);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "checkpoint copy");
                chain(m0, m1 - m0, segB, 2);
            }
            const int yb = self ? 0 : (int)segoff;  // where the mirror piece's slices are
            // pairs (x(t), y(n-1-t)) for t in [a0, a1): x in segment A, y in the mirror
            for (int t = a0; t < a1; t++) {
                const int u = n - 1 - t;
                if (homo)
                    pairs.push_back({t - a0, 1, yb + (u - m0), 1, 1, 1});
                else
                    pairs.push_back({t - a0, 0, yb + (u - m0), 1, q_table(g, t), 0});
            }
            if (!self)
                for (int t = m0; t < m1; t++) {
                    const int u = n - 1 - t;
                    if (homo)
                        pairs.push_back({(int)segoff + (t - m0), 1, u - a0, 1, 1, 1});
                    else
                        pairs.push_back({(int)segoff + (t - m0), 0, u - a0, 1, q_table(g, t), 0});
                }
            scft_status st = stress_pairs(ctx, ii, 0, seg, pairs, dQC, dQ2);
            if (st != SCFT_OK) return st;
        }
        return SCFT_OK;
    };
    s = sweep(bc, N, false);
    if (s != SCFT_OK) return s;
    if (Nh > 0) {
        s = sweep(bh, Nh, true);
        if (s != SCFT_OK) return s;
    }
    stress_finish(ctx, Q2, QC, dQC, dQ2, dlnQ_dL, dF_dL);
    return SCFT_OK;
}

// density::props of replica ii (density.h:344-459) with the propagators held
// only at checkpoints (CkptRun): the forward pass gives Q2, QC, lnQ and the
// ensemble weights; each piece [a, b) of [0, N) recomputed with its mirror
// [N-b, N-a) holds q(s) and q^dagger(N-s) for every s of both pieces, whose
// products are Kahan-accumulated per point with the reference's Simpson
// weights (1 at s = 0, n1, N; 4, 2, 4, ... restarting after each block end;
// no odd-count correction), and likewise q^dagger(j) q^dagger(Nh-j) for the
// homopolymer.  Writes the replica's densities and phis as scft_props does;
// the context's full store is not touched.  Equal to scft_props up to the
// order of the FP64 sums.
scft_status scft_props_ckpt(scft_ctx *ctx, int ii, int K, double *lnQ_out, double *phis_out, double *bytes_out)
{
    if (!ctx || ii < 0 || ii >= ctx->strn || K < 1) return SCFT_BAD_INPUT;
    return props_ckpt_impl(ctx, ii, K, lnQ_out, phis_out, bytes_out);
}

}  // extern "C"

namespace {

// scft_props_ckpt for any replica slot of the context (the scratch replica of
// scft_props_host included)
scft_status props_ckpt_impl(scft_ctx *ctx, int ii, int K, double *lnQ_out, double *phis_out, double *bytes_out)
{
    const Geo &g = ctx->g;
    const int N = g.Ns, Nh = g.Nh, n1 = g.n1;
    const size_t M = g.M, T = ctx->prec == SCFT_FP32 ? 4 : 8;
    CkptRun R;
    scft_status s = ckpt_forward(ctx, ii, K, 6 * M * sizeof(double), R);
    if (s != SCFT_OK) return s;
    if (bytes_out) *bytes_out = R.bytes;
    double *acc = reinterpret_cast<double *>(R.extra);
    CK(cudaMemsetAsync(acc, 0, 6 * M * sizeof(double), ctx->st));
    // raw Simpson weights (density.h:404-422; the continuous A fraction moves
    // theta of the junction step's trapezoid weight from B to A)
    auto wA = [&](int t) {
        double w = (t == 0) + (t == n1);
        if (t > 0 && t < n1) w += ((t - 1) & 1) ? 2 : 4;
        if (g.jon && (t == n1 || t == n1 + 1)) w += 1.5 * g.theta;
        return w;
    };
    auto wB = [&](int t) {
        double w = (t == n1) + (t == N);
        if (t > n1 && t < N) w += ((t - n1 - 1) & 1) ? 2 : 4;
        if (g.jon && (t == n1 || t == n1 + 1)) w -= 1.5 * g.theta;
        return w;
    };
    auto wH = [&](int j) {
        double w = (j == 0) + (j == Nh);
        if (j > 0 && j < Nh) w += ((j - 1) & 1) ? 2 : 4;
        return w;
    };
    // element offset of slice `sl`, field `fld` of a slice-pair buffer inside ck_mem
    auto off = [&](const unsigned char *buf, int sl, int fld) {
        return (long long)((buf - R.ck) / T) + (long long)sl * 2 * (long long)M + (long long)fld * (long long)M;
    };
    DensPairs P;
    std::memset(&P, 0, sizeof(P));
    auto flush = [&]() {
        if (P.n == 0) return;
        ctx->stats.kernel_launches += T == 4 ? launch_density_acc<float>((const float *)R.ck, M, P, acc,
                                                                         ctx->L.red_blocks, ctx->st)
                                             : launch_density_acc<double>((const double *)R.ck, M, P, acc,
                                                                          ctx->L.red_blocks, ctx->st);
        P.n = 0;
    };
    auto add = [&](long long x, long long y, double a, double b, double h) {
        if (P.n == kDensPairs) flush();
        P.x[P.n] = x;
        P.y[P.n] = y;
        P.wA[P.n] = a;
        P.wB[P.n] = b;
        P.wH[P.n] = h;
        P.n++;
    };
    auto cp = [&](void *dst, const void *src) {
        return cudaMemcpyAsync(dst, src, R.pairB, cudaMemcpyDeviceToDevice, ctx->st);
    };
    // pieces with their mirrors: products x(t) y(n - t), x in field fx, y in field 1
    auto sweep = [&](const std::vector<int> &b, int n, bool homo) -> scft_status {
        for (size_t k = 0; k + 1 < b.size(); k++) {
            const int a0 = b[k], a1 = b[k + 1], m0 = n - a1, m1 = n - a0;
            if (a0 > m0) continue;  // right half: done as a mirror
            const bool self = (a0 == m0);
            cudaError_t e = cp(R.seg, R.ck + R.row_of[a0] * R.pairB);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "checkpoint copy");
            ckpt_chain(ctx, a0, a1 - a0, R.seg, 2);
            if (!self) {
                e = cp(R.segB, R.ck + R.row_of[m0] * R.pairB);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "checkpoint copy");
                ckpt_chain(ctx, m0, m1 - m0, R.segB, 2);
            }
            const unsigned char *mir = self ? R.seg : R.segB;  // holds slices m0 .. m1
            const int fx = homo ? 1 : 0;
            for (int t = a0; t < a1; t++) {  // y(n - t) in (m0, m1]
                const int u = n - t;
                add(off(R.seg, t - a0, fx), off(mir, u - m0, 1), homo ? 0 : wA(t), homo ? 0 : wB(t), homo ? wH(t) : 0);
            }
            if (!self)
                for (int t = m0; t < m1; t++) {  // y(n - t) in (a0, a1]
                    const int u = n - t;
                    add(off(R.segB, t - m0, fx), off(R.seg, u - a0, 1), homo ? 0 : wA(t), homo ? 0 : wB(t),
                        homo ? wH(t) : 0);
                }
            flush();  // the next piece overwrites the segments
        }
        return SCFT_OK;
    };
    s = sweep(R.bc, N, false);
    if (s != SCFT_OK) return s;
    if (Nh > 0) {
        s = sweep(R.bh, Nh, true);
        if (s != SCFT_OK) return s;
    }
    // end points: q(N) q^dagger(0) and q^dagger(Nh) q^dagger(0) (slice 0 is the
    // first checkpoint; q(N) and q^dagger(Nh) were kept by the forward pass)
    const unsigned char *c0 = R.ck + R.row_of[0] * R.pairB;
    add(off(R.qb + R.pairB, 0, 0), off(c0, 0, 1), wA(N), wB(N), 0);
    add(off(R.qb, 0, 1), off(c0, 0, 1), 0, 0, wH(Nh));
    flush();
    ctx->stats.kernel_launches += launch_density_final(acc, M, ctx->rs + (size_t)ii * kRsStride, 1.0 / N,
                                                       ctx->p.chi, ctx->conc + (size_t)ii * 4 * M, ctx->partials,
                                                       ctx->L.red_blocks, ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&ctx->rs_h[(size_t)ii * kRsStride], ctx->rs + (size_t)ii * kRsStride,
                       sizeof(double) * kRsStride, cudaMemcpyDeviceToHost, ctx->st));
    s = check_device_err(ctx);
    if (s != SCFT_OK) return s;
    if (lnQ_out) *lnQ_out = rsv(ctx, ii, kRsLnQ);
    if (phis_out)
        for (int k = 0; k < 5; k++) phis_out[k] = rsv(ctx, ii, kRsPhis + k);
    return SCFT_OK;
}

}  // namespace

extern "C" {

// d lnQ/df of replica ii at its current fields with a continuous A fraction
// (fcont): f moves the junction inside q's step n1 = floor(N f), whose field is
// theta wA + (1-theta) wB with theta = N f - n1, so d/df = N d/dtheta and only
// QC depends on f:  dQC/dtheta = (1/M) <q^dagger(N-1-n1), dS_J/dtheta q(n1)>
// (the adjoint of the junction step, stress_kernels.cu).  dF/df = -d lnQ/df
// at a converged saddle point.
scft_status scft_dF_df(scft_ctx *ctx, int ii, double *dlnQ_df, double *dF_df)
{
    if (!ctx || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    if (ctx->nostore) {
        ctx->lasterr = "scft_dF_df needs the full propagator store (context created with nostore)";
        return SCFT_UNSUPPORTED;
    }
    const Geo &g = ctx->g;
    if (!g.jon) {
        ctx->lasterr = "scft_dF_df: needs a continuous A fraction (scft_problem.fcont = 1)";
        return SCFT_BAD_INPUT;
    }
    scft_status s = stress_alloc(ctx);
    if (s != SCFT_OK) return s;
    const size_t T = ctx->prec == SCFT_FP32 ? 4 : 8;
    if (!ctx->jd_rbuf) CK(cudaMalloc(&ctx->jd_rbuf, T * 6 * (size_t)g.M));
    s = props_list(ctx, {ii});
    if (s != SCFT_OK) return s;
    const int slot = ctx->slot_of[ii];
    const double QC = rsv(ctx, ii, kRsQC), zC = rsv(ctx, ii, kRsZC);
    StressPairs P;
    std::memset(&P, 0, sizeof(P));
    P.n = 1;
    P.xs[0] = g.n1;                  // q(n1), the junction step's input
    P.xf[0] = 0;
    P.ys[0] = g.Ns - 1 - g.n1;       // q^dagger(N-1-n1), its adjoint
    P.yf[0] = 1;
    P.sel[0] = 2;
    const double *wm = ctx->W + (size_t)ii * 2 * ctx->M;
    int nl;
    if (T == 4) {
        StressArgs<float> a{g, slot, (const float *)ctx->hist, (const float *)ctx->etab,
                            (const cplx<float> *)ctx->tw, (const float *)ctx->kfac + (size_t)ii * ctx->kf_n,
                            (cplx<float> *)ctx->st_S4, (cplx<float> *)ctx->st_S2,
                            (cplx<float> *)ctx->st_S4p, ctx->st_part,
                            {ctx->Dr[3 * (size_t)ii], ctx->Dr[3 * (size_t)ii + 1], ctx->Dr[3 * (size_t)ii + 2]}, (float)(1.0 / g.M), ctx->err};
        a.jtab = (const float *)ctx->jtab;
        a.rbuf = (float *)ctx->jd_rbuf;
        a.wminus = wm;
        nl = launch_junction_dtheta<float>(a, P, ctx->rt_slab_threads, ctx->rt_slab_smem, ctx->rt_pencil_threads,
                                           ctx->rt_pencil_smem, ctx->partials, ctx->L.red_blocks, ctx->redout,
                                           ctx->st);
    } else {
        StressArgs<double> a{g, slot, (const double *)ctx->hist, (const double *)ctx->etab,
                             (const cplx<double> *)ctx->tw, (const double *)ctx->kfac + (size_t)ii * ctx->kf_n,
                             (cplx<double> *)ctx->st_S4, (cplx<double> *)ctx->st_S2,
                             (cplx<double> *)ctx->st_S4p, ctx->st_part,
                             {ctx->Dr[3 * (size_t)ii], ctx->Dr[3 * (size_t)ii + 1], ctx->Dr[3 * (size_t)ii + 2]}, 1.0 / g.M, ctx->err};
        a.jtab = (const double *)ctx->jtab;
        a.rbuf = (double *)ctx->jd_rbuf;
        a.wminus = wm;
        nl = launch_junction_dtheta<double>(a, P, ctx->rt_slab_threads, ctx->rt_slab_smem, ctx->rt_pencil_threads,
                                            ctx->rt_pencil_smem, ctx->partials, ctx->L.red_blocks, ctx->redout,
                                            ctx->st);
    }
    ctx->stats.kernel_launches += nl;
    CK(cudaGetLastError());
    double sum = 0;
    CK(cudaMemcpyAsync(&sum, ctx->redout, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    s = check_device_err(ctx);
    if (s != SCFT_OK) return s;
    const double dQC = sum / g.M;  // dQC/dtheta
    // lnQ = phic ln QC + ... (ens 1, density.h:390); zB Q2 + zC QC (ens 2, density.h:398)
    const double dth = ctx->p.ens == 1 ? ctx->p.phidb * dQC / QC : zC * dQC;
    const double d = g.Ns * dth;
    if (dlnQ_df) *dlnQ_df = d;
    if (dF_df) *dF_df = -d;
    return SCFT_OK;
}

// All parameter derivatives of replica ii at its current fields in one call:
// dF/dL (scft_stress), dF/dchiN (scft_dF_dchi) and, for a continuous A
// fraction, dF/df (scft_dF_df); dF/df is NaN otherwise (f enters the
// reference discretisation only through the integer n1).
scft_status scft_gradients(scft_ctx *ctx, int ii, double *dF_dL, double *dF_dchi, double *dF_df)
{
    if (!ctx || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    scft_status s = scft_stress(ctx, ii, nullptr, dF_dL);
    if (s == SCFT_OK && dF_dchi) s = scft_dF_dchi(ctx, ii, dF_dchi);
    if (s == SCFT_OK && dF_df) {
        if (ctx->g.jon)
            s = scft_dF_df(ctx, ii, nullptr, dF_df);
        else
            *dF_df = std::nan("");
    }
    return s;
}

// Anderson-accelerated solution of replica ii's field equations (no
// reference counterpart; the reference keeps only its scaffolding,
// scft.cu:30-31): residual d = (chi (phiB - phiA) - 2 W-, chi (phiA + phiB - 1))
// as in scft.cu:605-607, history of up to nhist previous (W, d), least squares
// in FP64 on the host over the device-computed Gram matrix of the residuals,
// W <- (W_k + lam d_k) - sum_i theta_i ((W_k + lam d_k) - (W_i + lam d_i)),
// with the history restarted every 16 nhist iterations.
scft_status scft_anderson_solve(scft_ctx *ctx, int ii, int maxIter, double tol, int nhist, double lam,
                                int *iters, double *err_out)
{
    if (!ctx || ii < 0 || ii >= ctx->strn || maxIter < 1 || nhist < 1 || nhist > 30 || !(lam > 0))
        return SCFT_BAD_INPUT;
    const size_t n2M = 2 * (size_t)ctx->M;
    const int H = nhist + 1;
    if (ctx->and_H < H) {
        if (ctx->and_X) cudaFree(ctx->and_X);
        if (ctx->and_D) cudaFree(ctx->and_D);
        ctx->and_X = ctx->and_D = nullptr;
        CK(cudaMalloc(&ctx->and_X, sizeof(double) * n2M * H));
        CK(cudaMalloc(&ctx->and_D, sizeof(double) * n2M * H));
        ctx->and_H = H;
    }
    std::vector<double> G((size_t)H * H, 0.0);
    std::vector<int> hist;  // slots of previous iterates, most recent first
    double err = 0;
    int it = 0;
    scft_status s;
    for (; it < maxIter; it++) {
        s = props_list(ctx, {ii});
        if (s != SCFT_OK) return s;
        s = upload_list(ctx, {ii});
        if (s != SCFT_OK) return s;
        launch_dev(field_args(ctx, ctx->rep_dev), 1, kRedBlocks, 0, 0.0, ctx->st);
        s = reduce_rows(ctx, 2, kRedBlocks);
        if (s != SCFT_OK) return s;
        err = std::sqrt(ctx->red_h[0] / (double)n2M);
        if (!(err == err)) {
            ctx->lasterr = "anderson: residual is NaN";
            return SCFT_NAN_DETECTED;
        }
        if (err <= tol) break;
        const int k = it % H;
        // restart: the history is cleared every 16 nhist iterations (a stale
        // history stalls the extrapolation on slowly ordering 3-D states)
        if (it > 0 && it % (16 * nhist) == 0) hist.clear();
        double *W = ctx->W + (size_t)ii * n2M;
        CK(cudaMemcpyAsync(ctx->and_X + (size_t)k * n2M, W, sizeof(double) * n2M, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->and_D + (size_t)k * n2M, ctx->DEV + (size_t)ii * n2M, sizeof(double) * n2M,
                           cudaMemcpyDeviceToDevice, ctx->st));
        hist.erase(std::remove(hist.begin(), hist.end(), k), hist.end());
        if ((int)hist.size() > nhist) hist.resize(nhist);
        std::vector<int> dslots(1, k);
        dslots.insert(dslots.end(), hist.begin(), hist.end());
        launch_hist_dots(ctx->and_D, n2M, k, dslots.data(), (int)dslots.size(), kRedBlocks, ctx->partials, ctx->st);
        s = reduce_rows(ctx, (int)dslots.size(), kRedBlocks);
        if (s != SCFT_OK) return s;
        for (size_t j = 0; j < dslots.size(); j++) G[(size_t)k * H + dslots[j]] = G[(size_t)dslots[j] * H + k] = ctx->red_h[j];
        const int m = (int)hist.size();
        std::vector<double> theta(m, 0.0);
        if (m > 0) {
            // U theta = v, U_ij = <d_k - d_i, d_k - d_j>, v_i = <d_k, d_k - d_i>
            std::vector<double> U((size_t)m * m), v(m);
            const double gkk = G[(size_t)k * H + k];
            for (int a = 0; a < m; a++) {
                const int ia = hist[a];
                v[a] = gkk - G[(size_t)k * H + ia];
                for (int b = 0; b < m; b++) {
                    const int ib = hist[b];
                    U[(size_t)a * m + b] = gkk - G[(size_t)k * H + ia] - G[(size_t)k * H + ib] + G[(size_t)ia * H + ib];
                }
            }
            double tr = 0;
            for (int a = 0; a < m; a++) tr += U[(size_t)a * m + a];
            for (int a = 0; a < m; a++) U[(size_t)a * m + a] += 1e-12 * tr + 1e-300;
            // Gaussian elimination with partial pivoting
            for (int c = 0; c < m; c++) {
                int piv = c;
                for (int r = c + 1; r < m; r++)
                    if (std::fabs(U[(size_t)r * m + c]) > std::fabs(U[(size_t)piv * m + c])) piv = r;
                if (piv != c) {
                    for (int j = 0; j < m; j++) std::swap(U[(size_t)c * m + j], U[(size_t)piv * m + j]);
                    std::swap(v[c], v[piv]);
                }
                for (int r = c + 1; r < m; r++) {
                    const double fct = U[(size_t)r * m + c] / U[(size_t)c * m + c];
                    for (int j = c; j < m; j++) U[(size_t)r * m + j] -= fct * U[(size_t)c * m + j];
                    v[r] -= fct * v[c];
                }
            }
            for (int r = m - 1; r >= 0; r--) {
                double t = v[r];
                for (int j = r + 1; j < m; j++) t -= U[(size_t)r * m + j] * theta[j];
                theta[r] = t / U[(size_t)r * m + r];
            }
        }
        launch_anderson_update(W, ctx->and_X, ctx->and_D, n2M, k, m, hist.data(), theta.data(), lam, ctx->st);
        ctx->stats.kernel_launches += 2;
        CK(cudaGetLastError());
        hist.insert(hist.begin(), k);
        if ((int)hist.size() > nhist) hist.resize(nhist);
    }
    CK(cudaStreamSynchronize(ctx->st));
    if (iters) *iters = it;
    if (err_out) *err_out = err;
    return SCFT_OK;
}

// Variable-cell relaxation of replica ii: `inner` SCFT iterations (the
// solve_field loop restricted to this replica, scft.cu:598-608, without the
// periodic FreeE) or, with inner <= 0, an Anderson re-solve to RMS 1e-9; then
// the replica's own box L_i -= gamma dF/dL_i with each relative change capped
// at 2 %, until max |dF/dL_i| <= stressTol.
scft_status scft_relax_cell(scft_ctx *ctx, int ii, int maxOuter, int inner, double stressTol, double gamma,
                            int *outer_out, double *stress_out)
{
    if (!ctx || ii < 0 || ii >= ctx->strn || maxOuter < 1 || !(gamma > 0)) return SCFT_BAD_INPUT;
    double dF[3] = {0, 0, 0};
    int outer = 0;
    scft_status s = SCFT_OK;
    for (; outer < maxOuter; outer++) {
        if (inner <= 0) {  // Anderson re-solve of the fields at the current box
            int it = 0;
            double e = 0;
            s = scft_anderson_solve(ctx, ii, 3000, 1e-9, 12, 0.1, &it, &e);
            if (s != SCFT_OK) return s;
        } else {
            s = scft_string_begin(ctx, ii, inner, 1e-3);
            if (s != SCFT_OK) return s;
            ctx->sf.skip_freee = true;
            for (int k = 0; k < inner; k++) {
                int done = 0;
                s = scft_string_step(ctx, nullptr, nullptr, nullptr, &done);
                if (s != SCFT_OK) return s;
                if (done) break;
            }
            scft_string_end(ctx, nullptr);
        }
        s = scft_stress(ctx, ii, nullptr, dF);
        if (s != SCFT_OK) return s;
        const double mx = std::max(std::fabs(dF[0]), std::max(std::fabs(dF[1]), std::fabs(dF[2])));
        if (mx <= stressTol) break;
        double D[3];
        for (int i = 0; i < 3; i++) {
            const double Di = ctx->Dr[3 * (size_t)ii + i];
            double step = -gamma * dF[i];
            const double cap = 0.02 * Di;
            step = std::max(-cap, std::min(cap, step));
            D[i] = Di + step;
        }
        s = scft_set_box_replica(ctx, ii, D);
        if (s != SCFT_OK) return s;
    }
    if (outer_out) *outer_out = outer;
    if (stress_out)
        for (int i = 0; i < 3; i++) stress_out[i] = dF[i];
    return SCFT_OK;
}

// dF/d(chi N) at the saddle point: F = -lnQ + <W-^2>/chi - <W+> + chi/4 there
// (the reference's F, scft.cu:823-826, with chi (phiB - phiA) = 2 W- and
// phiA + phiB = 1), so dF/dchi = 1/4 - <W-^2>/chi^2.
scft_status scft_dF_dchi(scft_ctx *ctx, int ii, double *out)
{
    if (!ctx || !out || ii < 0 || ii >= ctx->strn) return SCFT_BAD_INPUT;
    std::vector<double> w(2 * (size_t)ctx->M);
    scft_status s = scft_get_fields(ctx, ii, w.data());
    if (s != SCFT_OK) return s;
    double q = 0;
    for (int r = 0; r < ctx->M; r++) q += w[r] * w[r];
    q /= ctx->M;
    *out = 0.25 - q / (ctx->p.chi * ctx->p.chi);
    return SCFT_OK;
}

scft_status scft_get_stats(const scft_ctx *ctx, scft_stats *st)
{
    if (!ctx || !st) return SCFT_BAD_INPUT;
    *st = ctx->stats;
    return SCFT_OK;
}

scft_status scft_timer_mark(scft_ctx *ctx, int slot)
{
    if (!ctx || slot < 0 || slot > 3) return SCFT_BAD_INPUT;
    CK(cudaEventRecord(ctx->tev[slot], ctx->st));
    return SCFT_OK;
}

scft_status scft_timer_elapsed(scft_ctx *ctx, int a, int b, double *ms)
{
    if (!ctx || !ms || a < 0 || a > 3 || b < 0 || b > 3) return SCFT_BAD_INPUT;
    CK(cudaEventSynchronize(ctx->tev[b]));
    float f = 0;
    CK(cudaEventElapsedTime(&f, ctx->tev[a], ctx->tev[b]));
    *ms = f;
    return SCFT_OK;
}

scft_status scft_reset_stats(scft_ctx *ctx)
{
    if (!ctx) return SCFT_BAD_INPUT;
    ctx->stats = scft_stats{};
    return SCFT_OK;
}

// Times props rounds of every replica for each schedule -- one, two or four
// slot groups (two concurrent streams; four groups run two after another on
// each), x-pencil tiles of the default or twice the width (when the grid has
// tensor-map pencils), four launches or one persistent launch per contour
// step -- and keeps the fastest.  Each
// candidate re-captures its graphs, runs one untimed round, then the best of
// three timed rounds counts.  The rounds recompute every replica's densities
// at its current fields, so the state a caller sees afterwards is unchanged;
// the statistics are restored.
scft_status scft_autotune_ex(scft_ctx *ctx, int *groups_out, int *wide_out, int *persist_out, double *times_ms)
{
    if (!ctx) return SCFT_BAD_INPUT;
    if (times_ms)
        for (int c = 0; c < kTuneCandidates; c++) times_ms[c] = -1;
    if (ctx->nostore) {  // props run one replica at a time from checkpoints: nothing to schedule
        if (groups_out) *groups_out = 1;
        if (wide_out) *wide_out = ctx->L.ptile_wide;
        if (persist_out) *persist_out = 0;
        return SCFT_OK;
    }
    const scft_stats keep = ctx->stats;
    std::vector<int> all(ctx->strn);
    for (int i = 0; i < ctx->strn; i++) all[i] = i;
    auto drop_graphs = [&]() {
        for (auto &g : ctx->graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    };
    double best = 0;
    int best_g = 1, best_w = 0, best_p = 0;
    bool first = true;
    // axes: slot groups (1, 2, 4) x x-pencil tile width (default, wide;
    // tensor-map pencils of the shared-memory kernels only) x launches per
    // contour step (four, or one persistent launch); c = gi + 3 wide + 6 persist
    const int nw = (!ctx->L.reg && ctx->L.tmap_wide) ? 2 : 1;
    const int np = ctx->persist_ok ? 2 : 1;
    for (int c = 0; c < kTuneCandidates; c++) {
        const int ng = 1 << (c % 3), wide = (c / 3) & 1, persist = c / 6;
        if (wide >= nw || persist >= np) continue;
        if (effective_groups(ng, (int)all.size()) != ng) continue;  // props_list would run fewer groups
        drop_graphs();
        ctx->ngroups = ng;
        ctx->L.ptile_wide = wide;
        ctx->L.persist = persist;
        scft_status s = props_list(ctx, all);
        if (s != SCFT_OK) return s;
        double t = 1e300;
        for (int r = 0; r < 3; r++) {
            const double before = ctx->stats.props_seconds;
            s = props_list(ctx, all);
            if (s != SCFT_OK) return s;
            t = std::min(t, (ctx->stats.props_seconds - before) * 1e3);
        }
        if (times_ms) times_ms[c] = t;
        if (first || t < best) {
            first = false;
            best = t;
            best_g = ng;
            best_w = wide;
            best_p = persist;
        }
    }
    drop_graphs();
    ctx->ngroups = best_g;
    ctx->L.ptile_wide = best_w;
    ctx->L.persist = best_p;
    ctx->stats = keep;
    if (groups_out) *groups_out = best_g;
    if (wide_out) *wide_out = best_w;
    if (persist_out) *persist_out = best_p;
    return SCFT_OK;
}

scft_status scft_autotune(scft_ctx *ctx, int *groups_out, int *wide_out, double *times_ms)
{
    double t[kTuneCandidates];
    scft_status s = scft_autotune_ex(ctx, groups_out, wide_out, nullptr, t);
    if (times_ms) {  // four launches per step: (1, default), (2, default), (1, wide), (2, wide)
        times_ms[0] = t[0];
        times_ms[1] = t[1];
        times_ms[2] = t[3];
        times_ms[3] = t[4];
    }
    return s;
}

// ---- binary FP64 checkpoint (no reference counterpart: the reference keeps
// only the ASCII win files, scft.cu:785-788).  Layout, host byte order:
//   "SCFTCKP1" | u32 version (2) | u32 P = sizeof(scft_problem) | P bytes of
//   scft_problem (with the last common box) | i32 strn | i64 M | strn x 2M
//   doubles (W-, W+) | strn x 3 doubles (each replica's box) | u64 FNV-1a hash
//   of the field and box bytes.  Version 1 has no per-replica boxes.
// scft_problem only ever grows at its end, so the reader takes a problem block
// of any size that covers m and D: fields missing from a shorter (older)
// block read as 0, their defaults, and the tail of a longer one is skipped.
namespace {
constexpr char kCkptMagic[8] = {'S', 'C', 'F', 'T', 'C', 'K', 'P', '1'};
constexpr uint64_t kFnvBasis = 1469598103934665603ull;
constexpr uint32_t kMaxProblemBytes = 1u << 16;

uint64_t fnv1a(uint64_t h, const void *data, size_t n)
{
    const unsigned char *b = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

struct CkptFile {
    uint32_t version = 0;
    scft_problem p;
    int32_t strn = 0;
    int64_t M = 0;
    std::vector<double> fields, boxes;  // fields only when asked for
};

// reads and checks a checkpoint file; on failure returns false with `why`
bool read_checkpoint(const char *path, bool keep_fields, CkptFile &c, std::string &why)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        why = std::string("cannot open ") + path;
        return false;
    }
    auto fail = [&](const char *w) {
        fclose(f);
        why = w;
        return false;
    };
    char magic[8];
    uint32_t psz = 0;
    std::memset(&c.p, 0, sizeof(c.p));
    if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kCkptMagic, 8) != 0) return fail("not a checkpoint");
    if (fread(&c.version, 4, 1, f) != 1 || (c.version != 1 && c.version != 2) || fread(&psz, 4, 1, f) != 1)
        return fail("unsupported version");
    if (psz < offsetof(scft_problem, N) || psz > kMaxProblemBytes) return fail("unsupported problem block");
    const size_t take = std::min<size_t>(psz, sizeof(scft_problem));
    if (fread(&c.p, take, 1, f) != 1) return fail("truncated header");
    if (psz > take && fseek(f, (long)(psz - take), SEEK_CUR) != 0) return fail("truncated header");
    if (fread(&c.strn, 4, 1, f) != 1 || fread(&c.M, 8, 1, f) != 1) return fail("truncated header");
    const int64_t Mg = (int64_t)c.p.m[0] * c.p.m[1] * c.p.m[2];
    if (c.strn < 1 || c.p.m[0] < 1 || c.p.m[1] < 1 || c.p.m[2] < 1 || c.M != Mg) return fail("inconsistent header");
    const size_t nf = 2 * (size_t)c.M * (size_t)c.strn;
    uint64_t hh = kFnvBasis;
    if (keep_fields) {
        c.fields.resize(nf);
        if (fread(c.fields.data(), sizeof(double), nf, f) != nf) return fail("truncated fields");
        hh = fnv1a(hh, c.fields.data(), nf * sizeof(double));
    } else {
        std::vector<double> chunk(1 << 17);
        for (size_t done = 0; done < nf;) {
            const size_t n = std::min(chunk.size(), nf - done);
            if (fread(chunk.data(), sizeof(double), n, f) != n) return fail("truncated fields");
            hh = fnv1a(hh, chunk.data(), n * sizeof(double));
            done += n;
        }
    }
    c.boxes.clear();
    if (c.version == 2) {
        c.boxes.resize(3 * (size_t)c.strn);
        if (fread(c.boxes.data(), sizeof(double), c.boxes.size(), f) != c.boxes.size())
            return fail("truncated boxes");
        hh = fnv1a(hh, c.boxes.data(), c.boxes.size() * sizeof(double));
    }
    uint64_t h = 0;
    if (fread(&h, 8, 1, f) != 1) return fail("truncated hash");
    if (h != hh) return fail("hash mismatch");
    fclose(f);
    return true;
}
}  // namespace

scft_status scft_save_checkpoint(scft_ctx *ctx, const char *path)
{
    if (!ctx || !path) return SCFT_BAD_INPUT;
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) {
        ctx->lasterr = "scft_save_checkpoint: cannot open " + tmp;
        return SCFT_BAD_INPUT;
    }
    const uint32_t ver = 2, psz = sizeof(scft_problem);
    const int32_t strn = ctx->strn;
    const int64_t M = ctx->M;
    bool ok = fwrite(kCkptMagic, 1, 8, f) == 8 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&psz, 4, 1, f) == 1 &&
              fwrite(&ctx->p, psz, 1, f) == 1 && fwrite(&strn, 4, 1, f) == 1 && fwrite(&M, 8, 1, f) == 1;
    std::vector<double> w(2 * (size_t)M);
    uint64_t h = kFnvBasis;
    for (int ii = 0; ok && ii < ctx->strn; ii++) {
        scft_status s = scft_get_fields(ctx, ii, w.data());
        if (s != SCFT_OK) {
            fclose(f);
            std::remove(tmp.c_str());
            return s;
        }
        h = fnv1a(h, w.data(), w.size() * sizeof(double));
        ok = fwrite(w.data(), sizeof(double), w.size(), f) == w.size();
    }
    const size_t nb = 3 * (size_t)ctx->strn;
    h = fnv1a(h, ctx->Dr.data(), nb * sizeof(double));
    ok = ok && fwrite(ctx->Dr.data(), sizeof(double), nb, f) == nb;
    ok = ok && fwrite(&h, 8, 1, f) == 1;
    ok = (fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        ctx->lasterr = std::string("scft_save_checkpoint: write failed: ") + path;
        return SCFT_BAD_INPUT;
    }
    return SCFT_OK;
}

scft_status scft_load_checkpoint(scft_ctx *ctx, const char *path)
{
    if (!ctx || !path) return SCFT_BAD_INPUT;
    CkptFile c;
    std::string why;
    if (!read_checkpoint(path, true, c, why)) {
        ctx->lasterr = "scft_load_checkpoint: " + why;
        return SCFT_BAD_INPUT;
    }
    if (c.strn != ctx->strn || c.M != (int64_t)ctx->M || c.p.m[0] != ctx->p.m[0] || c.p.m[1] != ctx->p.m[1] ||
        c.p.m[2] != ctx->p.m[2]) {
        ctx->lasterr = "scft_load_checkpoint: grid or replica count differs from the context";
        return SCFT_BAD_INPUT;
    }
    scft_status s = scft_set_box(ctx, c.p.D);
    if (s != SCFT_OK) return s;
    for (int ii = 0; ii < (int)c.boxes.size() / 3; ii++) {
        s = scft_set_box_replica(ctx, ii, &c.boxes[3 * (size_t)ii]);
        if (s != SCFT_OK) return s;
    }
    for (int ii = 0; ii < c.strn; ii++) {
        s = scft_set_fields(ctx, ii, c.fields.data() + (size_t)ii * 2 * c.M);
        if (s != SCFT_OK) return s;
    }
    return SCFT_OK;
}

// header of a checkpoint file, checked as scft_load_checkpoint checks it (hash
// included), with no context and no device
scft_status scft_checkpoint_info(const char *path, int *version, int *strn, int *m, double *D)
{
    if (!path) return SCFT_BAD_INPUT;
    CkptFile c;
    std::string why;
    if (!read_checkpoint(path, false, c, why)) return SCFT_BAD_INPUT;
    if (version) *version = (int)c.version;
    if (strn) *strn = c.strn;
    for (int i = 0; i < 3; i++) {
        if (m) m[i] = c.p.m[i];
        if (D) D[i] = c.p.D[i];
    }
    return SCFT_OK;
}

}  // extern "C"
