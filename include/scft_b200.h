/*
 * scft_b200.h -- C ABI of the B200 (sm_100a) SCFT string-method field solver.
 *
 * Drop-in boundary for the hot path of PolymerTheory/SCFT_string: the
 * Richardson pseudo-spectral propagator, the composite-Simpson density sum,
 * the field mixing and the cubic-spline string reparametrisation
 * (solve_field and what it calls).  Plain C types only; every function
 * returns a status and never exits the process (the reference calls
 * exit(EXIT_FAILURE) on any CUDA error, GPU_kernels.h:16-48).
 *
 * Conventions (identical to the reference):
 *   grid point  r = z + m2*(y + m1*x)                    (scft.cu:462-464)
 *   replica fields are host arrays of doubles: [W-, W+] (2*M) and the
 *   concentrations [phiA, phiB, phih, phicB] (4*M)   (scft.cu:1037-1051)
 *
 * Ownership and threading: a context owns one CUDA stream and all device
 * memory it uses; the caller owns every host buffer.  A context is not
 * thread-safe; separate contexts may be used from separate threads.
 * The library runs only on sm_100a (B200); there is no CPU fallback.
 */
#ifndef SCFT_B200_H
#define SCFT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SCFT_OK = 0,
    SCFT_CUDA_ERROR = 1,     /* a CUDA call failed; see scft_last_error */
    SCFT_NAN_DETECTED = 2,   /* a residual became NaN (the reference asserts, scft.cu:539) */
    SCFT_BAD_INPUT = 3,      /* invalid argument or unsupported size */
    SCFT_TIMEOUT = 4,        /* a bounded device wait gave up */
    SCFT_OUT_OF_MEMORY = 5,
    SCFT_UNSUPPORTED = 6     /* no sm_100a device */
} scft_status;

typedef enum { SCFT_FP64 = 0, SCFT_FP32 = 1 } scft_precision;

/* Problem definition: the input.dat keys of the reference (scft.cu:120-251)
 * plus the replica count (compile-time `strn` in the reference, scft.cu:35). */
typedef struct {
    int    m[3];        /* mesh points per axis */
    double D[3];        /* box lengths in units of R0 */
    int    N;           /* contour steps of the copolymer */
    double alpha;       /* homopolymer/copolymer length ratio (Nh = (int)(alpha*N)) */
    int    ens;         /* 1 canonical, 2 grand canonical */
    double phidb;       /* copolymer volume fraction (ens 1) or fugacity (ens 2) */
    double chi;         /* chi*N */
    double f;           /* A fraction of the copolymer; rounded to round(N f)/N as scft.cu:1008
                         * unless fcont */
    int    strn;        /* replicas on the string, 1..64 */
    int    fix[2];      /* keep the first / last replica fixed */
    int    dostring;    /* 1: string method, 0: independent replicas */
    int    springsteps; /* initial iterations with spring coupling (missing win files) */
    int    precision;   /* scft_precision of the propagator bulk (reductions are FP64) */
    int    batched;     /* 1: all replicas advance together; 0: one replica at a time */
    int    device;      /* CUDA device ordinal */
    int    fcont;       /* 0: the reference's rounded f.  1: continuous A fraction (no
                         * reference counterpart): n1 = floor(N f) whole A steps, and step
                         * n1 sees the field theta wA + (1-theta) wB, theta = N f - n1, with
                         * theta of its Simpson weight moved from B to A; needs Nh < N - n1 */
    int    nostore;     /* 0: every props keeps all N+1 propagator slices (the reference's
                         * dev_qq).  1: no full store: props runs from checkpoints every ckpt_K
                         * contour steps (scft_props_ckpt), one replica at a time, about twice
                         * the work in a fraction of the memory; scft_stress uses the
                         * checkpointed adjoint; scft_do_step, scft_get_propagator and
                         * scft_dF_df return SCFT_UNSUPPORTED */
    int    ckpt_K;      /* checkpoint interval with nostore (0: ceil(sqrt(N))) */
} scft_problem;

typedef struct scft_ctx scft_ctx;

/* One record per solve_field iteration (scft.cu:592-806). */
typedef struct {
    int    k;
    double lambda;
    double errtot;      /* sqrt(mean over replicas of errs3^2), scft.cu:764-765 */
    double fitup;
    double stepav;      /* mean props calls per replica in this iteration */
    int    did_freee;   /* FreeE ran at the end of this iteration (k % 50 == 0 or last) */
    double FE;          /* total free energy of that FreeE */
} scft_iter_report;

typedef struct {
    long long props_calls;    /* replica props evaluations */
    long long contour_steps;  /* replica contour steps (Ns per props) */
    long long kernel_launches;
    double    props_seconds;  /* device time of props batches (CUDA events) */
} scft_stats;

/* ---- lifetime --------------------------------------------------------- */
/* Replaces `new density(N, D)` + setupSplineBuffers (scft.cu:1010-1011,
 * density.h:272-315, 462-476). */
scft_status scft_create(const scft_problem *p, scft_ctx **out);
void        scft_destroy(scft_ctx *ctx);
const char *scft_last_error(const scft_ctx *ctx);
const char *scft_status_string(scft_status s);

/* ---- fields ----------------------------------------------------------- */
/* Replica ii's [W-, W+] (2*M doubles): the first 2*M entries of W[ii]
 * (scft.cu:1062). */
scft_status scft_set_fields(scft_ctx *ctx, int ii, const double *w2M);
scft_status scft_get_fields(const scft_ctx *ctx, int ii, double *w2M);
/* Fields and boxes of every replica of src into ctx (no reference
 * counterpart): device to device, for contexts of the same grid and replica
 * count, e.g. an FP32 context handing its string to an FP64 one for the last
 * iterations of a solve.  Waits for src's stream. */
scft_status scft_copy_fields(scft_ctx *ctx, const scft_ctx *src);
/* Concentrations of the last props of replica ii: [phiA, phiB, phih, phicB]
 * (4*M doubles, W[ii]+2M of the reference), lnQ and phis[5]. */
scft_status scft_get_conc(const scft_ctx *ctx, int ii, double *out4M, double *lnQ, double *phis);
/* Replica ownership mask of the single process (doiis, scft.cu:953-975). */
scft_status scft_get_doiis(const scft_ctx *ctx, int *doiis);

/* ---- density ---------------------------------------------------------- */
/* density::props on the device-resident fields of replica ii
 * (density.h:344-459). */
scft_status scft_props(scft_ctx *ctx, int ii);
/* density::props with the reference's host-pointer signature
 * (density.h:344): w[0:2M) in, w[2M:6M) out; ii is unused as in the
 * reference; Ns, alpha, phic and f must match the context (BAD_INPUT
 * otherwise). */
scft_status scft_props_host(scft_ctx *ctx, double *w, double *lnQ, int ii, int Ns, double alpha,
                            double phic, double *phis, double f);
/* One Richardson contour step (step::do_step, density.h:129-220) of the
 * host slice in = [q, q^dagger] (2*M doubles) for the fields of replica ii
 * -> out (2*M doubles). */
scft_status scft_do_step(scft_ctx *ctx, int ii, const double *in, double *out, int s);
/* Propagator slice of the last props of replica ii: which 0 = q(s), 1 = q^dagger(s). */
scft_status scft_get_propagator(const scft_ctx *ctx, int ii, int which, int s, double *outM);

/* ---- solvers ---------------------------------------------------------- */
/* solve_field0 (scft.cu:516-554) on replica ii; *k_out = the reference's k. */
scft_status scft_solve_field0(scft_ctx *ctx, int ii, int maxIter, double errTol, int *k_out);
/* W+ relaxation of every replica (the prelude of main, scft.cu:1105). */
scft_status scft_solve_field0_all(scft_ctx *ctx, int maxIter, double errTol, int *k_out);
/* solve_field (scft.cu:559-809), doii = -1 for the whole string.  reports
 * (maxIter entries), errs and errs3 (maxIter*strn doubles) may be NULL. */
scft_status scft_solve_field(scft_ctx *ctx, int doii, int maxIter, double errTol,
                             scft_iter_report *reports, double *errs, double *errs3, int *k_out);
/* Iteration-at-a-time form of scft_solve_field: begin, then step until the
 * reference loop would stop (*done set), then end. */
scft_status scft_string_begin(scft_ctx *ctx, int doii, int maxIter, double errTol);
scft_status scft_string_step(scft_ctx *ctx, scft_iter_report *rep, double *errs, double *errs3,
                             int *done);
scft_status scft_string_end(scft_ctx *ctx, int *k_out);
/* scft_string_begin with the iteration counter set to k0 (no reference
 * counterpart): continues a string run from fields saved at iteration k0
 * (scft_save_checkpoint, or host copies), so that the FreeE cadence
 * (k % 50 == 0, scft.cu:761, 778) and the spring steps (k < springsteps,
 * scft.cu:594) follow the uninterrupted run.  The mixing parameter restarts
 * at 0.05, the value the reference's loop keeps (scft.cu:563, 793-797). */
scft_status scft_string_resume(scft_ctx *ctx, int doii, int maxIter, double errTol, int k0);
/* FreeE (scft.cu:812-853): W+ re-solve (100 iterations, 1e-4) and props of
 * every replica, then F = -lnQ + <chi phiA phiB - wA phiA - wB phiB>.
 * Arrays have strn entries; any may be NULL. */
scft_status scft_free_energy(scft_ctx *ctx, double *FE, double *FEs, double *FEs0, double *FEs1,
                             double *phctot, double *alf);

/* Results of the last FreeE evaluation (inside scft_solve_field every 50
 * iterations, or scft_free_energy) without recomputing; any may be NULL. */
scft_status scft_last_free_energy(const scft_ctx *ctx, double *FE, double *FEs, double *FEs0,
                                  double *FEs1, double *phctot, double *alf);

/* ---- box, stress and parameter derivatives (no reference counterpart) -- */
/* Box lengths D (the reference's D[3], used by setup_k_sq, density.h:79-95). */
scft_status scft_set_box(scft_ctx *ctx, const double *D);
scft_status scft_get_box(const scft_ctx *ctx, double *D);
/* The box of one replica: every replica of a context may own its cell (the
 * diffusion factors are kept per replica); scft_set_box sets all of them. */
scft_status scft_set_box_replica(scft_ctx *ctx, int ii, const double *D);
scft_status scft_get_box_replica(const scft_ctx *ctx, int ii, double *D);
/* d lnQ/dL_i of replica ii at its current fields by the adjoint of the
 * Richardson propagator (q^dagger is the adjoint of q's chain), and the box
 * stress dF/dL_i = -d lnQ/dL_i, exact at a converged saddle point.  Either
 * output may be NULL. */
scft_status scft_stress(scft_ctx *ctx, int ii, double *dlnQ_dL, double *dF_dL);
/* The same derivatives with the propagators held only at checkpoints at most
 * K contour steps apart (K ~ sqrt(N)): one forward pass keeps the checkpoint
 * slices, then every segment is recomputed once next to its mirror segment
 * (two chain passes in all).  Device memory: *bytes_out (may be NULL) instead
 * of the (N+1) slice pairs of the full store; the context's full store is not
 * touched.  Same values as scft_stress up to the order of the FP64 sums. */
scft_status scft_stress_ckpt(scft_ctx *ctx, int ii, int K, double *dlnQ_dL, double *dF_dL,
                             double *bytes_out);
/* d lnQ/df and dF/df = -d lnQ/df (exact at a converged saddle point) of
 * replica ii, for a context created with fcont = 1: the adjoint of the
 * junction step, whose field depends on f.  Either output may be NULL. */
scft_status scft_dF_df(scft_ctx *ctx, int ii, double *dlnQ_df, double *dF_df);
/* dF/dL_i (3 values), dF/dchiN and dF/df of replica ii in one call (the
 * gradients entry of the proposed ABI); dF/df needs fcont = 1 and is NaN
 * otherwise.  Exact at a converged saddle point; any output may be NULL. */
scft_status scft_gradients(scft_ctx *ctx, int ii, double *dF_dL, double *dF_dchi, double *dF_df);
/* density::props of replica ii (the same results as scft_props, up to the
 * order of the FP64 sums) with the propagators held only at checkpoints at
 * most K contour steps apart: a forward pass keeps the checkpoints, then every
 * segment is recomputed once next to its mirror segment and the Simpson terms
 * q(s) q^dagger(N-s) are accumulated per point.  Device memory: *bytes_out
 * (may be NULL); the context's full store is not touched.  lnQ_out and
 * phis_out[5] as scft_get_conc (either may be NULL). */
scft_status scft_props_ckpt(scft_ctx *ctx, int ii, int K, double *lnQ_out, double *phis_out, double *bytes_out);
/* Anderson-accelerated solution of replica ii's field equations (an option
 * beside the reference's simple mixing; no reference counterpart): residual
 * as scft.cu:605-607 without spring or string terms, history of nhist
 * (1..30) iterates restarted every 16 nhist iterations, FP64 least squares,
 * mixing parameter lam.  Stops when the
 * RMS residual <= tol; *iters = props evaluations, *err_out = last RMS. */
scft_status scft_anderson_solve(scft_ctx *ctx, int ii, int maxIter, double tol, int nhist, double lam,
                                int *iters, double *err_out);
/* Variable-cell relaxation of replica ii in its own box: `inner` iterations of the
 * solve_field loop on that replica (no FreeE), then a gradient step on the
 * box, L_i -= gamma dF/dL_i (each relative change capped at 2 %), until
 * max_i |dF/dL_i| <= stressTol or maxOuter rounds; inner <= 0 re-solves the
 * fields by Anderson mixing (to 1e-9) instead.  *outer_out = rounds run,
 * stress_out[3] = last dF/dL. */
scft_status scft_relax_cell(scft_ctx *ctx, int ii, int maxOuter, int inner, double stressTol,
                            double gamma, int *outer_out, double *stress_out);
/* dF/d(chi N) of replica ii at a converged saddle point: 1/4 - <W-^2>/chi^2. */
scft_status scft_dF_dchi(scft_ctx *ctx, int ii, double *out);

/* ---- string spline services (host pointers) --------------------------- */
/* density::splineDerivsChunked (density.h:491-508): ww[ii] -> W- of replica
 * ii; out[ii][r0..r0+n) = dW-/dalpha at knot x[ii] for doiis[ii] == 1. */
scft_status scft_spline_derivs(scft_ctx *ctx, const double *x, const double *const *ww, int r0,
                               int n, const int *doiis, double *const *out);
/* density::splineRedistChunked (density.h:511-528): ww[ii][r] += lambda *
 * (S(xref[ii]) - ww[ii][r]) for interior replicas with doiis[ii] == 1. */
scft_status scft_spline_redist(scft_ctx *ctx, const double *x, const double *xref,
                               double *const *ww, int r0, int n, const int *doiis, double lambda);

/* ---- allocation-free step (no counterpart in the reference) ------------ */
/* One Richardson contour step for callers that cannot allocate device memory
 * when they need a step: a real-time loop that must not stall on the
 * allocator (cudaMalloc can synchronise the device), or a framework that owns
 * every device allocation through its own pool.  Same kernels and result as
 * scft_do_step, but every working buffer lives in one static __device__
 * array of 4.2 MB, so it calls no cudaMalloc/cudaFree.  All pointers are the
 * caller's device memory: w2M = [W-, W+], in2M = [q(s), q^dagger(s)], out2M =
 * [q(s+1), q^dagger(s+1)], each 2*M doubles; f is the A fraction (0..1) as in
 * scft_problem; stream may be NULL.  Limits: FP64, M <= 32768, each m_i <= 64
 * (BAD_INPUT beyond).  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress).  Calls share the array, so calls that
 * overlap on the GPU race.  The call reads the kernels' error word back to
 * the host and waits for its stream before returning, so it cannot be
 * recorded into a CUDA graph. */
scft_status scft_do_step_noalloc(const int *m, const double *D, int N, double f, const double *w2M,
                                 const double *in2M, double *out2M, int s, void *stream);

/* ---- failure-path self-test (no reference counterpart) ----------------- */
/* Runs one bounded device wait on a barrier that no copy completes, so the
 * wait gives up after `polls` polls exactly as a wait on a lost bulk copy
 * would (the step kernels allow 2^20 polls).  Returns SCFT_TIMEOUT and clears
 * the error word, leaving the context usable; for tests of the error path. */
scft_status scft_selftest_timeout(scft_ctx *ctx, int polls);

/* ---- statistics (no reference counterpart) ---------------------------- */
/* Records CUDA event `slot` (0..3) on the context's stream; elapsed device
 * time between two recorded slots (waits for the later one). */
scft_status scft_timer_mark(scft_ctx *ctx, int slot);
scft_status scft_timer_elapsed(scft_ctx *ctx, int slot_a, int slot_b, double *ms);
scft_status scft_get_stats(const scft_ctx *ctx, scft_stats *st);
scft_status scft_reset_stats(scft_ctx *ctx);

/* Binary FP64 checkpoint (no reference counterpart; the ASCII win files stay
 * the drop-in format): problem record with the current box, the fields and
 * the box of every replica, and a hash of the field and box bytes.  Loading
 * checks the grid and replica count against the context and the hash, then
 * sets boxes and fields.  Files of earlier versions and of shorter (older) or
 * longer problem records load too: the record only grows at its end. */
scft_status scft_save_checkpoint(scft_ctx *ctx, const char *path);
scft_status scft_load_checkpoint(scft_ctx *ctx, const char *path);
/* The header of a checkpoint file, checked as scft_load_checkpoint checks the
 * file (hash included) but with no context and no device: format version,
 * replica count, m[3] and the common box D[3].  Any output may be NULL;
 * BAD_INPUT for a file that cannot be opened or that a load would refuse for
 * its content. */
scft_status scft_checkpoint_info(const char *path, int *version, int *strn, int *m, double *D);
/* Picks the schedule of a props round by timing rounds of all replicas at
 * their current fields: 1 or 2 concurrent slot groups, and x-pencil tiles of
 * the default or twice the width (grids with tensor-map pencils), each with
 * four launches per contour step and, where the context has it, one
 * persistent launch per step (see scft_autotune_ex).  The densities are
 * recomputed, the statistics left unchanged.  *groups_out, *wide_out = the
 * setting kept; times_ms[0..3] = best round time with four launches per step
 * for (1 group, default tile), (2, default), (1, wide), (2, wide), -1 where
 * not available (any pointer may be NULL).  Performance-only: results do not
 * depend on the setting. */
scft_status scft_autotune(scft_ctx *ctx, int *groups_out, int *wide_out, double *times_ms);
/* scft_autotune over more schedules: 1, 2 or 4 slot groups (four groups run
 * two after another on each of the two streams, so fewer spectra are live
 * at once; only with at least 16 replicas, and batches of fewer than 16
 * replicas then run as 2 groups), the two tile widths, and four
 * launches per contour step or one persistent launch per step (work items
 * claimed in order, bounded waits) where the context has one (compile-time
 * grid shapes).  times_ms[12]: times_ms[c] for c = gi + 3 wide + 6 persist
 * with gi = 0, 1, 2 for 1, 2, 4 groups, -1 where not available;
 * *persist_out = the launch form kept.  Performance-only: results do not
 * depend on the setting. */
scft_status scft_autotune_ex(scft_ctx *ctx, int *groups_out, int *wide_out, int *persist_out, double *times_ms);

#ifdef __cplusplus
}
#endif
#endif
