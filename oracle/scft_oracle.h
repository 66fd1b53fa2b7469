/*
 * scft_oracle.h -- FP64 CPU restatement of the SCFT_string field-solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * in scft_string_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it.  Nothing in the
 * product links against it.
 *
 * Every function restates the reference algorithm (PolymerTheory/SCFT_string)
 * and cites the file:line it follows.  The one component that the reference
 * takes from a closed library, the 3-D real FFT (cuFFT D2Z/Z2D, density.h:67-74),
 * is replaced here by a project-written mixed-radix Stockham FFT with the same
 * conventions (unnormalised, forward sign -1, half spectrum along the last axis).
 *
 * Layout conventions (identical to the reference):
 *   real grid     r  = z + m2*(y + m1*x)                  (scft.cu:462-464)
 *   half spectrum k  = kz + (m2/2+1)*(ky + m1*kx)         (density.h:90)
 *   complex data is interleaved (re, im) doubles.
 *   replica field  W[ii] = [W-, W+, phiA, phiB, phih, phicB, dWda], 7*M doubles
 *                                                          (scft.cu:1037-1051)
 */
#ifndef SCFT_ORACLE_H
#define SCFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- FFT ---- */
typedef struct oc_grid oc_grid;

/* m[3] mesh points, D[3] box lengths (units of R0).  Returns NULL when a mesh
 * size has a prime factor above 7 or is < 1. */
oc_grid *oc_grid_create(const int m[3], const double D[3]);
void     oc_grid_destroy(oc_grid *g);
int      oc_grid_M(const oc_grid *g);
int      oc_grid_Mk(const oc_grid *g);

/* 1-D complex FFT of length n (in place, interleaved), sign -1 forward, +1 inverse,
 * unnormalised.  Used by the FFT unit tests. */
int  oc_fft1d(int n, double *x, int sign);
/* 3-D real-to-half-complex forward transform (cufftExecD2Z semantics). */
void oc_fft_r2c(const oc_grid *g, const double *in, double *out);
/* 3-D half-complex-to-real inverse transform (cufftExecZ2D semantics;
 * unnormalised; the input is not modified). */
void oc_fft_c2r(const oc_grid *g, const double *in, double *out);
/* k^2 table, density.h:79-95 (Mk doubles). */
void oc_ksq(const oc_grid *g, double *ksq);

/* ------------------------------------------------------------ density ---- */
typedef struct oc_density oc_density;

/* density(Ns, D) of density.h:272-315 (plus step(D), density.h:41-75). */
oc_density *oc_density_create(const int m[3], const double D[3], int Ns);
void        oc_density_destroy(oc_density *d);
/* step::prepareFactors, density.h:118-125 with the kernels of
 * GPU_kernels.h:207-225.  W2M = [W-, W+]. */
void oc_prepare_factors(oc_density *d, double ds, const double *W2M);
/* step::do_step, density.h:129-220: in/out are [q, q^dagger] (2*M doubles). */
void oc_do_step(oc_density *d, const double *in, double *out, int s, int n1, int n2);
/* density::props, density.h:344-459.  w: in w[0:2M) = [W-, W+]; out
 * w[2M:6M) = [phiA, phiB, phih, phicB].  phis[5] = <rC>,<rA>,<rB>,<rhA>,<rhB>.
 * ens is the reference global `ens` (1 canonical, 2 grand canonical).
 * Returns 0, or -1 for an ens outside {1,2}. */
int  oc_props(oc_density *d, double *w, double *lnQ, int Ns, double alpha,
              double phic, double *phis, double f, int ens);
/* the continuous-f variant of oc_props (no reference counterpart; the
   restatement of scft_problem.fcont): f is not rounded, the junction step
   n1 = floor(Ns f) sees theta wA + (1 - theta) wB */
int  oc_props_fcont(oc_density *d, double *w, double *lnQ, int Ns, double alpha,
                    double phic, double *phis, double f, int ens);
/* d lnQ / d L_i of the fields w2M (W-, W+) by the adjoint of the Richardson
   step applied in real space (no reference counterpart; the restatement of
   scft_stress); runs oc_props first */
int  oc_stress(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f,
               int ens, double dlnQ_dL[3]);
/* oc_stress for the continuous-f variant: the chain of oc_props_fcont, with
   the junction step's tables at q's step n1 */
int  oc_stress_fcont(oc_density *d, const double *w2M, int Ns, double alpha, double phic,
                     double f, int ens, double dlnQ_dL[3]);
/* d lnQ / df of the continuous-f variant (the restatement of scft_dF_df):
   Ns times the derivative of lnQ in the junction step's theta, with
   dS/dtheta applied in real space; runs oc_props_fcont first.  Returns -1
   where oc_props_fcont does. */
int  oc_dlnq_df(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f,
                int ens, double *dlnQ_df);
/* Propagator slice access after oc_props: which=0 -> q(s), 1 -> q^dagger(s). */
const double *oc_density_q(const oc_density *d, int which, int s);
/* Q2 = <q^dagger(Nh)>, QC = <q(Ns)> of the last props call. */
void oc_density_Q(const oc_density *d, double *Q2, double *QC);

/* The single-block tree reduction of GPU_kernels.h:58-90 launched <<<1,1024>>>,
 * restated in its exact summation order. */
double oc_reduction_sum(const double *a, int n);

/* ------------------------------------------------------------- spline ---- */
/* density::splineDerivsChunked (density.h:491-508) with cubefit_chunk_g and
 * eval_spline_deriv_chunk_g (GPU_kernels.h:232-306) restated per point.
 * ww[ii] points at replica ii's W- (only [r0, r0+n) is read). */
void oc_spline_derivs(int strn, const double *x, double *const *ww, int r0, int n,
                      const int *doiis, double *const *out);
/* density::splineRedistChunked (density.h:511-528) with eval_spline_value_chunk_g
 * (GPU_kernels.h:308-329). Updates interior replicas with doiis==1 in place. */
void oc_spline_redist(int strn, const double *x, const double *xref, double *const *ww,
                      int r0, int n, const int *doiis, double lambda);
/* Coefficients of one point's natural spline (c, b, d, a per knot). */
void oc_spline_coeffs(int strn, const double *x, const double *a, double *c, double *b,
                      double *d);

/* ------------------------------------------------------------- solver ---- */
typedef struct {
    int    m[3];
    double D[3];
    int    N;          /* contour steps (reference global N) */
    double alpha;      /* homopolymer / copolymer length ratio */
    int    ens;        /* 1 canonical, 2 grand canonical */
    double phidb;      /* copolymer volume fraction (ens 1) or fugacity (ens 2) */
    double chi;        /* chi*N */
    double f;          /* A fraction, rounded to n1/N by the caller as scft.cu:1008 */
    int    strn;       /* replicas on the string (reference compile-time strn) */
    int    fix[2];
    int    dostring;
    int    springsteps;
} oc_problem;

typedef struct oc_solver oc_solver;

/* Per-iteration record of solve_field (scft.cu:592-806). */
typedef struct {
    int    k;
    double lambda;
    double errtot;      /* sqrt(mean errs3^2), scft.cu:764-765 */
    double fitup;
    double stepav;
    int    did_freee;   /* FreeE was evaluated at the end of this iteration */
    double FE;          /* its total (valid when did_freee) */
} oc_iter_record;

oc_solver *oc_solver_create(const oc_problem *p);
void       oc_solver_destroy(oc_solver *s);
/* W[ii] (7*M doubles, reference layout). */
double    *oc_solver_W(oc_solver *s, int ii);
int       *oc_solver_doiis(oc_solver *s);
/* solve_field0, scft.cu:516-554.  Returns the reference's k. */
int  oc_solve_field0(oc_solver *s, int ii, int maxIter, double errTol);
/* solve_field, scft.cu:559-809.  rec (may be NULL) receives one record per
 * iteration (capacity maxIter); errs_out/errs3_out (may be NULL) receive the
 * strn errors of every iteration (maxIter*strn doubles each).  Returns k. */
int  oc_solve_field(oc_solver *s, int doii, int maxIter, double errTol,
                    oc_iter_record *rec, double *errs_out, double *errs3_out);
/* FreeE, scft.cu:812-853 (single process).  FEs/FEs0/FEs1/phctot/alf: strn each. */
double oc_free_energy(oc_solver *s, double *alf, double *FEs0, double *FEs1, double *FEs,
                      double *phctot);
/* Number of props calls made so far (all replicas). */
long oc_solver_props_calls(const oc_solver *s);
/* Last values of FreeE for the drop-in FEs file. */
const double *oc_solver_alf(const oc_solver *s);

/* EDist, scft.cu:351-355 over M points. */
double oc_edist(const double *a, const double *b, int M);

/* Worker threads used by the OpenMP loops (0 = library default). */
void oc_set_threads(int n);
int  oc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
