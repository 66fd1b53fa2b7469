/*
 * scft_oracle.c -- FP64 CPU restatement of the SCFT_string field-solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never the product).  See
 * scft_oracle.h for the layout conventions.  Citations are file:line into the
 * reference project PolymerTheory/SCFT_string (scft.cu, density.h,
 * GPU_kernels.h).
 *
 * Parallelism: OpenMP over independent FFT lines and grid points.  All sums
 * are evaluated serially in the reference's order, so results do not depend
 * on the thread count.
 */
#include "scft_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.14159265358979323846264338327950288;

void oc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ===================================================================== FFT
 * Mixed-radix Stockham autosort FFT.  Stage with radix R and accumulated size
 * Ns: butterfly j reads src[j + r*n/R] (r < R), multiplies by
 * exp(sign*2*pi*i*r*(j%Ns)/(Ns*R)), does an R-point DFT and writes
 * dst[(j/Ns)*Ns*R + j%Ns + r*Ns].  Natural order in, natural order out.
 * Replaces cuFFT (closed library, called by density.h:149-205). */
typedef struct {
    int     n;
    int     nst;
    int     radix[40];
    double *tw; /* 2n: exp(-2 pi i t / n) */
} oc_plan1;

static int plan_init(oc_plan1 *p, int n)
{
    int rem = n, k = 0;
    static const int pr[] = {4, 2, 3, 5, 7};
    if (n < 1) return -1;
    for (int i = 0; i < 5; i++)
        while (rem % pr[i] == 0) {
            p->radix[k++] = pr[i];
            rem /= pr[i];
        }
    if (rem != 1) return -1;
    p->n = n;
    p->nst = k;
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int t = 0; t < n; t++) {
        double a = 2.0 * PI * (double)t / (double)n;
        p->tw[2 * t] = cos(a);
        p->tw[2 * t + 1] = -sin(a);
    }
    return 0;
}

static void plan_free(oc_plan1 *p)
{
    free(p->tw);
    p->tw = NULL;
}

/* x: 2n interleaved; work: 2n scratch.  Result in x.  Radix-2 and radix-4
 * butterflies are written out; radix 3, 5 and 7 use the direct R-point DFT. */
static void fft_line(const oc_plan1 *p, double *x, double *work, int sign)
{
    const int n = p->n;
    double *src = x, *dst = work;
    int Ns = 1;
    const double sg = sign < 0 ? 1.0 : -1.0; /* conjugates the stored twiddles for sign +1 */
    double vr[8], vi[8];
    for (int st = 0; st < p->nst; st++) {
        const int R = p->radix[st];
        const int nR = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < nR; j++) {
            const int k = j % Ns;
            for (int r = 0; r < R; r++) {
                const double ar = src[2 * (j + r * nR)], ai = src[2 * (j + r * nR) + 1];
                if (r == 0 || k == 0) {
                    vr[r] = ar;
                    vi[r] = ai;
                } else {
                    const int t = r * k * tstep;
                    const double wr = p->tw[2 * t], wi = sg * p->tw[2 * t + 1];
                    vr[r] = ar * wr - ai * wi;
                    vi[r] = ar * wi + ai * wr;
                }
            }
            const int idxD = (j / Ns) * Ns * R + k;
            double *o = dst + 2 * idxD;
            if (R == 2) {
                o[0] = vr[0] + vr[1];
                o[1] = vi[0] + vi[1];
                o[2 * Ns] = vr[0] - vr[1];
                o[2 * Ns + 1] = vi[0] - vi[1];
            } else if (R == 4) {
                const double ar = vr[0] + vr[2], ai = vi[0] + vi[2];
                const double br = vr[0] - vr[2], bi = vi[0] - vi[2];
                const double cr = vr[1] + vr[3], ci = vi[1] + vi[3];
                /* (sign * i) * (v1 - v3) */
                const double dr = -(double)sign * (vi[1] - vi[3]), di = (double)sign * (vr[1] - vr[3]);
                o[0] = ar + cr;
                o[1] = ai + ci;
                o[2 * Ns] = br + dr;
                o[2 * Ns + 1] = bi + di;
                o[4 * Ns] = ar - cr;
                o[4 * Ns + 1] = ai - ci;
                o[6 * Ns] = br - dr;
                o[6 * Ns + 1] = bi - di;
            } else {
                for (int q = 0; q < R; q++) {
                    double sr = 0, si = 0;
                    for (int r = 0; r < R; r++) {
                        const int t = ((r * q) % R) * nR;
                        const double wr = p->tw[2 * t], wi = sg * p->tw[2 * t + 1];
                        sr += vr[r] * wr - vi[r] * wi;
                        si += vr[r] * wi + vi[r] * wr;
                    }
                    o[2 * q * Ns] = sr;
                    o[2 * q * Ns + 1] = si;
                }
            }
        }
        double *tmp = src;
        src = dst;
        dst = tmp;
        Ns *= R;
    }
    if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

int oc_fft1d(int n, double *x, int sign)
{
    oc_plan1 p;
    if (plan_init(&p, n)) return -1;
    double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    fft_line(&p, x, w, sign);
    free(w);
    plan_free(&p);
    return 0;
}

struct oc_grid {
    int      m[3];
    int      M, Mk, mk2;
    double   D[3];
    oc_plan1 p[3];
};

oc_grid *oc_grid_create(const int m[3], const double D[3])
{
    oc_grid *g = (oc_grid *)calloc(1, sizeof(oc_grid));
    for (int i = 0; i < 3; i++) {
        g->m[i] = m[i];
        g->D[i] = D[i];
        if (plan_init(&g->p[i], m[i])) {
            for (int j = 0; j < i; j++) plan_free(&g->p[j]);
            free(g);
            return NULL;
        }
    }
    g->M = m[0] * m[1] * m[2];
    g->mk2 = m[2] / 2 + 1;
    g->Mk = m[0] * m[1] * g->mk2; /* scft.cu:1006 */
    return g;
}

void oc_grid_destroy(oc_grid *g)
{
    if (!g) return;
    for (int i = 0; i < 3; i++) plan_free(&g->p[i]);
    free(g);
}

int oc_grid_M(const oc_grid *g) { return g->M; }
int oc_grid_Mk(const oc_grid *g) { return g->Mk; }

/* complex passes along x (axis 0) and y (axis 1) over the half spectrum */
static void pass_xy(const oc_grid *g, double *h, int sign)
{
    const int m0 = g->m[0], m1 = g->m[1], mk2 = g->mk2;
    /* y lines: for each (x, kz) */
#pragma omp parallel
    {
        int nmax = m0 > m1 ? m0 : m1;
        double *line = (double *)malloc(sizeof(double) * 4 * (size_t)nmax);
        double *work = line + 2 * nmax;
        if (sign < 0) {
#pragma omp for collapse(2) schedule(static)
            for (int x = 0; x < m0; x++)
                for (int kz = 0; kz < mk2; kz++) {
                    double *base = h + 2 * ((size_t)x * m1 * mk2 + kz);
                    for (int y = 0; y < m1; y++) {
                        line[2 * y] = base[2 * (size_t)y * mk2];
                        line[2 * y + 1] = base[2 * (size_t)y * mk2 + 1];
                    }
                    fft_line(&g->p[1], line, work, sign);
                    for (int y = 0; y < m1; y++) {
                        base[2 * (size_t)y * mk2] = line[2 * y];
                        base[2 * (size_t)y * mk2 + 1] = line[2 * y + 1];
                    }
                }
        }
#pragma omp for collapse(2) schedule(static)
        for (int y = 0; y < m1; y++)
            for (int kz = 0; kz < mk2; kz++) {
                double *base = h + 2 * ((size_t)y * mk2 + kz);
                const size_t st = (size_t)m1 * mk2;
                for (int x = 0; x < m0; x++) {
                    line[2 * x] = base[2 * x * st];
                    line[2 * x + 1] = base[2 * x * st + 1];
                }
                fft_line(&g->p[0], line, work, sign);
                for (int x = 0; x < m0; x++) {
                    base[2 * x * st] = line[2 * x];
                    base[2 * x * st + 1] = line[2 * x + 1];
                }
            }
        if (sign > 0) {
#pragma omp for collapse(2) schedule(static)
            for (int x = 0; x < m0; x++)
                for (int kz = 0; kz < mk2; kz++) {
                    double *base = h + 2 * ((size_t)x * m1 * mk2 + kz);
                    for (int y = 0; y < m1; y++) {
                        line[2 * y] = base[2 * (size_t)y * mk2];
                        line[2 * y + 1] = base[2 * (size_t)y * mk2 + 1];
                    }
                    fft_line(&g->p[1], line, work, sign);
                    for (int y = 0; y < m1; y++) {
                        base[2 * (size_t)y * mk2] = line[2 * y];
                        base[2 * (size_t)y * mk2 + 1] = line[2 * y + 1];
                    }
                }
        }
        free(line);
    }
}

void oc_fft_r2c(const oc_grid *g, const double *in, double *out)
{
    const int m0 = g->m[0], m1 = g->m[1], m2 = g->m[2], mk2 = g->mk2;
#pragma omp parallel
    {
        double *line = (double *)malloc(sizeof(double) * 4 * (size_t)m2);
        double *work = line + 2 * m2;
#pragma omp for schedule(static)
        for (int xy = 0; xy < m0 * m1; xy++) {
            const double *src = in + (size_t)xy * m2;
            for (int z = 0; z < m2; z++) {
                line[2 * z] = src[z];
                line[2 * z + 1] = 0.0;
            }
            fft_line(&g->p[2], line, work, -1);
            memcpy(out + 2 * (size_t)xy * mk2, line, sizeof(double) * 2 * (size_t)mk2);
        }
        free(line);
    }
    pass_xy(g, out, -1);
}

void oc_fft_c2r(const oc_grid *g, const double *in, double *out)
{
    const int m0 = g->m[0], m1 = g->m[1], m2 = g->m[2], mk2 = g->mk2;
    double *h = (double *)malloc(sizeof(double) * 2 * (size_t)g->Mk);
    memcpy(h, in, sizeof(double) * 2 * (size_t)g->Mk);
    pass_xy(g, h, +1);
#pragma omp parallel
    {
        double *line = (double *)malloc(sizeof(double) * 4 * (size_t)m2);
        double *work = line + 2 * m2;
#pragma omp for schedule(static)
        for (int xy = 0; xy < m0 * m1; xy++) {
            const double *src = h + 2 * (size_t)xy * mk2;
            /* Hermitian extension of the half line; the imaginary parts of the
             * self-conjugate bins drop out of the real part taken below. */
            for (int k = 0; k < m2; k++) {
                if (k < mk2) {
                    line[2 * k] = src[2 * k];
                    line[2 * k + 1] = src[2 * k + 1];
                } else {
                    line[2 * k] = src[2 * (m2 - k)];
                    line[2 * k + 1] = -src[2 * (m2 - k) + 1];
                }
            }
            fft_line(&g->p[2], line, work, +1);
            double *dst = out + (size_t)xy * m2;
            for (int z = 0; z < m2; z++) dst[z] = line[2 * z];
        }
        free(line);
    }
    free(h);
}

/* step::setup_k_sq, density.h:79-95 */
void oc_ksq(const oc_grid *g, double *ksq)
{
    const int *m = g->m;
    const double *DA = g->D;
    for (int k0 = -(m[0] - 1) / 2; k0 <= m[0] / 2; k0++) {
        const int K0 = (k0 < 0) ? (k0 + m[0]) : k0;
        double A0 = k0 * k0 / (DA[0] * DA[0]);
        for (int k1 = -(m[1] - 1) / 2; k1 <= m[1] / 2; k1++) {
            const int K1 = (k1 < 0) ? (k1 + m[1]) : k1;
            double A1 = A0 + k1 * k1 / (DA[1] * DA[1]);
            for (int k2 = 0; k2 <= m[2] / 2; k2++) {
                double A2 = A1 + k2 * k2 / (DA[2] * DA[2]);
                int k = k2 + (m[2] / 2 + 1) * (K1 + m[1] * K0);
                ksq[k] = 4 * PI * PI * A2;
            }
        }
    }
}

/* ================================================================ density */
struct oc_density {
    oc_grid *g;
    int      Ns;
    int      M, Mk;
    double  *ksq;                /* Mk */
    double  *expKsq, *expKsq2;   /* Mk each */
    double  *E2p1, *Ep1, *E2m1, *Em1; /* M each: e^{-wA ds/4}, e^{-wA ds/2}, wB ... */
    double  *E2j, *Ej;           /* M each: the junction step's tables (continuous f only) */
    double  *qs0, *qs1;          /* 2M each */
    double  *h;                  /* 2 fields * 2*Mk */
    double  *qq;                 /* 2*(Ns+1)*M: q(s) at 2sM, q^dagger(s) at (2s+1)M */
    double  *cs;                 /* 10*M concentrations of density.h:357 */
    double   Q2, QC;
};

oc_density *oc_density_create(const int m[3], const double D[3], int Ns)
{
    oc_grid *g = oc_grid_create(m, D);
    if (!g || Ns < 1) {
        oc_grid_destroy(g);
        return NULL;
    }
    oc_density *d = (oc_density *)calloc(1, sizeof(oc_density));
    d->g = g;
    d->Ns = Ns;
    d->M = g->M;
    d->Mk = g->Mk;
    size_t M = (size_t)d->M, Mk = (size_t)d->Mk;
    d->ksq = (double *)malloc(sizeof(double) * Mk);
    oc_ksq(g, d->ksq);
    d->expKsq = (double *)malloc(sizeof(double) * Mk);
    d->expKsq2 = (double *)malloc(sizeof(double) * Mk);
    d->E2p1 = (double *)malloc(sizeof(double) * 4 * M);
    d->Ep1 = d->E2p1 + M;
    d->E2m1 = d->E2p1 + 2 * M;
    d->Em1 = d->E2p1 + 3 * M;
    d->E2j = (double *)malloc(sizeof(double) * 2 * M);
    d->Ej = d->E2j + M;
    d->qs0 = (double *)malloc(sizeof(double) * 4 * M);
    d->qs1 = d->qs0 + 2 * M;
    d->h = (double *)malloc(sizeof(double) * 4 * Mk);
    d->qq = (double *)malloc(sizeof(double) * 2 * (size_t)(Ns + 1) * M);
    d->cs = (double *)malloc(sizeof(double) * 10 * M);
    return d;
}

void oc_density_destroy(oc_density *d)
{
    if (!d) return;
    oc_grid_destroy(d->g);
    free(d->ksq);
    free(d->expKsq);
    free(d->expKsq2);
    free(d->E2p1);
    free(d->E2j);
    free(d->qs0);
    free(d->h);
    free(d->qq);
    free(d->cs);
    free(d);
}

const double *oc_density_q(const oc_density *d, int which, int s)
{
    return d->qq + (size_t)(2 * s + (which ? 1 : 0)) * d->M;
}

void oc_density_Q(const oc_density *d, double *Q2, double *QC)
{
    *Q2 = d->Q2;
    *QC = d->QC;
}

/* step::prepareFactors, density.h:118-125; kernels GPU_kernels.h:207-225 */
void oc_prepare_factors(oc_density *d, double ds, const double *W)
{
    const int M = d->M, Mk = d->Mk;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Mk; k++) {
        d->expKsq2[k] = exp(-d->ksq[k] * ds / 12) / M;
        d->expKsq[k] = d->expKsq2[k] * d->expKsq2[k] * M;
    }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        d->E2p1[r] = exp(-(W[r] + W[r + M]) * ds / 4);
        d->Ep1[r] = d->E2p1[r] * d->E2p1[r];
        d->E2m1[r] = exp(-(-W[r] + W[r + M]) * ds / 4);
        d->Em1[r] = d->E2m1[r] * d->E2m1[r];
    }
}

static void fwd2(oc_density *d, const double *a) /* both fields -> h */
{
    oc_fft_r2c(d->g, a, d->h);
    oc_fft_r2c(d->g, a + d->M, d->h + 2 * (size_t)d->Mk);
}

static void inv2(oc_density *d, double *a)
{
    oc_fft_c2r(d->g, d->h, a);
    oc_fft_c2r(d->g, d->h + 2 * (size_t)d->Mk, a + d->M);
}

static void mult_k(oc_density *d, const double *K) /* Mult_self complex x real, GPU_kernels.h:175-181 */
{
    const int Mk = d->Mk;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < 2 * Mk; k++) {
        double v = K[k % Mk];
        d->h[2 * k] *= v;
        d->h[2 * k + 1] *= v;
    }
}

/* step::do_step, density.h:129-220, with the tables of q (E2q, Eq) and of
   q^dagger (E2d, Ed) for this step given */
static void do_step_tables(oc_density *d, const double *in, double *out, const double *E2q, const double *Eq,
                           const double *E2d, const double *Ed);

void oc_do_step(oc_density *d, const double *in, double *out, int s, int n1, int n2)
{
    const double *E2q = (s < n1) ? d->E2p1 : d->E2m1, *Eq = (s < n1) ? d->Ep1 : d->Em1;
    const double *E2d = (s < n2) ? d->E2m1 : d->E2p1, *Ed = (s < n2) ? d->Em1 : d->Ep1;
    do_step_tables(d, in, out, E2q, Eq, E2d, Ed);
}

static void do_step_tables(oc_density *d, const double *in, double *out, const double *E2q, const double *Eq,
                           const double *E2d, const double *Ed)
{
    const int M = d->M;
    double *qs0 = d->qs0, *qs1 = d->qs1;
    /* first half step (Mult, GPU_kernels.h:192-196) */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        qs0[r] = in[r] * E2q[r];
        qs0[r + M] = in[r + M] * E2d[r];
    }
    fwd2(d, qs0);
    mult_k(d, d->expKsq2);
    inv2(d, qs0);
    /* second half step (Mult_self real, GPU_kernels.h:184-189) */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        qs0[r] *= Eq[r];
        qs0[r + M] *= Ed[r];
    }
    fwd2(d, qs0);
    mult_k(d, d->expKsq2);
    inv2(d, qs0);
    /* full step */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        qs1[r] = in[r] * Eq[r];
        qs1[r + M] = in[r + M] * Ed[r];
    }
    fwd2(d, qs1);
    mult_k(d, d->expKsq);
    inv2(d, qs1);
    /* Richardson, GPU_kernels.h:199-203 */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        out[r] = (qs0[r] * E2q[r] * 4 - qs1[r] * Eq[r]) / 3;
        out[r + M] = (qs0[r + M] * E2d[r] * 4 - qs1[r + M] * Ed[r]) / 3;
    }
}

/* reduction_sum<<<1,1024>>>, GPU_kernels.h:58-90, in its exact order */
double oc_reduction_sum(const double *a, int n)
{
    enum { T = 1024 };
    double cache[T];
    for (int t = 0; t < T; t++) {
        double temp = 0;
        for (int i = t; i < n; i += T) temp += a[i];
        cache[t] = temp;
    }
    for (int i = T / 2; i != 0; i /= 2)
        for (int t = 0; t < i; t++) cache[t] += cache[t + i];
    return cache[0];
}

/* density::props, density.h:344-459.  fcont = 1 is the continuous-f variant
   (no reference counterpart): n1 = floor(Ns f) whole A steps; q's step n1 and
   q^dagger's step n2 - 1 see the field theta wA + (1 - theta) wB, theta = Ns f
   - n1; theta of that step's trapezoid weight moves from the B block to the A
   block of the Simpson sums.  At theta = 0 it is the reference
   discretisation. */
static int props_impl(oc_density *d, double *w, double *lnQ, int Ns, double alpha, double phic,
                      double *phis, double f, int ens, int fcont);

int oc_props(oc_density *d, double *w, double *lnQ, int Ns, double alpha, double phic,
             double *phis, double f, int ens)
{
    return props_impl(d, w, lnQ, Ns, alpha, phic, phis, f, ens, 0);
}

int oc_props_fcont(oc_density *d, double *w, double *lnQ, int Ns, double alpha, double phic,
                   double *phis, double f, int ens)
{
    return props_impl(d, w, lnQ, Ns, alpha, phic, phis, f, ens, 1);
}

static int props_impl(oc_density *d, double *w, double *lnQ, int Ns, double alpha, double phic,
                      double *phis, double f, int ens, int fcont)
{
    const int M = d->M;
    const int n1 = fcont ? (int)floor(Ns * f) : (int)round(Ns * f), n2 = Ns - n1, Nh = alpha * Ns;
    const double theta = fcont ? Ns * f - n1 : 0.0;
    const double ds = 1.0 / Ns;
    double Q1 = 0, Q2 = 0, QC = 0, zA = 0, zB = 0, zC = 0;
    double *c = d->cs;
    double *rA = c + 0 * (size_t)M, *rB = c + 1 * (size_t)M, *rh = c + 2 * (size_t)M,
           *rCB = c + 3 * (size_t)M, *rhA = c + 4 * (size_t)M, *rP = c + 5 * (size_t)M,
           *rM = c + 6 * (size_t)M, *rCA = c + 7 * (size_t)M, *rC = c + 8 * (size_t)M,
           *rhB = c + 9 * (size_t)M;
    if (ens != 1 && ens != 2) return -1;
    if (Ns > d->Ns || Nh > Ns || n1 < 0 || n1 > Ns) return -1;
    if (fcont && (n1 >= Ns || Nh > n2 - 1)) return -1;

    oc_prepare_factors(d, ds, w);
    if (fcont) {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < M; r++) { /* theta wA + (1 - theta) wB = W+ + (2 theta - 1) W- */
            d->E2j[r] = exp(-(w[r + M] + (2.0 * theta - 1.0) * w[r]) * ds / 4);
            d->Ej[r] = d->E2j[r] * d->E2j[r];
        }
    }
    double *q0 = d->qq;
    for (int r = 0; r < 2 * M; r++) q0[r] = 1.0; /* Array_set_value, density.h:368-369 */
    for (int s = 0; s < Ns; s++) {
        double *in = d->qq + (size_t)2 * s * M, *out = d->qq + (size_t)2 * (s + 1) * M;
        if (!fcont) {
            oc_do_step(d, in, out, s, n1, n2);
            continue;
        }
        const int jq = (s == n1), jd = (s == n2 - 1);
        const double *E2q = jq ? d->E2j : (s < n1) ? d->E2p1 : d->E2m1;
        const double *Eq = jq ? d->Ej : (s < n1) ? d->Ep1 : d->Em1;
        const double *E2d = jd ? d->E2j : (s < n2) ? d->E2m1 : d->E2p1;
        const double *Ed = jd ? d->Ej : (s < n2) ? d->Em1 : d->Ep1;
        do_step_tables(d, in, out, E2q, Eq, E2d, Ed);
    }

#define Q1S(s) (d->qq + (size_t)2 * (s) * M)
#define Q2S(s) (d->qq + (size_t)(2 * (s) + 1) * M)
    Q2 = oc_reduction_sum(Q2S(Nh), M);
    QC = oc_reduction_sum(Q1S(Ns), M);
    Q1 /= M;
    Q2 /= M;
    QC /= M;
    d->Q2 = Q2;
    d->QC = QC;
    if (ens == 1) { /* density.h:389-393 */
        *lnQ = phic * log(QC) + ((1.0 - phic) / alpha) * log(Q2);
        zA = 0;
        zB = (1.0 - phic) / (Q2 * alpha);
        zC = phic / QC;
    } else { /* density.h:394-398 */
        zA = 0;
        zB = 1.0;
        zC = phic;
        *lnQ = zA * Q1 + zB * Q2 + zC * QC;
    }
    /* rA_rB_init_Ns_homo, GPU_kernels.h:92-101 */
    {
        const double *q2Nh = Q2S(Nh), *q1Ns = Q1S(Ns), *q2Ns = Q2S(Ns), *q1n1 = Q1S(n1),
                     *q2n2 = Q2S(n2);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < M; r++) {
            rhA[r] = 0;
            rhB[r] = 2.0 * q2Nh[r];
            rCA[r] = q2Ns[r] + q1n1[r] * q2n2[r];
            rCB[r] = q1Ns[r] + q1n1[r] * q2n2[r];
        }
    }
    /* middle segments, density.h:404-422 with rA_rB_mid_segments (GPU_kernels.h:152-157) */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        int s, wt;
        for (s = 1, wt = 4; s < Nh; s++, wt = 6 - wt) rhA[r] += wt * Q1S(s)[r] * Q1S(Nh - s)[r];
        for (s = 1, wt = 4; s < Nh; s++, wt = 6 - wt) rhB[r] += wt * Q2S(s)[r] * Q2S(Nh - s)[r];
        for (s = 1, wt = 4; s < n1; s++, wt = 6 - wt) rCA[r] += wt * Q1S(s)[r] * Q2S(Ns - s)[r];
        for (s = n1 + 1, wt = 4; s < Ns; s++, wt = 6 - wt)
            rCB[r] += wt * Q1S(s)[r] * Q2S(Ns - s)[r];
        if (fcont) { /* theta of the junction step's trapezoid weight: B -> A */
            const double tj = 1.5 * theta * (Q1S(n1)[r] * Q2S(Ns - n1)[r] + Q1S(n1 + 1)[r] * Q2S(Ns - n1 - 1)[r]);
            rCA[r] += tj;
            rCB[r] -= tj;
        }
    }
    /* scale_concentrations (GPU_kernels.h:129-139) and sumconcs2 (GPU_kernels.h:114-127) */
#pragma omp parallel for schedule(static)
    for (int r = 0; r < M; r++) {
        rhA[r] = rhA[r] * zA * ds / 3.0;
        rhB[r] = rhB[r] * zB * ds / 3.0;
        rCA[r] = rCA[r] * zC * ds / 3.0;
        rCB[r] = rCB[r] * zC * ds / 3.0;
        rA[r] = rhA[r] + rCA[r];
        rB[r] = rhB[r] + rCB[r];
        rh[r] = rhA[r] + rhB[r];
        rC[r] = rCA[r] + rCB[r];
        rP[r] = rA[r] + rB[r] - 1.0;
        rM[r] = rA[r] - rB[r];
    }
#undef Q1S
#undef Q2S
    /* averages, density.h:433-454 */
    phis[1] = oc_reduction_sum(rA, M);
    phis[2] = oc_reduction_sum(rB, M);
    phis[0] = oc_reduction_sum(rC, M);
    phis[3] = oc_reduction_sum(rhA, M);
    phis[4] = oc_reduction_sum(rhB, M);
    for (int i = 0; i < 5; i++) phis[i] /= M;
    /* D2H of rA, rB, rh, rCB into w[2M:6M), density.h:457 */
    memcpy(w + 2 * (size_t)M, rA, sizeof(double) * 4 * (size_t)M);
    return 0;
}

/* ================================================================ box stress
   d lnQ / d L_i by the adjoint of the Richardson step, in real space: one
   step is S = (4 E4 D2 E2 D2 E4 - E2 D1 E2)/3 (E4 = e^{-w ds/4}, E2 = E4^2,
   D = FFT^-1 K FFT with K2 = e^{-k^2 ds/12}/M, K1 = e^{-k^2 ds/6}/M,
   density.h:129-220), so
     dS/dL_i x = 4/3 [E4 dD2_i(E2 D2 E4 x) + E4 D2(E2 dD2_i(E4 x))] - 1/3 E2 dD1_i(E2 x)
   with dK/dL_i = K c 8 pi^2 n_i^2 / L_i^3, c = ds/12 (K2) or ds/6 (K1), and
   dQC/dL = (1/M) sum_s <q^dagger(N-1-s), dS_s/dL q(s)>,
   dQ2/dL = (1/M) sum_j <q^dagger(Nh-1-j), dS_B/dL q^dagger(j)> (q^dagger of a
   step is the adjoint of q's mirrored step: S is symmetric).  A restatement
   of the CUDA adjoint (no reference counterpart) that shares none of its
   Fourier-space (Parseval) formulation. */
static void apply_k(oc_density *d, const double *in, double *out, const double *K, int axis, double c)
{
    const oc_grid *g = d->g;
    const int m0 = g->m[0], m1 = g->m[1], mk2 = g->mk2, Mk = d->Mk;
    double *h = (double *)malloc(sizeof(double) * 2 * (size_t)Mk);
    oc_fft_r2c(g, in, h);
    for (int k = 0; k < Mk; k++) {
        double v = K[k];
        if (axis >= 0) {
            const int K0 = k / (mk2 * m1), K1 = (k / mk2) % m1, k2 = k % mk2;
            const int n = axis == 0 ? (K0 > m0 / 2 ? K0 - m0 : K0) : axis == 1 ? (K1 > m1 / 2 ? K1 - m1 : K1) : k2;
            const double L = g->D[axis];
            v *= c * 8.0 * PI * PI * (double)n * n / (L * L * L);
        }
        h[2 * k] *= v;
        h[2 * k + 1] *= v;
    }
    oc_fft_c2r(g, h, out);
    free(h);
}

/* <y, dS/dL_i x> for i = 0..2 with the step's tables E4, E2 */
static void pair_stress(oc_density *d, const double *x, const double *y, const double *E4, const double *E2,
                        double ds, double out[3])
{
    const int M = d->M;
    double *a = (double *)calloc(6 * (size_t)M, sizeof(double));
    double *b = a + M, *c = b + M, *t = c + M, *u = t + M, *v = u + M;
    for (int r = 0; r < M; r++) a[r] = E4[r] * x[r];
    apply_k(d, a, b, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) c[r] = E2[r] * b[r];
    for (int i = 0; i < 3; i++) {
        double acc = 0;
        apply_k(d, c, t, d->expKsq2, i, ds / 12); /* E4 dD2 (E2 D2 E4 x) */
        for (int r = 0; r < M; r++) acc += 4.0 / 3.0 * y[r] * E4[r] * t[r];
        apply_k(d, a, t, d->expKsq2, i, ds / 12); /* E4 D2 (E2 dD2 (E4 x)) */
        for (int r = 0; r < M; r++) u[r] = E2[r] * t[r];
        apply_k(d, u, v, d->expKsq2, -1, 0);
        for (int r = 0; r < M; r++) acc += 4.0 / 3.0 * y[r] * E4[r] * v[r];
        for (int r = 0; r < M; r++) u[r] = E2[r] * x[r]; /* E2 dD1 (E2 x) */
        apply_k(d, u, t, d->expKsq, i, ds / 6);
        for (int r = 0; r < M; r++) acc -= 1.0 / 3.0 * y[r] * E2[r] * t[r];
        out[i] = acc;
    }
    free(a);
}

/* props of w2M (W-, W+) into the density's propagator store, fcont as props_impl */
static int props_of(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f, int ens,
                    int fcont)
{
    const int M = d->M;
    double *w = (double *)calloc(6 * (size_t)M, sizeof(double));
    memcpy(w, w2M, sizeof(double) * 2 * (size_t)M);
    double lnQ, phis[5];
    const int rc = props_impl(d, w, &lnQ, Ns, alpha, phic, phis, f, ens, fcont);
    free(w);
    return rc;
}

static int stress_impl(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f, int ens,
                       int fcont, double dlnQ_dL[3])
{
    const int M = d->M;
    const int n1 = fcont ? (int)floor(Ns * f) : (int)round(Ns * f), Nh = alpha * Ns;
    const double ds = 1.0 / Ns;
    const int rc = props_of(d, w2M, Ns, alpha, phic, f, ens, fcont);
    if (rc != 0) return rc;
    double dQC[3] = {0, 0, 0}, dQ2[3] = {0, 0, 0}, o[3];
    for (int s = 0; s < Ns; s++) {
        const int A = s < n1, J = fcont && s == n1;
        pair_stress(d, oc_density_q(d, 0, s), oc_density_q(d, 1, Ns - 1 - s),
                    J ? d->E2j : A ? d->E2p1 : d->E2m1, J ? d->Ej : A ? d->Ep1 : d->Em1, ds, o);
        for (int i = 0; i < 3; i++) dQC[i] += o[i];
    }
    for (int j = 0; j < Nh; j++) {
        pair_stress(d, oc_density_q(d, 1, j), oc_density_q(d, 1, Nh - 1 - j), d->E2m1, d->Em1, ds, o);
        for (int i = 0; i < 3; i++) dQ2[i] += o[i];
    }
    for (int i = 0; i < 3; i++) {
        dQC[i] /= M;
        dQ2[i] /= M;
        dlnQ_dL[i] = ens == 1 ? phic * dQC[i] / d->QC + ((1.0 - phic) / alpha) * dQ2[i] / d->Q2
                              : dQ2[i] + phic * dQC[i]; /* density.h:390, 398 */
    }
    return 0;
}

int oc_stress(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f, int ens,
              double dlnQ_dL[3])
{
    return stress_impl(d, w2M, Ns, alpha, phic, f, ens, 0, dlnQ_dL);
}

int oc_stress_fcont(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f, int ens,
                    double dlnQ_dL[3])
{
    return stress_impl(d, w2M, Ns, alpha, phic, f, ens, 1, dlnQ_dL);
}

/* d lnQ/df of the continuous-f chain.  Only q's step n1 and q^dagger's step
   n2 - 1 depend on f, through theta = Ns f - n1 in their field
   wj = W+ + (2 theta - 1) W-, so with E4 = e^{-wj ds/4}, E2 = E4^2 and
   g = dE4/dtheta / E4 = -(ds/2) W-:
     dS/dtheta x = 4/3 [g E4 D2 E2 D2 E4 x + E4 D2 (2g E2) D2 E4 x + E4 D2 E2 D2 (g E4 x)]
                 - 1/3 [2g E2 D1 E2 x + E2 D1 (2g E2 x)].
   QC = <q(Ns)> sees it once, as <q^dagger(n2 - 1), dS/dtheta q(n1)> / M (S is
   symmetric, so q^dagger carries the adjoint of q's later steps).  Q2 =
   <q^dagger(Nh)> does not see it: Nh <= n2 - 1 puts q^dagger's junction step
   after slice Nh. */
int oc_dlnq_df(oc_density *d, const double *w2M, int Ns, double alpha, double phic, double f, int ens,
               double *dlnQ_df)
{
    const int M = d->M;
    const int n1 = (int)floor(Ns * f), n2 = Ns - n1;
    const double ds = 1.0 / Ns;
    const int rc = props_of(d, w2M, Ns, alpha, phic, f, ens, 1);
    if (rc != 0) return rc;
    const double *x = oc_density_q(d, 0, n1), *y = oc_density_q(d, 1, n2 - 1);
    const double *E4 = d->E2j, *E2 = d->Ej;
    double *g = (double *)calloc(5 * (size_t)M, sizeof(double));
    double *a = g + M, *b = a + M, *c = b + M, *e = c + M;
    for (int r = 0; r < M; r++) g[r] = -0.5 * ds * w2M[r];
    double t = 0;
    for (int r = 0; r < M; r++) a[r] = E4[r] * x[r]; /* first half-step pair: E4 D2 E2 D2 E4 x */
    apply_k(d, a, b, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) c[r] = E2[r] * b[r];
    apply_k(d, c, e, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) t += 4.0 / 3.0 * y[r] * g[r] * E4[r] * e[r];
    for (int r = 0; r < M; r++) c[r] = 2.0 * g[r] * E2[r] * b[r];
    apply_k(d, c, e, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) t += 4.0 / 3.0 * y[r] * E4[r] * e[r];
    for (int r = 0; r < M; r++) a[r] = g[r] * E4[r] * x[r];
    apply_k(d, a, b, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) c[r] = E2[r] * b[r];
    apply_k(d, c, e, d->expKsq2, -1, 0);
    for (int r = 0; r < M; r++) t += 4.0 / 3.0 * y[r] * E4[r] * e[r];
    for (int r = 0; r < M; r++) a[r] = E2[r] * x[r]; /* full step: E2 D1 E2 x */
    apply_k(d, a, b, d->expKsq, -1, 0);
    for (int r = 0; r < M; r++) t -= 1.0 / 3.0 * y[r] * 2.0 * g[r] * E2[r] * b[r];
    for (int r = 0; r < M; r++) a[r] = 2.0 * g[r] * E2[r] * x[r];
    apply_k(d, a, b, d->expKsq, -1, 0);
    for (int r = 0; r < M; r++) t -= 1.0 / 3.0 * y[r] * E2[r] * b[r];
    free(g);
    const double dQC = t / M;
    *dlnQ_df = Ns * (ens == 1 ? phic * dQC / d->QC : phic * dQC); /* density.h:390, 398 */
    return 0;
}

/* ================================================================ spline */
/* cubefit_chunk_g, GPU_kernels.h:232-284, for one point */
void oc_spline_coeffs(int strn, const double *x, const double *a_in, double *c, double *b,
                      double *d)
{
    const int n = strn - 1;
    double *a = (double *)malloc(sizeof(double) * 7 * (size_t)strn);
    double *h = a + strn, *A = a + 2 * strn, *l = a + 3 * strn, *u = a + 4 * strn,
           *z = a + 5 * strn;
    for (int ii = 0; ii < strn; ++ii) {
        a[ii] = a_in[ii];
        b[ii] = c[ii] = d[ii] = 0.0;
        h[ii] = A[ii] = l[ii] = u[ii] = z[ii] = 0.0;
    }
    for (int i = 0; i <= n - 1; ++i) h[i] = x[i + 1] - x[i];
    for (int i = 1; i <= n - 1; ++i)
        A[i] = 3.0 * (a[i + 1] - a[i]) / h[i] - 3.0 * (a[i] - a[i - 1]) / h[i - 1];
    l[0] = 1.0;
    u[0] = 0.0;
    z[0] = 0.0;
    for (int i = 1; i <= n - 1; ++i) {
        l[i] = 2.0 * (x[i + 1] - x[i - 1]) - h[i - 1] * u[i - 1];
        u[i] = h[i] / l[i];
        z[i] = (A[i] - h[i - 1] * z[i - 1]) / l[i];
    }
    l[n] = 1.0;
    z[n] = 0.0;
    c[n] = 0.0;
    for (int j = n - 1; j >= 0; --j) {
        c[j] = z[j] - u[j] * c[j + 1];
        b[j] = (a[j + 1] - a[j]) / h[j] - h[j] * (c[j + 1] + 2.0 * c[j]) / 3.0;
        d[j] = (c[j + 1] - c[j]) / (3.0 * h[j]);
    }
    free(a);
}

/* interval search of eval_spline_*_chunk_g, GPU_kernels.h:292-297 */
static int spline_interval(int strn, const double *x, double xx)
{
    int nm = 0;
    for (int i = 0; i < strn; ++i) {
        if (x[i] < xx)
            nm = i;
        else
            break;
    }
    return nm;
}

void oc_spline_derivs(int strn, const double *x, double *const *ww, int r0, int n,
                      const int *doiis, double *const *out)
{
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)strn);
        double *a = buf, *c = buf + strn, *b = buf + 2 * strn, *d = buf + 3 * strn;
#pragma omp for schedule(static)
        for (int rc = 0; rc < n; rc++) {
            for (int ii = 0; ii < strn; ii++) a[ii] = ww[ii][r0 + rc];
            oc_spline_coeffs(strn, x, a, c, b, d);
            for (int ev = 0; ev < strn; ++ev) {
                const double xx = x[ev];
                int nm = spline_interval(strn, x, xx);
                const double dx = xx - x[nm];
                double v = b[nm] + 2.0 * dx * c[nm] + 3.0 * dx * dx * d[nm];
                if (doiis[ev] == 1) out[ev][r0 + rc] = v;
            }
        }
        free(buf);
    }
}

void oc_spline_redist(int strn, const double *x, const double *xref, double *const *ww,
                      int r0, int n, const int *doiis, double lambda)
{
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 5 * (size_t)strn);
        double *a = buf, *c = buf + strn, *b = buf + 2 * strn, *d = buf + 3 * strn,
               *ev = buf + 4 * strn;
#pragma omp for schedule(static)
        for (int rc = 0; rc < n; rc++) {
            for (int ii = 0; ii < strn; ii++) a[ii] = ww[ii][r0 + rc];
            oc_spline_coeffs(strn, x, a, c, b, d);
            for (int e = 0; e < strn; ++e) {
                const double xx = xref[e];
                int nm = spline_interval(strn, x, xx);
                const double dx = xx - x[nm];
                ev[e] = a[nm] + dx * b[nm] + dx * dx * c[nm] + dx * dx * dx * d[nm];
            }
            for (int ii = 1; ii < strn - 1; ii++)
                if (doiis[ii] == 1) ww[ii][r0 + rc] += (ev[ii] - ww[ii][r0 + rc]) * lambda;
        }
        free(buf);
    }
}

/* ================================================================ solver */
struct oc_solver {
    oc_problem  p;
    int         M;
    oc_density *dens;
    double    **W;    /* strn x 7M */
    double    **DEV;  /* strn x 2M (DEV[ii][0] of the reference) */
    int        *doiis;
    double      phis[6];
    long        props_calls;
    double     *alf;  /* strn */
};

oc_solver *oc_solver_create(const oc_problem *p)
{
    if (p->strn < 1 || (p->ens != 1 && p->ens != 2)) return NULL;
    oc_density *d = oc_density_create(p->m, p->D, p->N);
    if (!d) return NULL;
    oc_solver *s = (oc_solver *)calloc(1, sizeof(oc_solver));
    s->p = *p;
    s->dens = d;
    s->M = d->M;
    s->W = (double **)malloc(sizeof(double *) * p->strn);
    s->DEV = (double **)malloc(sizeof(double *) * p->strn);
    for (int ii = 0; ii < p->strn; ii++) {
        s->W[ii] = (double *)calloc(7 * (size_t)s->M, sizeof(double));
        s->DEV[ii] = (double *)calloc(2 * (size_t)s->M, sizeof(double));
    }
    s->doiis = (int *)malloc(sizeof(int) * p->strn);
    for (int ii = 0; ii < p->strn; ii++) s->doiis[ii] = 1; /* one process owns all, scft.cu:952-975 */
    s->alf = (double *)calloc(p->strn, sizeof(double));
    return s;
}

void oc_solver_destroy(oc_solver *s)
{
    if (!s) return;
    for (int ii = 0; ii < s->p.strn; ii++) {
        free(s->W[ii]);
        free(s->DEV[ii]);
    }
    free(s->W);
    free(s->DEV);
    free(s->doiis);
    free(s->alf);
    oc_density_destroy(s->dens);
    free(s);
}

double *oc_solver_W(oc_solver *s, int ii) { return s->W[ii]; }
int    *oc_solver_doiis(oc_solver *s) { return s->doiis; }
long    oc_solver_props_calls(const oc_solver *s) { return s->props_calls; }
const double *oc_solver_alf(const oc_solver *s) { return s->alf; }

static void solver_props(oc_solver *s, int ii, double *lnQ)
{
    oc_props(s->dens, s->W[ii], lnQ, s->p.N, s->p.alpha, s->p.phidb, s->phis, s->p.f, s->p.ens);
    s->props_calls++;
}

/* EDist, scft.cu:351-355 */
double oc_edist(const double *a, const double *b, int M)
{
    double dist = 0;
    for (int r = 0; r < M; r++) dist += pow(a[r] - b[r], 2.0);
    return sqrt(dist);
}

/* solve_field0, scft.cu:516-554 */
int oc_solve_field0(oc_solver *s, int ii, int maxIter, double errTol)
{
    const int M = s->M;
    const double chi = s->p.chi;
    double lambda = 0.05, err = 1.0, lnQ, S1, errt = 1, dlam1 = 1.09, dlam2 = 1.10;
    int k, r;
    double *W = s->W[ii], *DEV = s->DEV[ii];
    const double *phiA = W + 2 * (size_t)M, *phiB = W + 3 * (size_t)M;
    for (k = 1; k < maxIter && err > errTol; k++) {
        solver_props(s, ii, &lnQ);
        for (r = 0; r < M; r++) {
            DEV[r] = 0;
            DEV[r + M] = chi * (phiB[r] + phiA[r] - 1.0);
        }
        for (r = 0, S1 = 0.0; r < 2 * M; r++) S1 += DEV[r] * DEV[r];
        err = pow(S1 / (M), 0.5);
        for (r = 0; r < 2 * M; r++) W[r] = W[r] + lambda * DEV[r];
        if (err < errt)
            lambda = fmin(0.1, lambda * dlam1);
        else
            lambda = fmax(0.005, lambda / dlam2);
        errt = err;
    }
    return k;
}

/* FreeE, scft.cu:812-853 (one process: procid==0==numprocs-1) */
double oc_free_energy(oc_solver *s, double *alf, double *FEs0, double *FEs1, double *FEs,
                      double *phctot)
{
    const int M = s->M, strn = s->p.strn;
    const double chi = s->p.chi, f = s->p.f;
    double wa, wb, FE = 0, lnQ;
    alf[0] = 0;
    for (int ii = 0; ii < strn; ii++) {
        if (s->doiis[ii] == 1 || ii == 0 || ii == strn - 1) {
            double *W = s->W[ii];
            const double *phiA = W + 2 * (size_t)M, *phiB = W + 3 * (size_t)M;
            oc_solve_field0(s, ii, 1E2, 1E-4);
            solver_props(s, ii, &lnQ);
            FEs0[ii] = -lnQ;
            FEs1[ii] = 0;
            phctot[ii] = 0;
            for (int r = 0; r < M; r++) {
                wa = W[r] + W[r + M];
                wb = W[r + M] - W[r];
                FEs1[ii] += (chi * phiA[r] * phiB[r] - wa * phiA[r] - wb * phiB[r]) / M;
                phctot[ii] += phiA[r] / (M * f);
            }
            FEs[ii] = FEs0[ii] + FEs1[ii];
        }
        if (ii > 0) alf[ii] = alf[ii - 1] + oc_edist(s->W[ii], s->W[ii - 1], M);
    }
    for (int ii = 0; ii < strn; ii++) FE += FEs[ii];
    for (int ii = 0; ii < strn; ii++) s->alf[ii] = alf[ii];
    return FE;
}

/* arc-length coordinates, scft.cu:612-621 and 725-736 */
static void arc_length(oc_solver *s, double *x)
{
    const int strn = s->p.strn, M = s->M;
    double *Del = (double *)malloc(sizeof(double) * (strn > 1 ? strn - 1 : 1));
    double Delsum = 0;
    for (int ii = 0; ii < strn - 1; ii++) {
        Del[ii] = oc_edist(s->W[ii], s->W[ii + 1], M);
        Delsum += Del[ii];
    }
    for (int ii = 0; ii < strn - 1; ii++) Del[ii] /= Delsum;
    x[0] = 0;
    x[strn - 1] = 1;
    for (int ii = 1; ii < strn - 1; ii++) x[ii] = x[ii - 1] + Del[ii - 1];
    free(Del);
}

/* solve_field, scft.cu:559-809 (one process, numprocs==1) */
int oc_solve_field(oc_solver *s, int doii, int maxIter, double errTol, oc_iter_record *rec,
                   double *errs_out, double *errs3_out)
{
    const int M = s->M, strn = s->p.strn;
    const double chi = s->p.chi;
    double lambda = 0.05, err = 1, lnQ, S1, errt = 1, dlam1 = 1.015, dlam2 = 1.016;
    const int skip = 50;
    const double eps = 0.5;
    double *errs = (double *)calloc(strn, sizeof(double)), *errs3 = (double *)calloc(strn, sizeof(double));
    double *normDER = (double *)calloc(strn, sizeof(double)), *normDEV = (double *)calloc(strn, sizeof(double));
    double *dotWs = (double *)calloc(strn, sizeof(double)), *x = (double *)calloc(strn, sizeof(double));
    double *xref = (double *)calloc(strn, sizeof(double)), *fitups = (double *)calloc(strn, sizeof(double));
    double *FEs0 = (double *)calloc(strn, sizeof(double)), *FEs1 = (double *)calloc(strn, sizeof(double));
    double *FEs = (double *)calloc(strn, sizeof(double)), *phctot = (double *)calloc(strn, sizeof(double));
    double *alf = (double *)calloc(strn, sizeof(double));
    int *steps = (int *)calloc(strn, sizeof(int));
    double **Wm = (double **)malloc(sizeof(double *) * strn);
    double **dWda = (double **)malloc(sizeof(double *) * strn);
    double fitup = 0, stepav, FE = 0;
    int k, r, ii;
    for (ii = 0; ii < strn; ii++) {
        Wm[ii] = s->W[ii];
        dWda[ii] = s->W[ii] + 6 * (size_t)M;
    }
    int dospring = 1, doredist = 0, doperp = 0;
    if (doii > -1 || s->p.dostring != 1) dospring = 0, doredist = 0, doperp = 0;
    if (s->p.fix[0] == 1) s->doiis[0] = 0;
    if (s->p.fix[1] == 1) s->doiis[strn - 1] = 0;

    for (k = 0; k < maxIter && err > errTol; k++) {
        if (k >= s->p.springsteps && doii == -1 && s->p.dostring == 1) {
            dospring = 0;
            doredist = 1;
            doperp = 1;
        }
        for (ii = 0; ii < strn; ii++) memset(s->DEV[ii], 0, sizeof(double) * 2 * (size_t)M);
        for (ii = 0; ii < strn; ii++) {
            steps[ii] = 0;
            if ((s->doiis[ii] == 1 && doii == -1) || doii == ii) {
                double *W = s->W[ii], *DEV = s->DEV[ii];
                const double *phiA = W + 2 * (size_t)M, *phiB = W + 3 * (size_t)M;
                steps[ii]++;
                steps[ii] += oc_solve_field0(s, ii, 20, errTol);
                solver_props(s, ii, &lnQ);
                for (r = 0; r < M; r++) {
                    DEV[r] = chi * (phiB[r] - phiA[r]) - 2.0 * W[r];
                    if (ii > 0 && ii < strn - 1 && dospring == 1)
                        DEV[r] += eps * (s->W[ii + 1][r] + s->W[ii - 1][r] - 2.0 * W[r]);
                    DEV[r + M] = chi * (phiB[r] + phiA[r] - 1.0);
                }
            }
        }
        if (doii == -1) {
            arc_length(s, x);
            for (ii = 0; ii < strn; ii++) xref[ii] = (1.0 * ii) / (strn - 1.0);
        }
        if (doii == -1) {
            for (ii = 0; ii < strn; ii++) {
                for (r = 0, S1 = 0.0; r < 2 * M; r++) S1 += s->DEV[ii][r] * s->DEV[ii][r];
                errs[ii] = pow(S1 / (2 * M), 0.5);
            }
        } else {
            for (ii = 0; ii < strn; ii++) errs[ii] = 0;
            for (r = 0, S1 = 0.0; r < 2 * M; r++) S1 += s->DEV[doii][r] * s->DEV[doii][r];
            errs[doii] = pow(S1 / (2 * M), 0.5);
        }
        if (doperp == 1) {
            for (ii = 0; ii < strn; ii++)
                if (s->doiis[ii] == 1) memset(dWda[ii], 0, sizeof(double) * (size_t)M);
            oc_spline_derivs(strn, x, Wm, 0, M, s->doiis, dWda);
            for (ii = 0; ii < strn; ii++) {
                normDER[ii] = 0;
                if (s->doiis[ii] == 1)
                    for (r = 0; r < M; r++) normDER[ii] += dWda[ii][r] * dWda[ii][r];
                normDER[ii] = sqrt(normDER[ii]);
            }
            for (ii = 0; ii < strn; ii++) {
                normDEV[ii] = 0;
                if (s->doiis[ii] == 1)
                    for (r = 0; r < M; r++) normDEV[ii] += s->DEV[ii][r] * s->DEV[ii][r];
                normDEV[ii] = sqrt(normDEV[ii]);
            }
            for (ii = 0; ii < strn; ii++) {
                dotWs[ii] = 0;
                if (s->doiis[ii] == 1)
                    for (r = 0; r < M; r++)
                        dotWs[ii] += (s->DEV[ii][r] / normDEV[ii]) * (dWda[ii][r] / normDER[ii]);
            }
            for (ii = 0; ii < strn; ii++) errs3[ii] = 0;
            for (ii = 1; ii < strn - 1; ii++) {
                if (s->doiis[ii] == 1 && normDER[ii] > 0 && normDEV[ii] > 0) {
                    for (r = 0; r < M; r++)
                        s->DEV[ii][r] -= (dotWs[ii] / normDER[ii]) * dWda[ii][r] * normDEV[ii];
                    for (r = 0; r < 2 * M; r++) errs3[ii] += s->DEV[ii][r] * s->DEV[ii][r];
                    errs3[ii] = pow(errs3[ii] / (2 * M), 0.5);
                }
            }
        } else
            for (ii = 0; ii < strn; ii++) errs3[ii] = errs[ii];
        errs3[0] = errs[0];
        errs3[strn - 1] = errs[strn - 1];
        for (ii = 0; ii < strn; ii++)
            for (r = 0; r < 2 * M; r++) s->W[ii][r] = s->W[ii][r] + lambda * s->DEV[ii][r];
        stepav = 0;
        for (ii = 0; ii < strn; ii++) stepav += steps[ii];
        stepav /= strn;
        if (doii == -1) {
            arc_length(s, x);
            fitup = 0;
            for (ii = 0; ii < strn; ii++) alf[ii] = x[ii];
            for (ii = 0; ii < strn; ii++) fitups[ii] = x[ii] - xref[ii];
            for (ii = 1; ii < strn - 1; ii++) fitup += pow(fitups[ii], 2.0);
            fitup /= strn - 2.0;
            fitup = sqrt(fitup);
            fitup /= strn - 1.0;
        }
        if (doredist == 1) oc_spline_redist(strn, x, xref, Wm, 0, M, s->doiis, lambda);

        double errtot = 0;
        for (ii = 0; ii < strn; ii++) errtot += errs3[ii] * errs3[ii] / strn;
        errtot = sqrt(errtot);
        int did_fe = 0;
        if (k % skip == 0 || k == maxIter - 1 || !(err > errTol)) {
            FE = oc_free_energy(s, alf, FEs0, FEs1, FEs, phctot);
            did_fe = 1;
        }
        if (rec) {
            rec[k].k = k;
            rec[k].lambda = lambda;
            rec[k].errtot = errtot;
            rec[k].fitup = fitup;
            rec[k].stepav = stepav;
            rec[k].did_freee = did_fe;
            rec[k].FE = did_fe ? FE : 0.0;
        }
        if (errs_out) memcpy(errs_out + (size_t)k * strn, errs, sizeof(double) * strn);
        if (errs3_out) memcpy(errs3_out + (size_t)k * strn, errs3, sizeof(double) * strn);
        if (err < errt)
            lambda = fmin(0.2, lambda * dlam1);
        else
            lambda = fmax(0.05, lambda / dlam2);
        errt = err;
    }
    free(errs); free(errs3); free(normDER); free(normDEV); free(dotWs); free(x); free(xref);
    free(fitups); free(FEs0); free(FEs1); free(FEs); free(phctot); free(alf); free(steps);
    free(Wm); free(dWda);
    return k;
}
