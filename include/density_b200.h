/*
 * density_b200.h -- the reference's `density` class (density.h:225-548) on top
 * of the C ABI in scft_b200.h, so that scft.cu builds unchanged against
 * libscft_b200.so: place a `density.h` that holds only
 *     #include "density_b200.h"
 * where scft.cu includes "density.h" (scft.cu:73), and link -lscft_b200.
 * scft.cu sees the same members it calls: props (scft.cu:526, 603, 819),
 * setupSplineBuffers (scft.cu:1011), setSplineX / setSplineXRef and the two
 * chunked spline services (scft.cu:643-650, 746-751).  Like the reference, a
 * failing call prints the error and exits (GPU_kernels.h:16-48).
 *
 * It uses the globals scft.cu defines before that include: m, ens and the
 * compile-time strn (scft.cu:35-38).  density(Ns, D) does not receive the A
 * fraction or the homopolymer parameters, which the reference passes to
 * every props call instead, so the context is made by the first props call
 * and made again if a later call brings other values; scft.cu passes the same
 * ones throughout.
 */
#pragma once
#include <cstdio>
#include <cstdlib>

#include "scft_b200.h"

#ifdef __CUDACC__
/* scft.cu:879 launches this to check that the device answers (nvcc builds
 * scft.cu; a host compiler sees only the class) */
__global__ void print_from_gpu(void) { printf("Testing GPUs: [%d,%d] (From device)\n", threadIdx.x, blockIdx.x); }
#endif

class density {
    scft_ctx *ctx_ = nullptr;
    int Ns_ = 0;
    double D_[3] = {0, 0, 0};
    double alpha_ = -1, phic_ = -1, f_ = -1;
    const double *x_ = nullptr, *xref_ = nullptr;

    static void ck(scft_status s, scft_ctx *c, const char *what)
    {
        if (s == SCFT_OK) return;
        fprintf(stderr, "%s: %s (%s)\n", what, scft_status_string(s), c ? scft_last_error(c) : "");
        exit(EXIT_FAILURE);
    }
    void make(int Ns, double alpha, double phic, double f)
    {
        if (ctx_ && Ns == Ns_ && alpha == alpha_ && phic == phic_ && f == f_) return;
        if (ctx_) scft_destroy(ctx_);
        ctx_ = nullptr;
        scft_problem p{};
        for (int i = 0; i < 3; i++) {
            p.m[i] = m[i];
            p.D[i] = D_[i];
        }
        p.N = Ns;
        p.alpha = alpha;
        p.ens = ens;
        p.phidb = phic;
        p.f = f;
        p.strn = strn;  /* the spline services work over all strn knots */
        p.dostring = 1;
        p.precision = SCFT_FP64;
        p.batched = 0;
        ck(scft_create(&p, &ctx_), ctx_, "scft_create");
        Ns_ = Ns;
        alpha_ = alpha;
        phic_ = phic;
        f_ = f;
    }

public:
    density(int Ns, double *D) : Ns_(Ns)
    {
        for (int i = 0; i < 3; i++) D_[i] = D[i];
    }
    ~density()
    {
        if (ctx_) scft_destroy(ctx_);
    }
    density(const density &) = delete;
    density &operator=(const density &) = delete;

    /* the library sizes its own spline work space */
    void setupSplineBuffers(int) {}
    void setSplineX(double *x) { x_ = x; }
    void setSplineXRef(double *xref) { xref_ = xref; }

    void props(double *w, double *lnQ, int ii, int Ns, double alpha, double phic, double *phis, double f)
    {
        make(Ns, alpha, phic, f);
        ck(scft_props_host(ctx_, w, lnQ, ii, Ns, alpha, phic, phis, f), ctx_, "props");
    }
    void splineDerivsChunked(double **ww, double *x, int r0, int n, int *doiis, double **out)
    {
        if (!ctx_) make(Ns_, 0.0, 1.0, 0.5);  /* the spline services do not use the chain */
        ck(scft_spline_derivs(ctx_, x ? x : x_, ww, r0, n, doiis, out), ctx_, "splineDerivsChunked");
    }
    void splineRedistChunked(double **ww, double *x, double *xref, int r0, int n, int *doiis, double lambda)
    {
        if (!ctx_) make(Ns_, 0.0, 1.0, 0.5);
        ck(scft_spline_redist(ctx_, x ? x : x_, xref ? xref : xref_, ww, r0, n, doiis, lambda), ctx_,
           "splineRedistChunked");
    }
};
