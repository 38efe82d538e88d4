/*
 * tcs_oracle.c -- TEST INFRASTRUCTURE ONLY (see tcs_oracle.h).
 *
 * A line-by-line CPU restatement of the PaScaL_TCS time step on ONE MPI rank
 * (np1 = np2 = np3 = 1).  Every function names the reference routine it
 * follows (paths relative to the PaScaL_TCS source tree).  Expression order is
 * kept where practical; the file is compiled with -ffp-contract=off so that no
 * fused multiply-adds change the rounding of the restated expressions.
 *
 * One-rank semantics worth knowing (all mirrored here on purpose):
 *  - MPI self-exchange: periodic ghost copy x then z, full faces; y is a no-op
 *    (module_mpi_subdomain.f90:758-791).
 *  - mpi_thermal_boundary sets only the bottom ghost row of T when the y
 *    communicator has one rank (else-if at module_solve_thermal.f90:102-110);
 *    the top ghost row of T therefore stays 0.  top_wall_mode=1 sets it to Tup,
 *    which is what the reference computes when y is split over >= 2 ranks.
 *  - Stale loop indices and scalars in the ADI coefficient loops, row-wise Mu
 *    and invRho, buoyancy on U only, swapped y masks in solvedV, the one-rank
 *    2x2 cyclic closure with e(2) overwritten, the sequential-sweep reads of
 *    already-updated dPhat in the projection.
 *
 * Parity: UNPINNED against the reference program itself (no Fortran/MPI/FFTW
 * toolchain and no golden vectors exist); pinned by the mathematical KATs in
 * tests/test_oracle.py.
 */
#include "tcs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct tcs_oracle {
    tcs_oracle_params p;
    int top_wall_mode;
    /* module_global */
    int n1m, n2m, n3m, n1, n2, n3;
    double L1, L2, L3, dtMax, Cmu, Cmt, Ct, Cmp, Gr;
    double a10, a11, a12, a13, a14, a15, a12pera11;
    double b10, b11, b12, b13, b14, b15;
    double c10, c11, c12, c13, c14, c15;
    double d10, d11, d12, d13, d14, d15;
    double KPP0, Rho0, Cp0, Mu0;
    double Uup, Vup, Wup, Tup, Ubt, Vbt, Wbt, Tbt;
    /* module_mpi_subdomain (one rank) */
    int n1sub, n2sub, n3sub, n1msub, n2msub, n3msub;
    int i_indexS, j_indexS, k_indexS;
    int h1p, h3p;
    double *x1, *dx1, *dmx1, *x2, *dx2, *dmx2, *x3, *dx3, *dmx3;
    int *jC_BC, *jS_BC;
    /* padded fields (0:n1sub, 0:n2sub, 0:n3sub), i fastest */
    size_t P1, P2, P3, NP;
    double *T, *U, *V, *W, *P, *dPhat, *dP0, *dU, *dV, *dW, *dP;
    double *KPP, *dKPP, *invRhoCp, *dinvRhoCp, *Mu, *invRho;
    /* wall boundary arrays are constants per wall in the reference (module_global.f90:107-110) */
    double *PRHS;                    /* (1:n1m,1:n2m,1:n3m) */
    double *dzk, *dxk2;              /* module_solve_pressure.f90:93-129 */
    double time, dt, CFL, maxDivU;
};

#define IX(s, i, j, k) ((size_t)(i) + (s)->P1 * ((size_t)(j) + (s)->P2 * (size_t)(k)))
#define F(a, i, j, k) (a)[IX(s, i, j, k)]
/* interior (1:n1m,1:n2m,1:n3m)-shaped arrays */
#define IN(s, i, j, k) ((size_t)((i) - 1) + (size_t)(s)->n1m * ((size_t)((j) - 1) + (size_t)(s)->n2m * (size_t)((k) - 1)))

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

int tcs_oracle_set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

/* ---------------------------------------------------------------------------
 * module_global.f90:75-167 (global_inputpara) after the namelist read.
 * ------------------------------------------------------------------------- */
static void global_inputpara(tcs_oracle *s)
{
    const tcs_oracle_params *p = &s->p;
    s->n1m = p->n1m; s->n2m = p->n2m; s->n3m = p->n3m;
    s->Uup = 0.0; s->Ubt = 0.0; s->Vup = 0.0; s->Vbt = 0.0; s->Wup = 0.0; s->Wbt = 0.0;
    s->Tup = -0.5; s->Tbt = 0.5;                                   /* :107-110 */
    if (p->property_set == 1) {                                    /* water, :113-116 */
        s->a10 = 0.9922e+3; s->a11 = -3.736e-4; s->a12 = -3.98e-6; s->a13 = 0.; s->a14 = 0.; s->a15 = 0.;
        s->b10 = 4.1690e+3; s->b11 = 0.084e-4;  s->b12 = 4.60e-6;  s->b13 = 0.; s->b14 = 0.; s->b15 = 0.;
        s->c10 = (double)0.6297f; s->c11 = 21.99e-4; s->c12 = -17.8e-6; s->c13 = 0.; s->c14 = 0.; s->c15 = 0.;
        s->d10 = 0.6690e-6; s->d11 = -175.9e-4; s->d12 = 295.8e-6; s->d13 = -460.e-8; s->d14 = 0.; s->d15 = 0.;
    } else if (p->property_set == 2) {                             /* glycerol, :129-132 */
        s->a10 = 1.2477e+3; s->a11 = -4.789e-4; s->a12 = -0.3795e-6; s->a13 = 0.; s->a14 = 0.; s->a15 = 0.;
        s->b10 = 2.5108e+3; s->b11 = 22.511e-4; s->b12 = 0.; s->b13 = 0.; s->b14 = 0.; s->b15 = 0.;
        s->c10 = 2.9351e-3; s->c11 = 3.863e-4;  s->c12 = 0.; s->c13 = 0.; s->c14 = 0.; s->c15 = 0.;
        s->d10 = 238.71e-6; s->d11 = -702.83e-4; s->d12 = 2393.1e-6; s->d13 = -6923.0e-8; s->d14 = 33131.3e-10; s->d15 = -71517.5e-12;
    } else {                                                       /* constant, :117-120 */
        s->a10 = 1.0; s->a11 = 0.0; s->a12 = 0.0; s->a13 = 0.0; s->a14 = 0.; s->a15 = 0.;
        s->b10 = 1.0; s->b11 = 0.0; s->b12 = 0.0; s->b13 = 0.0; s->b14 = 0.; s->b15 = 0.;
        s->c10 = 1.0; s->c11 = 0.0; s->c12 = 0.0; s->c13 = 0.0; s->c14 = 0.; s->c15 = 0.;
        s->d10 = 1.0; s->d11 = 0.0; s->d12 = 0.0; s->d13 = 0.0; s->d14 = 0.; s->d15 = 0.;
    }
    if (s->a12 < 1.0e-14) s->a12pera11 = 0.0; else s->a12pera11 = s->a12 / s->a11;   /* :122-126 */
    s->Rho0 = s->a10; s->Cp0 = s->b10; s->KPP0 = s->c10; s->Mu0 = s->a10 * s->d10; /* :134-137 */
    s->Cmu = sqrt(p->Pr / p->Ra); s->Cmt = 1.0; s->Ct = 1.0 / sqrt(p->Ra * p->Pr);  /* :139 */
    s->Gr = p->Ra / p->Pr;
    s->Cmp = 1.0;
    s->n1 = s->n1m + 1; s->n2 = s->n2m + 1; s->n3 = s->n3m + 1;
    s->L1 = p->H * p->aspect1; s->L2 = p->H; s->L3 = p->H * p->aspect3;
    {
        double t1 = s->L1 / (double)(s->n1 - 1), t2 = s->L2 / (double)(s->n2 - 1), t3 = s->L3 / (double)(s->n3 - 1);
        double mn = t1; if (t2 < mn) mn = t2; if (t3 < mn) mn = t3;
        s->dtMax = mn * 100;                                       /* :161-165 */
    }
}

/* ---------------------------------------------------------------------------
 * module_mpi_subdomain.f90:98-121 (make), :153-299 (mesh), :304-374 (indices)
 * on one rank with pbc = (T, F, T).
 * ------------------------------------------------------------------------- */
static void coord_periodic(int uniform, double L, double gamma, int nm, int nsub,
                           double *x, double *dx, double *dmx)
{
    int i;
    for (i = 0; i <= nsub; i++) {
        if (uniform == 1) x[i] = (double)(i - 1) * L / (double)nm + 0.0;
        else x[i] = L * 0.5 * (1.0 + tanh(0.5 * gamma * (2.0 * (double)(i - 1) / (double)nm - 1.0)) / tanh(gamma * 0.5)) + 0.0;
    }
    for (i = 1; i <= nsub - 1; i++) dx[i] = x[i + 1] - x[i];
    dx[0] = dx[nsub - 1];          /* self-exchange, :186-191 */
    dx[nsub] = dx[1];
    for (i = 1; i <= nsub - 1; i++) dmx[i] = 0.5 * (dx[i - 1] + dx[i]);
    dmx[0] = dmx[nsub - 1];        /* :202-207 */
    dmx[nsub] = dmx[1];
}

static void subdomain_mesh(tcs_oracle *s)
{
    const tcs_oracle_params *p = &s->p;
    int j;
    coord_periodic(p->uniform1, s->L1, p->gamma1, s->n1m, s->n1sub, s->x1, s->dx1, s->dmx1);
    coord_periodic(p->uniform3, s->L3, p->gamma3, s->n3m, s->n3sub, s->x3, s->dx3, s->dmx3);
    /* y: walls, no neighbour (MPI_PROC_NULL) -- :211-253 */
    for (j = 0; j <= s->n2sub; j++) {
        if (p->uniform2 == 1) s->x2[j] = (double)(j - 1) * s->L2 / (double)s->n2m + 0.0;
        else s->x2[j] = s->L2 * 0.5 * (1. + tanh(0.5 * p->gamma2 * (2. * (double)(j - 1) / (double)s->n2m - 1.0)) / tanh(p->gamma2 * 0.5)) + 0.0;
    }
    s->x2[0] = s->x2[1];
    for (j = 1; j <= s->n2msub; j++) s->dx2[j] = s->x2[j + 1] - s->x2[j];
    s->dx2[0] = 0.0; s->dx2[s->n2sub] = 0.0;
    for (j = 1; j <= s->n2msub; j++) s->dmx2[j] = 0.5 * (s->dx2[j - 1] + s->dx2[j]);
    s->dmx2[0] = 0.0;
    s->dmx2[s->n2sub] = 0.5 * (s->dx2[s->n2msub] + s->dx2[s->n2sub]);
}

static void subdomain_indices(tcs_oracle *s)
{
    int j;
    s->i_indexS = 1; s->j_indexS = 1; s->k_indexS = 1;
    for (j = 0; j <= s->n2sub; j++) { s->jC_BC[j] = 1; s->jS_BC[j] = 1; }
    s->j_indexS = 2;                     /* pbc2 false, first and last rank: :340-355 */
    s->jC_BC[0] = 0; s->jS_BC[0] = 0; s->jS_BC[1] = 0;
    s->jC_BC[s->n2sub] = 0; s->jS_BC[s->n2sub] = 0;
}

/* module_mpi_subdomain.f90:758-791: x faces, y (no-op on one rank), z faces. */
static void ghostcell_update(tcs_oracle *s, double *a)
{
    int i, j, k;
    const int n1sub = s->n1sub, n2sub = s->n2sub, n3sub = s->n3sub;
#pragma omp parallel for private(j)
    for (k = 0; k <= n3sub; k++)
        for (j = 0; j <= n2sub; j++) {
            F(a, 0, j, k) = F(a, n1sub - 1, j, k);
            F(a, n1sub, j, k) = F(a, 1, j, k);
        }
#pragma omp parallel for private(i)
    for (j = 0; j <= n2sub; j++)
        for (i = 0; i <= n1sub; i++) {
            F(a, i, j, 0) = F(a, i, j, n3sub - 1);
            F(a, i, j, n3sub) = F(a, i, j, 1);
        }
}

/* ---------------------------------------------------------------------------
 * PaScaL_TDMA on one rank: pascal_tdma.f90:487-578 / 715-806 with the
 * reduced 2-row systems of tdmas.f90:113-146 / 159-212 (Alltoallw with one
 * process is the identity).  Arrays are (n_sys, n_row), system index fastest.
 * ------------------------------------------------------------------------- */
#define A2(a, i, j) (a)[(size_t)(i) + (size_t)n_sys * (size_t)(j)]

static void modified_thomas(double *A, double *B, double *C, double *D, int n_sys, int n_row,
                            double *Ard, double *Crd, double *Drd)
{
    int i, j;
#pragma omp parallel for private(j)
    for (i = 0; i < n_sys; i++) {
        double r;
        A2(A, i, 0) = A2(A, i, 0) / A2(B, i, 0);
        A2(D, i, 0) = A2(D, i, 0) / A2(B, i, 0);
        A2(C, i, 0) = A2(C, i, 0) / A2(B, i, 0);
        A2(A, i, 1) = A2(A, i, 1) / A2(B, i, 1);
        A2(D, i, 1) = A2(D, i, 1) / A2(B, i, 1);
        A2(C, i, 1) = A2(C, i, 1) / A2(B, i, 1);
        for (j = 2; j < n_row; j++) {
            r = 1.0 / (A2(B, i, j) - A2(A, i, j) * A2(C, i, j - 1));
            A2(D, i, j) = r * (A2(D, i, j) - A2(A, i, j) * A2(D, i, j - 1));
            A2(C, i, j) = r * A2(C, i, j);
            A2(A, i, j) = -r * A2(A, i, j) * A2(A, i, j - 1);
        }
        for (j = n_row - 3; j >= 1; j--) {
            A2(D, i, j) = A2(D, i, j) - A2(C, i, j) * A2(D, i, j + 1);
            A2(A, i, j) = A2(A, i, j) - A2(C, i, j) * A2(A, i, j + 1);
            A2(C, i, j) = -A2(C, i, j) * A2(C, i, j + 1);
        }
        r = 1.0 / (1.0 - A2(A, i, 1) * A2(C, i, 0));
        A2(D, i, 0) = r * (A2(D, i, 0) - A2(C, i, 0) * A2(D, i, 1));
        A2(A, i, 0) = r * A2(A, i, 0);
        A2(C, i, 0) = -r * A2(C, i, 0) * A2(C, i, 1);
        /* reduced rows (A_rd, B_rd=1, C_rd, D_rd) at j=1 and j=n_row */
        Ard[i] = A2(A, i, 0); Ard[i + n_sys] = A2(A, i, n_row - 1);
        Crd[i] = A2(C, i, 0); Crd[i + n_sys] = A2(C, i, n_row - 1);
        Drd[i] = A2(D, i, 0); Drd[i + n_sys] = A2(D, i, n_row - 1);
    }
}

static void modified_thomas_update(double *A, double *C, double *D, int n_sys, int n_row, const double *Drd)
{
    int i, j;
#pragma omp parallel for private(j)
    for (i = 0; i < n_sys; i++) {
        A2(D, i, 0) = Drd[i];
        A2(D, i, n_row - 1) = Drd[i + n_sys];
        for (j = 1; j < n_row - 1; j++)
            A2(D, i, j) = A2(D, i, j) - A2(A, i, j) * A2(D, i, 0) - A2(C, i, j) * A2(D, i, n_row - 1);
    }
}

void tcs_oracle_tdma_many(double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    double *Ard = dalloc(2 * (size_t)n_sys), *Crd = dalloc(2 * (size_t)n_sys), *Drd = dalloc(2 * (size_t)n_sys);
    int i;
    modified_thomas(A, B, C, D, n_sys, n_row, Ard, Crd, Drd);
    /* tdma_many on (n_sys, 2) with b = 1 (tdmas.f90:113-146) */
#pragma omp parallel for
    for (i = 0; i < n_sys; i++) {
        double d1 = Drd[i] / 1.0, c1 = Crd[i] / 1.0, d2, c2, r;
        r = 1.0 / (1.0 - Ard[i + n_sys] * c1);
        d2 = r * (Drd[i + n_sys] - Ard[i + n_sys] * d1);
        c2 = r * Crd[i + n_sys]; (void)c2;
        d1 = d1 - c1 * d2;
        Drd[i] = d1; Drd[i + n_sys] = d2;
    }
    modified_thomas_update(A, C, D, n_sys, n_row, Drd);
    free(Ard); free(Crd); free(Drd);
}

void tcs_oracle_tdma_many_cycle(double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    double *Ard = dalloc(2 * (size_t)n_sys), *Crd = dalloc(2 * (size_t)n_sys), *Drd = dalloc(2 * (size_t)n_sys);
    int i;
    modified_thomas(A, B, C, D, n_sys, n_row, Ard, Crd, Drd);
    /* tdma_cycl_many on (n_sys, 2) with b = 1 (tdmas.f90:159-212): e(2) = -a(2)
     * is immediately overwritten by e(n2) = -c(2), so A_rd(:,2) drops out. */
#pragma omp parallel for
    for (i = 0; i < n_sys; i++) {
        double a1 = Ard[i], c1 = Crd[i], d1 = Drd[i];
        double c2 = Crd[i + n_sys], d2 = Drd[i + n_sys];
        double e2 = -c2;
        d2 = d2 / 1.0; e2 = e2 / 1.0; c2 = c2 / 1.0;
        d1 = (d1 - a1 * d2 - c1 * d2) / (1.0 + a1 * e2 + c1 * e2);
        d2 = d2 + d1 * e2;
        Drd[i] = d1; Drd[i + n_sys] = d2;
    }
    modified_thomas_update(A, C, D, n_sys, n_row, Drd);
    free(Ard); free(Crd); free(Drd);
}
#undef A2

/* ---------------------------------------------------------------------------
 * FFT: stands in for FFTW3 (a third-party dependency the reference calls at
 * module_solve_pressure.f90:565-567, 586-588, 660-662, 681-683; version not
 * pinned by the reference build, src/Makefile:16).  FFTW computes the
 * unnormalised DFT  Y_k = sum_x X_x exp(sign * 2 pi i x k / n), sign = -1 for
 * FFTW_FORWARD; c2r ignores the imaginary parts of the k=0 and k=n/2 inputs.
 * This is a plain recursive mixed-radix decimation-in-time FFT.
 * ------------------------------------------------------------------------- */
static int smallest_factor(int n)
{
    int f;
    if (n % 4 == 0) return 4;
    for (f = 2; f * f <= n; f++) if (n % f == 0) return f;
    return n;
}

/* Twiddle table for length N: w[2e] = cos(2 pi e / N), w[2e+1] = sin(2 pi e / N). */
static double *twiddles(int N)
{
    double *w = dalloc(2 * (size_t)N);
    int e;
    for (e = 0; e < N; e++) {
        w[2 * e] = cos(2.0 * M_PI * (double)e / (double)N);
        w[2 * e + 1] = sin(2.0 * M_PI * (double)e / (double)N);
    }
    return w;
}

/* Decimation in time: X[t + u m] = sum_q W_n^{q (t + u m)} S_q[t], where S_q is
 * the length-m transform of the q-th decimated sequence.  W_n^e is read from
 * the length-N table at e * (N / n). */
static void fft_rec(int n, int stride, const double *in, double *out, int sign, double *tmp,
                    const double *w, int wstride)
{
    int r, m, q, t, u;
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    r = smallest_factor(n);
    m = n / r;
    for (q = 0; q < r; q++)
        fft_rec(m, stride * r, in + 2 * (size_t)q * stride, tmp + 2 * (size_t)q * m, sign, out, w, wstride * r);
    for (t = 0; t < m; t++) {
        for (u = 0; u < r; u++) {
            double sr = 0.0, si = 0.0;
            for (q = 0; q < r; q++) {
                long e = ((long)q * (long)(t + u * m)) % n;
                double c = w[2 * e * wstride], sn = sign * w[2 * e * wstride + 1];
                double xr = tmp[2 * ((size_t)q * m + t)], xi = tmp[2 * ((size_t)q * m + t) + 1];
                sr += xr * c - xi * sn;
                si += xr * sn + xi * c;
            }
            out[2 * ((size_t)t + (size_t)u * m)] = sr;
            out[2 * ((size_t)t + (size_t)u * m) + 1] = si;
        }
    }
}

/* One in-place transform of length n; w1, w2 are scratch of 2n doubles each. */
static void fft1(int n, double *data, int sign, double *w1, double *w2, const double *tw)
{
    memcpy(w1, data, sizeof(double) * 2 * (size_t)n);
    fft_rec(n, 1, w1, data, sign, w2, tw, 1);
}

int tcs_oracle_fft_c2c(int n, int howmany, double *data, int sign)
{
    int h;
    double *tw;
    if (n < 1 || (sign != 1 && sign != -1)) return -1;
    tw = twiddles(n);
#pragma omp parallel
    {
        double *w1 = dalloc(2 * (size_t)n), *w2 = dalloc(2 * (size_t)n);
#pragma omp for
        for (h = 0; h < howmany; h++) fft1(n, data + 2 * (size_t)n * h, sign, w1, w2, tw);
        free(w1); free(w2);
    }
    free(tw);
    return 0;
}

/* ---------------------------------------------------------------------------
 * module_solve_thermal.f90
 * ------------------------------------------------------------------------- */
/* :116-156 mpi_thermal_coeffi */
static void thermal_coeffi(tcs_oracle *s)
{
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 0; k <= s->n3sub; k++)
        for (j = 0; j <= s->n2sub; j++)
            for (i = 0; i <= s->n1sub; i++) {
                double tmp1 = s->p.DeltaT * F(s->T, i, j, k);
                double tmp2 = tmp1 * tmp1, tmp3 = tmp2 * tmp1, tmp4 = tmp3 * tmp1, tmp5 = tmp4 * tmp1;
                double q1, q2;
                F(s->KPP, i, j, k) = s->c10 * (1.0 + s->c11 * tmp1 + s->c12 * tmp2 + s->c13 * tmp3 + s->c14 * tmp4 + s->c15 * tmp5) / s->KPP0;
                F(s->dKPP, i, j, k) = s->c10 * (s->c11 + 2.0 * s->c12 * tmp1 + 3.0 * s->c13 * tmp2 + 4.0 * s->c14 * tmp3 + 5.0 * s->c15 * tmp4) / s->KPP0;
                F(s->invRhoCp, i, j, k) = s->Rho0 * s->Cp0
                    / (s->a10 + s->a10 * (s->a11 * tmp1 + s->a12 * tmp2 + s->a13 * tmp3 + s->a14 * tmp4 + s->a15 * tmp5))
                    / (s->b10 + s->b10 * (s->b11 * tmp1 + s->b12 * tmp2 + s->b13 * tmp3 + s->b14 * tmp4 + s->b15 * tmp5));
                q1 = (1.0 + s->a11 * tmp1 + s->a12 * tmp2 + s->a13 * tmp3);
                q2 = (1.0 + s->b11 * tmp1 + s->b12 * tmp2 + s->b13 * tmp3);
                F(s->dinvRhoCp, i, j, k) = -(s->b11 * (1.0 + 3.0 * s->a12 * tmp2 + 4.0 * s->a13 * tmp3)
                    + s->a11 * (1.0 + 2.0 * s->b11 * tmp1 + 3.0 * s->b12 * tmp2 + 4.0 * s->b13 * tmp3)
                    + tmp1 * (s->b12 * (2.0 + 5.0 * s->a13 * tmp3)
                              + s->a12 * (2.0 + 4.0 * s->b12 * tmp2 + 5.0 * s->b13 * tmp3)
                              + 3.0 * tmp1 * (s->a13 + s->b13 + 2.0 * s->a13 * s->b13 * tmp3)))
                    / (q1 * q1) / (q2 * q2);
            }
}

/* :175-532 mpi_thermal_solver */
static void thermal_solver(tcs_oracle *s)
{
    const int n1m = s->n1msub, n2m = s->n2msub, n3m = s->n3msub;
    const size_t nin = (size_t)n1m * n2m * n3m;
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Ct = s->Ct, dt = s->dt;
    double *T = s->T, *U = s->U, *V = s->V, *W = s->W;
    double *KPP = s->KPP, *dKPP = s->dKPP, *invRhoCp = s->invRhoCp, *dinvRhoCp = s->dinvRhoCp;
    double *RHS = dalloc(nin), *am = dalloc(nin), *ac = dalloc(nin), *ap = dalloc(nin), *RHSI, *RHSJ;
    int i, j, k;
    /* stale values left by the last stage-1 iteration (k=n3m, j=n2m): Appendix of the loop nest */
    const int jm_s = n2m - 1, jp_s = n2m + 1, km_s = n3m - 1, kp_s = n3m + 1;

    /* stage 1: z-direction (:236-361) */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++) {
        int km = k - 1, kp = k + 1;
        for (j = 1; j <= n2m; j++) {
            int jm = j - 1, jp = j + 1, jem = s->jC_BC[jm], jep = s->jC_BC[jp];
            for (i = 1; i <= n1m; i++) {
                int ip = i + 1, im = i - 1;
                double invRhoCpCt_half = 0.5 * Ct * F(invRhoCp, i, j, k);
                double dinvRhoCpCt_half = 0.5 * Ct * F(dinvRhoCp, i, j, k);
                double e1 = (dx1[i] * F(T, im, j, k) + dx1[im] * F(T, i, j, k)) * (0.5 / dmx1[i]);
                double e2 = (dx1[ip] * F(T, i, j, k) + dx1[i] * F(T, ip, j, k)) * (0.5 / dmx1[ip]);
                double e3 = (dx2[j] * F(T, i, jm, k) + dx2[jm] * F(T, i, j, k)) * (0.5 / dmx2[j]);
                double e4 = (dx2[jp] * F(T, i, j, k) + dx2[j] * F(T, i, jp, k)) * (0.5 / dmx2[jp]);
                double e5 = (dx3[k] * F(T, i, j, km) + dx3[km] * F(T, i, j, k)) * (0.5 / dmx3[k]);
                double e6 = (dx3[kp] * F(T, i, j, k) + dx3[k] * F(T, i, j, kp)) * (0.5 / dmx3[kp]);
                double dedx1 = (F(T, i, j, k) - F(T, im, j, k)) / dmx1[i];
                double dedx2 = (F(T, ip, j, k) - F(T, i, j, k)) / dmx1[ip];
                double dedy3 = (F(T, i, j, k) - F(T, i, jm, k)) / dmx2[j];
                double dedy4 = (F(T, i, jp, k) - F(T, i, j, k)) / dmx2[jp];
                double dedz5 = (F(T, i, j, k) - F(T, i, j, km)) / dmx3[k];
                double dedz6 = (F(T, i, j, kp) - F(T, i, j, k)) / dmx3[kp];
                double convect_e1 = (F(U, i, j, k) * dedx1 + F(U, ip, j, k) * dedx2) * 0.5;
                double convect_e2 = (F(V, i, j, k) * dedy3 + F(V, i, jp, k) * dedy4) * 0.5;
                double convect_e3 = (F(W, i, j, k) * dedz5 + F(W, i, j, kp) * dedz6) * 0.5;
                double rhs = -0.5 * (convect_e1 + convect_e2 + convect_e3);
                double kPP1 = 0.5 / dmx1[i] * (dx1[i] * F(KPP, im, j, k) + dx1[im] * F(KPP, i, j, k));
                double kPP2 = 0.5 / dmx1[ip] * (dx1[ip] * F(KPP, i, j, k) + dx1[i] * F(KPP, ip, j, k));
                double kPP3 = 0.5 / dmx2[j] * (dx2[j] * F(KPP, i, jm, k) + dx2[jm] * F(KPP, i, j, k));
                double kPP4 = 0.5 / dmx2[jp] * (dx2[jp] * F(KPP, i, j, k) + dx2[j] * F(KPP, i, jp, k));
                double kPP5 = 0.5 / dmx3[k] * (dx3[k] * F(KPP, i, j, km) + dx3[km] * F(KPP, i, j, k));
                double kPP6 = 0.5 / dmx3[kp] * (dx3[kp] * F(KPP, i, j, k) + dx3[k] * F(KPP, i, j, kp));
                double dkPP1 = 0.5 / dmx1[i] * (dx1[i] * F(dKPP, im, j, k) + dx1[im] * F(dKPP, i, j, k));
                double dkPP2 = 0.5 / dmx1[ip] * (dx1[ip] * F(dKPP, i, j, k) + dx1[i] * F(dKPP, ip, j, k));
                double dkPP3 = 0.5 / dmx2[j] * (dx2[j] * F(dKPP, i, jm, k) + dx2[jm] * F(dKPP, i, j, k));
                double dkPP4 = 0.5 / dmx2[jp] * (dx2[jp] * F(dKPP, i, j, k) + dx2[j] * F(dKPP, i, jp, k));
                double dkPP5 = 0.5 / dmx3[k] * (dx3[k] * F(dKPP, i, j, km) + dx3[km] * F(dKPP, i, j, k));
                double dkPP6 = 0.5 / dmx3[kp] * (dx3[kp] * F(dKPP, i, j, k) + dx3[k] * F(dKPP, i, j, kp));
                double viscous_e1 = (kPP2 * dedx2 - kPP1 * dedx1 - e2 * dkPP2 * dedx2 + e1 * dkPP1 * dedx1) / dx1[i];
                double viscous_e2 = (kPP4 * dedy4 - kPP3 * dedy3 - e4 * dkPP4 * dedy4 + e3 * dkPP3 * dedy3) / dx2[j];
                double viscous_e3 = (kPP6 * dedz6 - kPP5 * dedz5 - e6 * dkPP6 * dedz6 + e5 * dkPP5 * dedz5) / dx3[k];
                double ebc_up, ebc_down, eACK, eAPK, eAMK, eACI, eAPI, eAMI, eACJ, eAPJ, eAMJ;
                const double TBCup = s->Tup, TBCbt = s->Tbt;
                rhs = rhs + invRhoCpCt_half * (viscous_e1 + viscous_e2 + viscous_e3)
                    - dinvRhoCpCt_half * F(T, i, j, k) * ((kPP2 * dedx2 - kPP1 * dedx1) / dx1[i]
                                                        + (kPP4 * dedy4 - kPP3 * dedy3) / dx2[j]
                                                        + (kPP6 * dedz6 - kPP5 * dedz5) / dx3[k]);
                ebc_up = -0.25 * F(V, i, jp, k) / dmx2[jp] * TBCup;
                ebc_down = 0.25 * F(V, i, j, k) / dmx2[j] * TBCbt;
                ebc_up = ebc_up + invRhoCpCt_half / dx2[j] * kPP4 / dmx2[jp] * TBCup
                                + invRhoCpCt_half / dx2[j] * dkPP4 * dedy4 * TBCup;
                ebc_down = ebc_down + invRhoCpCt_half / dx2[j] * kPP3 / dmx2[j] * TBCbt
                                    - invRhoCpCt_half / dx2[j] * dkPP3 * dedy3 * TBCbt;
                rhs = rhs + (double)(1 - jem) * ebc_down + (double)(1 - jep) * ebc_up;
                eACK = invRhoCpCt_half / dx3[k] * (kPP6 / dmx3[kp] + kPP5 / dmx3[k]
                                                   - dx3[kp] * (0.5 / dmx3[kp]) * dkPP6 * dedz6
                                                   + dx3[km] * (0.5 / dmx3[k]) * dkPP5 * dedz5)
                     + (-0.25 * F(W, i, j, kp) / dmx3[kp] + 0.25 * F(W, i, j, k) / dmx3[k]);
                eAPK = -invRhoCpCt_half / dx3[k] * (kPP6 / dmx3[kp] + dx3[k] * (0.5 / dmx3[kp]) * dkPP6 * dedz6) + 0.25 * F(W, i, j, kp) / dmx3[kp];
                eAMK = -invRhoCpCt_half / dx3[k] * (kPP5 / dmx3[k] - dx3[k] * (0.5 / dmx3[k]) * dkPP5 * dedz5) - 0.25 * F(W, i, j, k) / dmx3[k];
                eACI = invRhoCpCt_half / dx1[i] * (kPP2 / dmx1[ip] + kPP1 / dmx1[i]
                                                   - dx1[ip] * (0.5 / dmx1[ip]) * dkPP2 * dedx2
                                                   + dx1[im] * (0.5 / dmx1[i]) * dkPP1 * dedx1)
                     + (0.25 * F(U, i, j, k) / dmx1[i] - 0.25 * F(U, ip, j, k) / dmx1[ip]);
                eAPI = -invRhoCpCt_half / dx1[i] * (kPP2 / dmx1[ip] + dx1[i] * (0.5 / dmx1[ip]) * dkPP2 * dedx2) + 0.25 * F(U, ip, j, k) / dmx1[ip];
                eAMI = -invRhoCpCt_half / dx1[i] * (kPP1 / dmx1[i] - dx1[i] * (0.5 / dmx1[i]) * dkPP1 * dedx1) - 0.25 * F(U, i, j, k) / dmx1[i];
                eACJ = invRhoCpCt_half / dx2[j] * (kPP4 / dmx2[jp] + kPP3 / dmx2[j]
                                                   - dx2[jp] * (0.5 / dmx2[jp]) * dkPP4 * dedy4 * (double)jep
                                                   + dx2[jm] * (0.5 / dmx2[j]) * dkPP3 * dedy3 * (double)jem)
                     + (0.25 * F(V, i, j, k) / dmx2[j] - 0.25 * F(V, i, jp, k) / dmx2[jp]);
                eAPJ = -invRhoCpCt_half / dx2[j] * (kPP4 / dmx2[jp] + dx2[j] * (0.5 / dmx2[jp]) * dkPP4 * dedy4) + 0.25 * F(V, i, jp, k) / dmx2[jp];
                eAMJ = -invRhoCpCt_half / dx2[j] * (kPP3 / dmx2[j] - dx2[j] * (0.5 / dmx2[j]) * dkPP3 * dedy3) - 0.25 * F(V, i, j, k) / dmx2[j];
                eAPJ = eAPJ * (double)jep;
                eAMJ = eAMJ * (double)jem;
                rhs = rhs - (eAPK * F(T, i, j, kp) + eACK * F(T, i, j, k) + eAMK * F(T, i, j, km)
                           + eAPJ * F(T, i, jp, k) + eACJ * F(T, i, j, k) + eAMJ * F(T, i, jm, k)
                           + eAPI * F(T, ip, j, k) + eACI * F(T, i, j, k) + eAMI * F(T, im, j, k)
                           - dinvRhoCpCt_half * F(T, i, j, k) * ((kPP2 * dedx2 - kPP1 * dedx1) / dx1[i]
                                                               + (kPP4 * dedy4 - kPP3 * dedy3) / dx2[j]
                                                               + (kPP6 * dedz6 - kPP5 * dedz5) / dx3[k]));
                ac[IN(s, i, j, k)] = eACK * dt
                    - 0.5 * dinvRhoCpCt_half * ((kPP2 * dedx2 - kPP1 * dedx1) / dx1[i]
                                               + (kPP4 * dedy4 - kPP3 * dedy3) / dx2[j]
                                               + (kPP6 * dedz6 - kPP5 * dedz5) / dx3[k]) * dt
                    + 1.0;
                ap[IN(s, i, j, k)] = eAPK * dt;
                am[IN(s, i, j, k)] = eAMK * dt;
                RHS[IN(s, i, j, k)] = rhs * dt;
            }
        }
    }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHS, n1m * n2m, n3m);   /* :364-366 */

    /* transpose (i,j,k) -> (j,k,i) (:372-379) */
    RHSI = dalloc(nin);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (i = 1; i <= n1m; i++)
            for (j = 1; j <= n2m; j++)
                RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))] = RHS[IN(s, i, j, k)];
    free(RHS);

    /* stage 2: x-direction with stale jm, jp, km, kp (:388-429) */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1, im = i - 1, jm = jm_s, jp = jp_s, km = km_s, kp = kp_s;
                double invRhoCpCt_half = 0.5 * Ct * F(invRhoCp, i, j, k);
                double kPP1 = 0.5 / dmx1[i] * (dx1[i] * F(KPP, im, j, k) + dx1[im] * F(KPP, i, j, k));
                double kPP2 = 0.5 / dmx1[ip] * (dx1[ip] * F(KPP, i, j, k) + dx1[i] * F(KPP, ip, j, k));
                double kPP3 = 0.5 / dmx2[j] * (dx2[j] * F(KPP, i, jm, k) + dx2[jm] * F(KPP, i, j, k));
                double kPP4 = 0.5 / dmx2[jp] * (dx2[jp] * F(KPP, i, j, k) + dx2[j] * F(KPP, i, jp, k));
                double kPP5 = 0.5 / dmx3[k] * (dx3[k] * F(KPP, i, j, km) + dx3[km] * F(KPP, i, j, k));
                double kPP6 = 0.5 / dmx3[kp] * (dx3[kp] * F(KPP, i, j, k) + dx3[k] * F(KPP, i, j, kp));
                double dkPP1 = 0.5 / dmx1[i] * (dx1[i] * F(dKPP, im, j, k) + dx1[im] * F(dKPP, i, j, k));
                double dkPP2 = 0.5 / dmx1[ip] * (dx1[ip] * F(dKPP, i, j, k) + dx1[i] * F(dKPP, ip, j, k));
                double dedx1 = (F(T, i, j, k) - F(T, im, j, k)) / dmx1[i];
                double dedx2 = (F(T, ip, j, k) - F(T, i, j, k)) / dmx1[ip];
                double dedy3 = (F(T, i, j, k) - F(T, i, jm, k)) / dmx2[j];
                double dedy4 = (F(T, i, jp, k) - F(T, i, j, k)) / dmx2[jp];
                double dedz5 = (F(T, i, j, k) - F(T, i, j, km)) / dmx3[k];
                double dedz6 = (F(T, i, j, kp) - F(T, i, j, k)) / dmx3[kp];
                double eACI = invRhoCpCt_half / dx1[i] * (kPP2 / dmx1[ip] + kPP1 / dmx1[i]
                                                          - dx1[ip] * (0.5 / dmx1[ip]) * dkPP2 * dedx2
                                                          + dx1[im] * (0.5 / dmx1[i]) * dkPP1 * dedx1)
                            + (0.25 * F(U, i, j, k) / dmx1[i] - 0.25 * F(U, ip, j, k) / dmx1[ip])
                            - 0.5 * invRhoCpCt_half * ((kPP2 * dedx2 - kPP1 * dedx1) / dx1[i]
                                                      + (kPP4 * dedy4 - kPP3 * dedy3) / dx2[j]
                                                      + (kPP6 * dedz6 - kPP5 * dedz5) / dx3[k]);
                double eAPI = -invRhoCpCt_half / dx1[i] * (kPP2 / dmx1[ip] + dx1[i] * (0.5 / dmx1[ip]) * dkPP2 * dedx2) + 0.25 * F(U, ip, j, k) / dmx1[ip];
                double eAMI = -invRhoCpCt_half / dx1[i] * (kPP1 / dmx1[i] - dx1[i] * (0.5 / dmx1[i]) * dkPP1 * dedx1) - 0.25 * F(U, i, j, k) / dmx1[i];
                size_t o = (size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1));
                ac[o] = eACI * dt + 1.0;
                ap[o] = eAPI * dt;
                am[o] = eAMI * dt;
            }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHSI, n2m * n3m, n1m);   /* :432-434 */

    /* transpose (j,k,i) -> (i,k,j) (:440-447) */
    RHSJ = dalloc(nin);
#pragma omp parallel for private(i, k)
    for (j = 1; j <= n2m; j++)
        for (k = 1; k <= n3m; k++)
            for (i = 1; i <= n1m; i++)
                RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))] =
                    RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))];
    free(RHSI);

    /* stage 3: y-direction with stale km, kp (:456-507) */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++) {
            const int jm = j - 1, jp = j + 1, jem = s->jC_BC[jm], jep = s->jC_BC[jp], km = km_s, kp = kp_s;
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1, im = i - 1;
                double invRhoCpCt_half = 0.5 * Ct * F(invRhoCp, i, j, k);
                double KPP1 = 0.5 / dmx1[i] * (dx1[i] * F(KPP, im, j, k) + dx1[im] * F(KPP, i, j, k));
                double KPP2 = 0.5 / dmx1[ip] * (dx1[ip] * F(KPP, i, j, k) + dx1[i] * F(KPP, ip, j, k));
                double kPP3 = 0.5 / dmx2[j] * (dx2[j] * F(KPP, i, jm, k) + dx2[jm] * F(KPP, i, j, k));
                double kPP4 = 0.5 / dmx2[jp] * (dx2[jp] * F(KPP, i, j, k) + dx2[j] * F(KPP, i, jp, k));
                double KPP5 = 0.5 / dmx3[k] * (dx3[k] * F(KPP, i, j, km) + dx3[km] * F(KPP, i, j, k));
                double KPP6 = 0.5 / dmx3[kp] * (dx3[kp] * F(KPP, i, j, k) + dx3[k] * F(KPP, i, j, kp));
                double dkPP3 = 0.5 / dmx2[j] * (dx2[j] * F(dKPP, i, jm, k) + dx2[jm] * F(dKPP, i, j, k));
                double dkPP4 = 0.5 / dmx2[jp] * (dx2[jp] * F(dKPP, i, j, k) + dx2[j] * F(dKPP, i, jp, k));
                double dedx1 = (F(T, i, j, k) - F(T, im, j, k)) / dmx1[i];
                double dedx2 = (F(T, ip, j, k) - F(T, i, j, k)) / dmx1[ip];
                double dedy3 = (F(T, i, j, k) - F(T, i, jm, k)) / dmx2[j];
                double dedy4 = (F(T, i, jp, k) - F(T, i, j, k)) / dmx2[jp];
                double dedz5 = (F(T, i, j, k) - F(T, i, j, km)) / dmx3[k];
                double dedz6 = (F(T, i, j, kp) - F(T, i, j, k)) / dmx3[kp];
                double eACJ = invRhoCpCt_half / dx2[j] * (kPP4 / dmx2[jp] + kPP3 / dmx2[j]
                                                          - dx2[jp] * (0.5 / dmx2[jp]) * dkPP4 * dedy4 * (double)jep
                                                          + dx2[jm] * (0.5 / dmx2[j]) * dkPP3 * dedy3 * (double)jem)
                            + (0.25 * F(V, i, j, k) / dmx2[j] - 0.25 * F(V, i, jp, k) / dmx2[jp])
                            - 0.5 * invRhoCpCt_half * ((KPP2 * dedx2 - KPP1 * dedx1) / dx1[i]
                                                      + (kPP4 * dedy4 - kPP3 * dedy3) / dx2[j]
                                                      + (KPP6 * dedz6 - KPP5 * dedz5) / dx3[k]);
                double eAPJ = -invRhoCpCt_half / dx2[j] * (kPP4 / dmx2[jp] + dx2[j] * (0.5 / dmx2[jp]) * dkPP4 * dedy4) + 0.25 * F(V, i, jp, k) / dmx2[jp];
                double eAMJ = -invRhoCpCt_half / dx2[j] * (kPP3 / dmx2[j] - dx2[j] * (0.5 / dmx2[j]) * dkPP3 * dedy3) - 0.25 * F(V, i, j, k) / dmx2[j];
                size_t o = (size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1));
                eAPJ = eAPJ * (double)jep;
                eAMJ = eAMJ * (double)jem;
                ac[o] = eACJ * dt + 1.0;
                ap[o] = eAPJ * dt;
                am[o] = eAMJ * dt;
            }
        }
    tcs_oracle_tdma_many(am, ac, ap, RHSJ, n3m * n1m, n2m);   /* :510-512 */

#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                F(T, i, j, k) = F(T, i, j, k) + RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))];
    free(RHSJ); free(am); free(ac); free(ap);
}

/* ---------------------------------------------------------------------------
 * module_solve_momentum.f90
 * ------------------------------------------------------------------------- */
/* :145-173 -- Mu(:,j,k) and invRho(:,j,k) are assigned whole rows inside the
 * i loop, so every row ends up holding the value of the last i (= n1sub). */
static void momentum_coeffi(tcs_oracle *s)
{
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 0; k <= s->n3sub; k++)
        for (j = 0; j <= s->n2sub; j++) {
            /* the row keeps the value computed at the last i, i = n1sub */
            double tmp1 = s->p.DeltaT * F(s->T, s->n1sub, j, k);
            double tmp2 = tmp1 * tmp1, tmp3 = tmp2 * tmp1, tmp4 = tmp3 * tmp1, tmp5 = tmp4 * tmp1;
            double mu = (s->a10 + s->a10 * (s->a11 * tmp1 + s->a12 * tmp2 + s->a13 * tmp3 + s->a14 * tmp4 + s->a15 * tmp5))
                      * (s->d10 + s->d10 * (s->d11 * tmp1 + s->d12 * tmp2 + s->d13 * tmp3 + s->d14 * tmp4 + s->d15 * tmp5)) / s->Mu0;
            double ir = s->Rho0 / (s->a10 + s->a10 * (s->a11 * tmp1 + s->a12 * tmp2 + s->a13 * tmp3 + s->a14 * tmp4 + s->a15 * tmp5));
            for (i = 0; i <= s->n1sub; i++) { F(s->Mu, i, j, k) = mu; F(s->invRho, i, j, k) = ir; }
        }
}

/* :178-208 */
static void momentum_pseudoupdate(tcs_oracle *s)
{
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        for (j = 2; j <= s->n2msub; j++)
            for (i = 1; i <= s->n1msub; i++) {
                F(s->U, i, j, k) = F(s->U, i, j, k) + F(s->dU, i, j, k);
                F(s->V, i, j, k) = F(s->V, i, j, k) + F(s->dV, i, j, k);
                F(s->W, i, j, k) = F(s->W, i, j, k) + F(s->dW, i, j, k);
            }
        j = 1;
        for (i = 1; i <= s->n1msub; i++) {
            F(s->U, i, j, k) = F(s->U, i, j, k) + F(s->dU, i, j, k);
            F(s->V, i, j, k) = F(s->V, i, j, k) + F(s->dV, i, j, k) * (double)(2 - s->j_indexS);
            F(s->W, i, j, k) = F(s->W, i, j, k) + F(s->dW, i, j, k);
        }
    }
}

/* :225-563 mpi_momentum_solvedU */
static void momentum_solvedU(tcs_oracle *s)
{
    const int n1m = s->n1msub, n2m = s->n2msub, n3m = s->n3msub;
    const size_t nin = (size_t)n1m * n2m * n3m;
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Cmu = s->Cmu, Cmp = s->Cmp, Cmt = s->Cmt, dt = s->dt, DeltaT = s->p.DeltaT, a12pera11 = s->a12pera11;
    const double UBCup = s->Uup, UBCbt = s->Ubt, VBCup = s->Vup, VBCbt = s->Vbt;
    double *U = s->U, *V = s->V, *W = s->W, *P = s->P, *T = s->T, *Mu = s->Mu, *invRho = s->invRho;
    double *RHS = dalloc(nin), *am = dalloc(nin), *ac = dalloc(nin), *ap = dalloc(nin), *RHSI, *RHSJ;
    int i, j, k;

#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++) {
        const int km = k - 1, kp = k + 1;
        for (j = 1; j <= n2m; j++) {
            const int jm = j - 1, jp = j + 1, jum = s->jC_BC[jm], jup = s->jC_BC[jp];
            for (i = s->i_indexS; i <= n1m; i++) {
                const int im = i - 1, ip = i + 1;
                double u1 = 0.5 * (F(U, im, j, k) + F(U, i, j, k));
                double u2 = 0.5 * (F(U, ip, j, k) + F(U, i, j, k));
                double v3 = 0.5 * (dx1[im] * F(V, i, j, k) + dx1[i] * F(V, im, j, k)) / dmx1[i];
                double v4 = 0.5 * (dx1[im] * F(V, i, jp, k) + dx1[i] * F(V, im, jp, k)) / dmx1[i];
                double w5 = 0.5 * (dx1[im] * F(W, i, j, k) + dx1[i] * F(W, im, j, k)) / dmx1[i];
                double w6 = 0.5 * (dx1[im] * F(W, i, j, kp) + dx1[i] * F(W, im, j, kp)) / dmx1[i];
                double dudx1 = (F(U, i, j, k) - F(U, im, j, k)) / dx1[im];
                double dudx2 = (F(U, ip, j, k) - F(U, i, j, k)) / dx1[i];
                double dudy3 = (F(U, i, j, k) - F(U, i, jm, k)) / dmx2[j];
                double dudy4 = (F(U, i, jp, k) - F(U, i, j, k)) / dmx2[jp];
                double dudz5 = (F(U, i, j, k) - F(U, i, j, km)) / dmx3[k];
                double dudz6 = (F(U, i, j, kp) - F(U, i, j, k)) / dmx3[kp];
                double dvdx3 = (F(V, i, j, k) - F(V, im, j, k)) / dmx1[i];
                double dvdx4 = (F(V, i, jp, k) - F(V, im, jp, k)) / dmx1[i];
                double dwdx5 = (F(W, i, j, k) - F(W, im, j, k)) / dmx1[i];
                double dwdx6 = (F(W, i, j, kp) - F(W, im, j, kp)) / dmx1[i];
                double mua = 0.5 * (dx1[im] * F(Mu, i, jm, k) + dx1[i] * F(Mu, im, jm, k)) / dmx1[i];
                double muc = 0.5 * (dx1[im] * F(Mu, i, j, k) + dx1[i] * F(Mu, im, j, k)) / dmx1[i];
                double mub = 0.5 * (dx1[im] * F(Mu, i, jp, k) + dx1[i] * F(Mu, im, jp, k)) / dmx1[i];
                double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) / dmx2[j];
                double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) / dmx2[jp];
                double mu5, mu6, invRhoc, invRhocCmu_half, viscous_u1, viscous_u2, viscous_u3, viscous_u12, viscous_u13;
                double rhs, Tc, ubc_down, ubc_up, mACI, mAPI, mAMI, mACJ, mAPJ, mAMJ, mACK, mAPK, mAMK;
                mua = 0.5 * (dx1[im] * F(Mu, i, j, km) + dx1[i] * F(Mu, im, j, km)) / dmx1[i];
                muc = 0.5 * (dx1[im] * F(Mu, i, j, k) + dx1[i] * F(Mu, im, j, k)) / dmx1[i];
                mub = 0.5 * (dx1[im] * F(Mu, i, j, kp) + dx1[i] * F(Mu, im, j, kp)) / dmx1[i];
                mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) / dmx3[k];
                mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) / dmx3[kp];
                invRhoc = 0.5 * (dx1[im] * F(invRho, i, j, k) + dx1[i] * F(invRho, im, j, k)) / dmx1[i];
                invRhocCmu_half = 0.5 * Cmu * invRhoc;
                viscous_u1 = 1.0 * (F(Mu, i, j, k) * dudx2 - F(Mu, im, j, k) * dudx1) / dmx1[i];
                viscous_u2 = 1.0 * (mu4 * dudy4 - mu3 * dudy3) / dx2[j];
                viscous_u3 = 1.0 * (mu6 * dudz6 - mu5 * dudz5) / dx3[k];
                viscous_u12 = 1.0 * (mu4 * dvdx4 - mu3 * dvdx3) / dx2[j];
                viscous_u13 = 1.0 * (mu6 * dwdx6 - mu5 * dwdx5) / dx3[k];
                rhs = invRhocCmu_half * (2.0 * viscous_u1 + viscous_u2 + viscous_u3 + viscous_u12 + viscous_u13);
                rhs = rhs - Cmp * invRhoc * (F(P, i, j, k) - F(P, im, j, k)) / dmx1[i];
                Tc = 0.5 * (dx1[im] * F(T, i, j, k) + dx1[i] * F(T, im, j, k)) / dmx1[i];
                rhs = rhs + Cmt * (Tc + a12pera11 * (Tc * Tc) * DeltaT) * invRhoc;
                ubc_down = 0.25 * v3 / dmx2[j] * UBCbt - 0.25 * dudy3 * (dx1[i] * VBCbt + dx1[im] * VBCbt) / dmx1[i] * 0.5;
                ubc_up = -0.25 * v4 / dmx2[jp] * UBCup - 0.25 * dudy4 * (dx1[i] * VBCup + dx1[im] * VBCup) / dmx1[i] * 0.5;
                ubc_down = ubc_down + invRhocCmu_half / dx2[j] * mu3 / dmx2[j] * UBCbt;
                ubc_down = ubc_down - invRhocCmu_half / dx2[j] * mu3 / dmx1[i] * (VBCbt - VBCbt);
                ubc_up = ubc_up + invRhocCmu_half / dx2[j] * mu4 / dmx2[jp] * UBCup;
                ubc_up = ubc_up + invRhocCmu_half / dx2[j] * mu4 / dmx1[i] * (VBCup - VBCup);
                rhs = rhs + (double)(1.0 - jum) * ubc_down + (double)(1.0 - jup) * ubc_up;
                mACI = invRhocCmu_half / dmx1[i] * (F(Mu, i, j, k) / dx1[i] + F(Mu, i, j, k) / dx1[im]) * 2.0
                     + 0.25 * (dudx2 * 0.5 + dudx1 * 0.5 - u2 / dx1[i] + u1 / dx1[im]);
                mAPI = -invRhocCmu_half / dmx1[i] * F(Mu, i, j, k) / dx1[i] * 2.0 + 0.25 * (u2 / dx1[i] + dudx2 * 0.5);
                mAMI = -invRhocCmu_half / dmx1[i] * F(Mu, i, j, k) / dx1[im] * 2.0 + 0.25 * (-u1 / dx1[im] + dudx1 * 0.5);
                mACJ = invRhocCmu_half / dx2[j] * (mu4 / dmx2[jp] + mu3 / dmx2[j]) + 0.25 * (-v4 / dmx2[jp] + v3 / dmx2[j]);
                mAPJ = -invRhocCmu_half / dx2[j] * mu4 / dmx2[jp] + 0.25 * (v4 / dmx2[jp]);
                mAMJ = -invRhocCmu_half / dx2[j] * mu3 / dmx2[j] + 0.25 * (-v3 / dmx2[j]);
                mAPJ = mAPJ * (double)jup;
                mAMJ = mAMJ * (double)jum;
                mACK = invRhocCmu_half / dx3[k] * (mu6 / dmx3[kp] + mu5 / dmx3[k]) + 0.25 * (-w6 / dmx3[kp] + w5 / dmx3[k]);
                mAPK = -invRhocCmu_half / dx3[k] * mu6 / dmx3[kp] + 0.25 * (w6 / dmx3[kp]);
                mAMK = -invRhocCmu_half / dx3[k] * mu5 / dmx3[k] + 0.25 * (-w5 / dmx3[k]);
                rhs = rhs - (mAPI * F(U, ip, j, k) + mACI * F(U, i, j, k) + mAMI * F(U, im, j, k)
                           + mAPJ * F(U, i, jp, k) + mACJ * F(U, i, j, k) + mAMJ * F(U, i, jm, k)
                           + mAPK * F(U, i, j, kp) + mACK * F(U, i, j, k) + mAMK * F(U, i, j, km));
                rhs = rhs - (0.25 * (v4 * (double)jup * dudy4 + v3 * (double)jum * dudy3)
                           - invRhocCmu_half / dx2[j] * (mu4 * dvdx4 * (double)jup - mu3 * dvdx3 * (double)jum));
                rhs = rhs - (0.25 * (w6 * dudz6 + w5 * dudz5)
                           - invRhocCmu_half / dx3[k] * (mu6 * dwdx6 - mu5 * dwdx5));
                ac[IN(s, i, j, k)] = mACK * dt + 1.0;
                ap[IN(s, i, j, k)] = mAPK * dt;
                am[IN(s, i, j, k)] = mAMK * dt;
                RHS[IN(s, i, j, k)] = rhs * dt;
            }
        }
    }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHS, n1m * n2m, n3m);

    RHSI = dalloc(nin);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = s->i_indexS; i <= n1m; i++)
                RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))] = RHS[IN(s, i, j, k)];
    free(RHS);

#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = s->i_indexS; i <= n1m; i++) {
                const int im = i - 1, ip = i + 1;
                double u1 = 0.5 * (F(U, im, j, k) + F(U, i, j, k));
                double u2 = 0.5 * (F(U, ip, j, k) + F(U, i, j, k));
                double dudx1 = (F(U, i, j, k) - F(U, im, j, k)) / dx1[im];
                double dudx2 = (F(U, ip, j, k) - F(U, i, j, k)) / dx1[i];
                double invRhoc = 0.5 * (dx1[im] * F(invRho, i, j, k) + dx1[i] * F(invRho, im, j, k)) / dmx1[i];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACI = invRhocCmu_half / dmx1[i] * (F(Mu, i, j, k) / dx1[i] + F(Mu, i, j, k) / dx1[im]) * 2.0
                            + 0.25 * (dudx2 * 0.5 + dudx1 * 0.5 - u2 / dx1[i] + u1 / dx1[im]);
                double mAPI = -invRhocCmu_half / dmx1[i] * F(Mu, i, j, k) / dx1[i] * 2.0 + 0.25 * (u2 / dx1[i] + dudx2 * 0.5);
                double mAMI = -invRhocCmu_half / dmx1[i] * F(Mu, i, j, k) / dx1[im] * 2.0 + 0.25 * (-u1 / dx1[im] + dudx1 * 0.5);
                size_t o = (size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1));
                ac[o] = mACI * dt + 1.0;
                ap[o] = mAPI * dt;
                am[o] = mAMI * dt;
            }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHSI, n2m * n3m, n1m);

    RHSJ = dalloc(nin);
#pragma omp parallel for private(i, k)
    for (j = 1; j <= n2m; j++)
        for (i = s->i_indexS; i <= n1m; i++)
            for (k = 1; k <= n3m; k++)
                RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))] =
                    RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))];
    free(RHSI);

#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++) {
            const int jm = j - 1, jp = j + 1, jum = s->jC_BC[jm], jup = s->jC_BC[jp];
            for (i = s->i_indexS; i <= n1m; i++) {
                const int im = i - 1;
                double v3 = 0.5 * (dx1[im] * F(V, i, j, k) + dx1[i] * F(V, im, j, k)) / dmx1[i];
                double v4 = 0.5 * (dx1[im] * F(V, i, jp, k) + dx1[i] * F(V, im, jp, k)) / dmx1[i];
                double mua = 0.5 * (dx1[im] * F(Mu, i, jm, k) + dx1[i] * F(Mu, im, jm, k)) / dmx1[i];
                double muc = 0.5 * (dx1[im] * F(Mu, i, j, k) + dx1[i] * F(Mu, im, j, k)) / dmx1[i];
                double mub = 0.5 * (dx1[im] * F(Mu, i, jp, k) + dx1[i] * F(Mu, im, jp, k)) / dmx1[i];
                double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) / dmx2[j];
                double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) / dmx2[jp];
                double invRhoc = 0.5 * (dx1[im] * F(invRho, i, j, k) + dx1[i] * F(invRho, im, j, k)) / dmx1[i];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACJ = invRhocCmu_half / dx2[j] * (mu4 / dmx2[jp] + mu3 / dmx2[j]) + 0.25 * (-v4 / dmx2[jp] + v3 / dmx2[j]);
                double mAPJ = -invRhocCmu_half / dx2[j] * mu4 / dmx2[jp] + 0.25 * (v4 / dmx2[jp]);
                double mAMJ = -invRhocCmu_half / dx2[j] * mu3 / dmx2[j] + 0.25 * (-v3 / dmx2[j]);
                size_t o = (size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1));
                mAPJ = mAPJ * (double)jup;
                mAMJ = mAMJ * (double)jum;
                ac[o] = mACJ * dt + 1.0;
                ap[o] = mAPJ * dt;
                am[o] = mAMJ * dt;
            }
        }
    tcs_oracle_tdma_many(am, ac, ap, RHSJ, n3m * n1m, n2m);

    /* dU is freshly allocated each step: zero it for determinism, then fill (:548-555) */
    memset(s->dU, 0, sizeof(double) * s->NP);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                F(s->dU, i, j, k) = RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))];
    free(RHSJ); free(am); free(ac); free(ap);
}

/* :569-924 mpi_momentum_solvedV.  Rows j=1 of the z and x stages are never
 * assigned in the reference (their lines carry uninitialised data that the y
 * transpose discards); here they are zero. */
static void momentum_solvedV(tcs_oracle *s)
{
    const int n1m = s->n1msub, n2m = s->n2msub, n3m = s->n3msub, jS = s->j_indexS;
    const size_t nin = (size_t)n1m * n2m * n3m;
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Cmu = s->Cmu, Cmp = s->Cmp, dt = s->dt;
    const double VBCup = s->Vup, VBCbt = s->Vbt;
    double *U = s->U, *V = s->V, *W = s->W, *P = s->P, *Mu = s->Mu, *invRho = s->invRho, *dU = s->dU;
    double *RHS = dalloc(nin), *am = dalloc(nin), *ac = dalloc(nin), *ap = dalloc(nin), *RHSI, *RHSJ;
    const int nyr = s->n2sub - jS;   /* rows of the y solve */
    double mu1_s = 0.0, mu2_s = 0.0;  /* stale from the last stage-1 iteration */
    int i, j, k;

#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++) {
        const int kp = k + 1, km = k - 1;
        for (j = jS; j <= n2m; j++) {
            const int jp = j + 1, jm = j - 1, jvp = s->jS_BC[jm], jvm = s->jS_BC[jp];
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1, im = i - 1;
                double v3 = 0.5 * (F(V, i, jm, k) + F(V, i, j, k));
                double v4 = 0.5 * (F(V, i, j, k) + F(V, i, jp, k));
                double u1 = (dx2[jm] * F(U, i, j, k) + dx2[j] * F(U, i, jm, k)) / dmx2[j] * 0.5;
                double u2 = (dx2[jm] * F(U, ip, j, k) + dx2[j] * F(U, ip, jm, k)) / dmx2[j] * 0.5;
                double w5 = (dx2[jm] * F(W, i, j, k) + dx2[j] * F(W, i, jm, k)) / dmx2[j] * 0.5;
                double w6 = (dx2[jm] * F(W, i, j, kp) + dx2[j] * F(W, i, jm, kp)) / dmx2[j] * 0.5;
                double ddu1 = (dx2[jm] * F(dU, i, j, k) + dx2[j] * F(dU, i, jm, k)) / dmx2[j] * 0.5;
                double ddu2 = (dx2[jm] * F(dU, ip, j, k) + dx2[j] * F(dU, ip, jm, k)) / dmx2[j] * 0.5;
                double dvdx1 = (F(V, i, j, k) - F(V, im, j, k)) / dmx1[i];
                double dvdx2 = (F(V, ip, j, k) - F(V, i, j, k)) / dmx1[ip];
                double dvdy3 = (F(V, i, j, k) - F(V, i, jm, k)) / dx2[jm];
                double dvdy4 = (F(V, i, jp, k) - F(V, i, j, k)) / dx2[j];
                double dvdz5 = (F(V, i, j, k) - F(V, i, j, km)) / dmx3[k];
                double dvdz6 = (F(V, i, j, kp) - F(V, i, j, k)) / dmx3[kp];
                double dudy1 = (F(U, i, j, k) - F(U, i, jm, k)) / dmx2[j];
                double dudy2 = (F(U, ip, j, k) - F(U, ip, jm, k)) / dmx2[j];
                double dwdy5 = (F(W, i, j, k) - F(W, i, jm, k)) / dmx2[j];
                double dwdy6 = (F(W, i, j, kp) - F(W, i, jm, kp)) / dmx2[j];
                double ddudy1 = (F(dU, i, j, k) - F(dU, i, jm, k)) / dmx2[j];
                double ddudy2 = (F(dU, ip, j, k) - F(dU, ip, jm, k)) / dmx2[j];
                double mua = 0.5 * (dx2[jm] * F(Mu, im, j, k) + dx2[j] * F(Mu, im, jm, k)) / dmx2[j];
                double muc = 0.5 * (dx2[jm] * F(Mu, i, j, k) + dx2[j] * F(Mu, i, jm, k)) / dmx2[j];
                double mub = 0.5 * (dx2[jm] * F(Mu, ip, j, k) + dx2[j] * F(Mu, ip, jm, k)) / dmx2[j];
                double mu1 = 0.5 * (dx1[im] * muc + dx1[i] * mua) / dmx1[i];
                double mu2 = 0.5 * (dx1[ip] * muc + dx1[i] * mub) / dmx1[ip];
                double mu5, mu6, invRhoc, invRhocCmu_half, viscous_v1, viscous_v2, viscous_v3, viscous_v21, viscous_v23;
                double rhs, vbc_down, vbc_up, mACI, mAPI, mAMI, mACJ, mAPJ, mAMJ, mACK, mAPK, mAMK;
                mua = 0.5 * (dx2[jm] * F(Mu, i, j, km) + dx2[j] * F(Mu, i, jm, km)) / dmx2[j];
                muc = 0.5 * (dx2[jm] * F(Mu, i, j, k) + dx2[j] * F(Mu, i, jm, k)) / dmx2[j];
                mub = 0.5 * (dx2[jm] * F(Mu, i, j, kp) + dx2[j] * F(Mu, i, jm, kp)) / dmx2[j];
                mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) / dmx3[k];
                mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) / dmx3[kp];
                invRhoc = 0.5 * (dx2[jm] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jm, k)) / dmx2[j];
                invRhocCmu_half = 0.5 * Cmu * invRhoc;
                viscous_v1 = 1.0 * (mu2 * dvdx2 - mu1 * dvdx1) / dx1[i];
                viscous_v2 = 1.0 * (F(Mu, i, j, k) * dvdy4 - F(Mu, i, jm, k) * dvdy3) / dmx2[j];
                viscous_v3 = 1.0 * (mu6 * dvdz6 - mu5 * dvdz5) / dx3[k];
                viscous_v21 = 1.0 * (mu2 * dudy2 - mu1 * dudy1) / dx1[i];
                viscous_v23 = 1.0 * (mu6 * dwdy6 - mu5 * dwdy5) / dx3[k];
                rhs = invRhocCmu_half * (viscous_v1 + 2. * viscous_v2 + viscous_v3 + viscous_v21 + viscous_v23);
                rhs = rhs - Cmp * invRhoc * (F(P, i, j, k) - F(P, i, jm, k)) / dmx2[j];
                vbc_down = (0.25 / dx2[jm] * v3 * VBCbt - 0.25 * 0.5 * dvdy3 * VBCbt);
                vbc_up = (-0.25 / dx2[j] * v4 * VBCup - 0.25 * 0.5 * dvdy4 * VBCup);
                vbc_down = vbc_down + invRhocCmu_half / dmx2[j] * F(Mu, i, jm, k) / dx2[jm] * VBCbt * 2.0;
                vbc_up = vbc_up + invRhocCmu_half / dmx2[j] * F(Mu, i, j, k) / dx2[j] * VBCup * 2.0;
                rhs = rhs + (double)(1.0 - jvm) * vbc_down + (double)(1.0 - jvp) * vbc_up;
                mACI = invRhocCmu_half / dx1[i] * (mu2 / dmx1[ip] + mu1 / dmx1[i]) + 0.25 * (-u2 / dmx1[ip] + u1 / dmx1[i]);
                mAPI = -invRhocCmu_half / dx1[i] * mu2 / dmx1[ip] + 0.25 * (u2 / dmx1[ip]);
                mAMI = -invRhocCmu_half / dx1[i] * mu1 / dmx1[i] + 0.25 * (-u1 / dmx1[i]);
                mACJ = invRhocCmu_half / dmx2[j] * (F(Mu, i, j, k) / dx2[j] + F(Mu, i, jm, k) / dx2[jm]) * 2.0
                     + 0.25 * (dvdy4 * 0.5 + dvdy3 * 0.5 - v4 / dx2[j] + v3 / dx2[jm]);
                mAPJ = -invRhocCmu_half / dmx2[j] * F(Mu, i, j, k) / dx2[j] * 2.0 + 0.25 * (v4 / dx2[j] + dvdy4 * 0.5);
                mAPJ = mAPJ * (double)jvp;
                mAMJ = -invRhocCmu_half / dmx2[j] * F(Mu, i, jm, k) / dx2[jm] * 2.0 + 0.25 * (-v3 / dx2[jm] + dvdy3 * 0.5);
                mAMJ = mAMJ * (double)jvm;
                mACK = invRhocCmu_half / dx3[k] * (mu6 / dmx3[kp] + mu5 / dmx3[k]) + 0.25 * (-w6 / dmx3[kp] + w5 / dmx3[k]);
                mAPK = -invRhocCmu_half / dx3[k] * mu6 / dmx3[kp] + 0.25 * (w6 / dmx3[kp]);
                mAMK = -invRhocCmu_half / dx3[k] * mu5 / dmx3[k] + 0.25 * (-w5 / dmx3[k]);
                rhs = rhs - (mAPI * F(V, ip, j, k) + mACI * F(V, i, j, k) + mAMI * F(V, im, j, k)
                           + mAPJ * F(V, i, jp, k) + mACJ * F(V, i, j, k) + mAMJ * F(V, i, jm, k)
                           + mAPK * F(V, i, j, kp) + mACK * F(V, i, j, k) + mAMK * F(V, i, j, km));
                rhs = rhs - (0.25 * (u2 * dvdx2 + u1 * dvdx1) - invRhocCmu_half / dx1[i] * (mu2 * dudy2 - mu1 * dudy1));
                rhs = rhs - (0.25 * (w6 * dvdz6 + w5 * dvdz5) - invRhocCmu_half / dx3[k] * (mu6 * dwdy6 - mu5 * dwdy5));
                rhs = rhs - (0.25 * (ddu2 * dvdx2 + ddu1 * dvdx1) - invRhocCmu_half / dx1[i] * (mu2 * ddudy2 - mu1 * ddudy1));
                ac[IN(s, i, j, k)] = mACK * dt + 1.0;
                ap[IN(s, i, j, k)] = mAPK * dt;
                am[IN(s, i, j, k)] = mAMK * dt;
                RHS[IN(s, i, j, k)] = rhs * dt;
                if (k == n3m && j == n2m && i == n1m) { mu1_s = mu1; mu2_s = mu2; }
            }
        }
    }
    /* rows j < j_indexS: identity lines (the reference leaves them unassigned) */
    for (k = 1; k <= n3m; k++)
        for (j = 1; j < jS; j++)
            for (i = 1; i <= n1m; i++) { ac[IN(s, i, j, k)] = 1.0; ap[IN(s, i, j, k)] = 0.0; am[IN(s, i, j, k)] = 0.0; RHS[IN(s, i, j, k)] = 0.0; }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHS, n1m * n2m, n3m);

    RHSI = dalloc(nin);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))] = RHS[IN(s, i, j, k)];
    free(RHS);

    /* stage 2 with the stale mu1, mu2 (:802-833) */
    for (k = 1; k <= n3m; k++)
        for (j = 1; j < jS; j++)
            for (i = 1; i <= n1m; i++) {
                size_t o = (size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1));
                ac[o] = 1.0; ap[o] = 0.0; am[o] = 0.0;
            }
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = jS; j <= n2m; j++) {
            const int jm = j - 1;
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1;
                const double mu1 = mu1_s, mu2 = mu2_s;
                double u1 = (dx2[jm] * F(U, i, j, k) + dx2[j] * F(U, i, jm, k)) / dmx2[j] * 0.5;
                double u2 = (dx2[jm] * F(U, ip, j, k) + dx2[j] * F(U, ip, jm, k)) / dmx2[j] * 0.5;
                double invRhoc = 0.5 * (dx2[jm] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jm, k)) / dmx2[j];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACI = invRhocCmu_half / dx1[i] * (mu2 / dmx1[ip] + mu1 / dmx1[i]) + 0.25 * (-u2 / dmx1[ip] + u1 / dmx1[i]);
                double mAPI = -invRhocCmu_half / dx1[i] * mu2 / dmx1[ip] + 0.25 * (u2 / dmx1[ip]);
                double mAMI = -invRhocCmu_half / dx1[i] * mu1 / dmx1[i] + 0.25 * (-u1 / dmx1[i]);
                size_t o = (size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1));
                ac[o] = mACI * dt + 1.0;
                ap[o] = mAPI * dt;
                am[o] = mAMI * dt;
            }
        }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHSI, n2m * n3m, n1m);

    RHSJ = dalloc((size_t)n1m * n3m * (size_t)nyr);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = jS; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - jS))] =
                    RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))];
    free(RHSI);

    /* stage 3: y, rows j = j_indexS..n2m; note jvp = jS_BC(jm) scales the
     * upper coefficient and jvm = jS_BC(jp) the lower one (:860-896). */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = jS; j <= n2m; j++) {
            const int jm = j - 1, jp = j + 1, jvp = s->jS_BC[jm], jvm = s->jS_BC[jp];
            for (i = 1; i <= n1m; i++) {
                double v3 = 0.5 * (F(V, i, jm, k) + F(V, i, j, k));
                double v4 = 0.5 * (F(V, i, j, k) + F(V, i, jp, k));
                double dvdy3 = (F(V, i, j, k) - F(V, i, jm, k)) / dx2[jm];
                double dvdy4 = (F(V, i, jp, k) - F(V, i, j, k)) / dx2[j];
                double invRhoc = 0.5 * (dx2[jm] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jm, k)) / dmx2[j];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACJ = invRhocCmu_half / dmx2[j] * (F(Mu, i, j, k) / dx2[j] + F(Mu, i, jm, k) / dx2[jm]) * 2.0
                            + 0.25 * (dvdy4 * 0.5 + dvdy3 * 0.5 - v4 / dx2[j] + v3 / dx2[jm]);
                double mAPJ = -invRhocCmu_half / dmx2[j] * F(Mu, i, j, k) / dx2[j] * 2.0 + 0.25 * (v4 / dx2[j] + dvdy4 * 0.5);
                double mAMJ;
                size_t o = (size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - jS));
                mAPJ = mAPJ * (double)jvp;
                mAMJ = -invRhocCmu_half / dmx2[j] * F(Mu, i, jm, k) / dx2[jm] * 2.0 + 0.25 * (-v3 / dx2[jm] + dvdy3 * 0.5);
                mAMJ = mAMJ * (double)jvm;
                ac[o] = mACJ * dt + 1.0;
                ap[o] = mAPJ * dt;
                am[o] = mAMJ * dt;
            }
        }
    tcs_oracle_tdma_many(am, ac, ap, RHSJ, n3m * n1m, nyr);

    memset(s->dV, 0, sizeof(double) * s->NP);   /* includes dV(:,0:1,:) = dV(:,n2sub,:) = 0 (:908-909) */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = jS; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                F(s->dV, i, j, k) = RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - jS))];
    free(RHSJ); free(am); free(ac); free(ap);
}

/* :930-1272 mpi_momentum_solvedW */
static void momentum_solvedW(tcs_oracle *s)
{
    const int n1m = s->n1msub, n2m = s->n2msub, n3m = s->n3msub;
    const size_t nin = (size_t)n1m * n2m * n3m;
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Cmu = s->Cmu, Cmp = s->Cmp, dt = s->dt;
    const double VBCup = s->Vup, VBCbt = s->Vbt, WBCup = s->Wup, WBCbt = s->Wbt;
    double *U = s->U, *V = s->V, *W = s->W, *P = s->P, *Mu = s->Mu, *invRho = s->invRho, *dU = s->dU, *dV = s->dV;
    double *RHS = dalloc(nin), *am = dalloc(nin), *ac = dalloc(nin), *ap = dalloc(nin), *RHSI, *RHSJ;
    double mu1_s = 0.0, mu2_s = 0.0, mu3_s = 0.0, mu4_s = 0.0;
    const int km_s = n3m - 1;   /* km left by the last stage-2 iteration */
    int i, j, k;

#pragma omp parallel for private(i, j)
    for (k = s->k_indexS; k <= n3m; k++) {
        const int kp = k + 1, km = k - 1;
        for (j = 1; j <= n2m; j++) {
            const int jp = j + 1, jm = j - 1, jwp = s->jC_BC[jp], jwm = s->jC_BC[jm];
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1, im = i - 1;
                double w5 = 0.5 * (F(W, i, j, k) + F(W, i, j, km));
                double w6 = 0.5 * (F(W, i, j, k) + F(W, i, j, kp));
                double u1 = (dx3[km] * F(U, i, j, k) + dx3[k] * F(U, i, j, km)) / dmx3[k] * 0.5;
                double u2 = (dx3[km] * F(U, ip, j, k) + dx3[k] * F(U, ip, j, km)) / dmx3[k] * 0.5;
                double v3 = (dx3[km] * F(V, i, j, k) + dx3[k] * F(V, i, j, km)) / dmx3[k] * 0.5;
                double v4 = (dx3[km] * F(V, i, jp, k) + dx3[k] * F(V, i, jp, km)) / dmx3[k] * 0.5;
                double dwdx1 = (F(W, i, j, k) - F(W, im, j, k)) / dmx1[i];
                double dwdx2 = (F(W, ip, j, k) - F(W, i, j, k)) / dmx1[ip];
                double dwdy3 = (F(W, i, j, k) - F(W, i, jm, k)) / dmx2[j];
                double dwdy4 = (F(W, i, jp, k) - F(W, i, j, k)) / dmx2[jp];
                double dwdz5 = (F(W, i, j, k) - F(W, i, j, km)) / dx3[km];
                double dwdz6 = (F(W, i, j, kp) - F(W, i, j, k)) / dx3[k];
                double dudz1 = (F(U, i, j, k) - F(U, i, j, km)) / dmx3[k];
                double dudz2 = (F(U, ip, j, k) - F(U, ip, j, km)) / dmx3[k];
                double dvdz3 = (F(V, i, j, k) - F(V, i, j, km)) / dmx3[k];
                double dvdz4 = (F(V, i, jp, k) - F(V, i, jp, km)) / dmx3[k];
                double ddudz1 = (F(dU, i, j, k) - F(dU, i, j, km)) / dmx3[k];
                double ddudz2 = (F(dU, ip, j, k) - F(dU, ip, j, km)) / dmx3[k];
                double ddvdz3 = (F(dV, i, j, k) - F(dV, i, j, km)) / dmx3[k];
                double ddvdz4 = (F(dV, i, jp, k) - F(dV, i, jp, km)) / dmx3[k];
                double ddu1 = (dx3[km] * F(dU, i, j, k) + dx3[k] * F(dU, i, j, km)) / dmx3[k] * 0.5;
                double ddu2 = (dx3[km] * F(dU, ip, j, k) + dx3[k] * F(dU, ip, j, km)) / dmx3[k] * 0.5;
                double ddv3 = (dx3[km] * F(dV, i, j, k) + dx3[k] * F(dV, i, j, km)) / dmx3[k] * 0.5 * (double)jwm;
                double ddv4 = (dx3[km] * F(dV, i, jp, k) + dx3[k] * F(dV, i, jp, km)) / dmx3[k] * 0.5 * (double)jwp;
                double mua = 0.5 * (dx3[km] * F(Mu, im, j, k) + dx3[k] * F(Mu, im, j, km)) / dmx3[k];
                double muc = 0.5 * (dx3[km] * F(Mu, i, j, k) + dx3[k] * F(Mu, i, j, km)) / dmx3[k];
                double mub = 0.5 * (dx3[km] * F(Mu, ip, j, k) + dx3[k] * F(Mu, ip, j, km)) / dmx3[k];
                double mu1 = 0.5 * (dx1[im] * muc + dx1[i] * mua) / dmx1[i];
                double mu2 = 0.5 * (dx1[ip] * muc + dx1[i] * mub) / dmx1[ip];
                double mu3, mu4, invRhoc, invRhocCmu_half, viscous_w1, viscous_w2, viscous_w3, viscous_w31, viscous_w32;
                double rhs, zbc_down, zbc_up, mACI, mAPI, mAMI, mACJ, mAPJ, mAMJ, mACK, mAPK, mAMK;
                mua = 0.5 * (dx3[km] * F(Mu, i, jm, k) + dx3[k] * F(Mu, i, jm, km)) / dmx3[k];
                muc = 0.5 * (dx3[km] * F(Mu, i, j, k) + dx3[k] * F(Mu, i, j, km)) / dmx3[k];
                mub = 0.5 * (dx3[km] * F(Mu, i, jp, k) + dx3[k] * F(Mu, i, jp, km)) / dmx3[k];
                mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) / dmx2[j];
                mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) / dmx2[jp];
                invRhoc = 0.5 * (dx3[km] * F(invRho, i, j, k) + dx3[k] * F(invRho, i, j, km)) / dmx3[k];
                invRhocCmu_half = 0.5 * Cmu * invRhoc;
                viscous_w1 = 1.0 * (mu2 * dwdx2 - mu1 * dwdx1) / dx1[i];
                viscous_w2 = 1.0 * (mu4 * dwdy4 - mu3 * dwdy3) / dx2[j];
                viscous_w3 = 1.0 * (F(Mu, i, j, k) * dwdz6 - F(Mu, i, j, km) * dwdz5) / dmx3[k];
                viscous_w31 = 1.0 * (mu2 * dudz2 - mu1 * dudz1) / dx1[i];
                viscous_w32 = 1.0 * (mu4 * dvdz4 - mu3 * dvdz3) / dx2[j];
                rhs = invRhocCmu_half * (viscous_w1 + viscous_w2 + 2. * viscous_w3 + viscous_w31 + viscous_w32);
                rhs = rhs - Cmp * invRhoc * (F(P, i, j, k) - F(P, i, j, km)) / dmx3[k];
                zbc_down = 0.25 * v3 / dmx2[j] * WBCbt - 0.25 * dwdy3 * (dx3[km] * VBCbt + dx3[k] * VBCbt) / dmx3[k] * 0.5;
                zbc_up = -0.25 * v4 / dmx2[jp] * WBCup - 0.25 * dwdy4 * (dx3[km] * VBCup + dx3[k] * VBCup) / dmx3[k] * 0.5;
                zbc_down = zbc_down + invRhocCmu_half / dx2[j] * mu3 / dmx2[jp] * WBCbt;
                zbc_up = zbc_up + invRhocCmu_half / dx2[j] * mu4 / dmx2[j] * WBCup;
                zbc_down = zbc_down - invRhocCmu_half / dx2[j] * mu3 / dmx3[k] * (VBCbt - VBCbt);
                zbc_up = zbc_up + invRhocCmu_half / dx2[j] * mu4 / dmx3[k] * (VBCup - VBCup);
                rhs = rhs + (double)(1.0 - jwm) * zbc_down + (double)(1.0 - jwp) * zbc_up;
                mACI = invRhocCmu_half / dx1[i] * (mu2 / dmx1[ip] + mu1 / dmx1[i]) + 0.25 * (-u2 / dmx1[ip] + u1 / dmx1[i]);
                mAPI = -invRhocCmu_half / dx1[i] * mu2 / dmx1[ip] + 0.25 * (u2 / dmx1[ip]);
                mAMI = -invRhocCmu_half / dx1[i] * mu1 / dmx1[i] + 0.25 * (-u1 / dmx1[i]);
                mACJ = invRhocCmu_half / dx2[j] * (mu4 / dmx2[jp] + mu3 / dmx2[j]) + 0.25 * (-v4 / dmx2[jp] + v3 / dmx2[j]);
                mAPJ = -invRhocCmu_half / dx2[j] * mu4 / dmx2[jp] + 0.25 * (v4 / dmx2[jp]);
                mAPJ = mAPJ * (double)jwp;
                mAMJ = -invRhocCmu_half / dx2[j] * mu3 / dmx2[j] + 0.25 * (-v3 / dmx2[j]);
                mAMJ = mAMJ * (double)jwm;
                mACK = invRhocCmu_half / dmx3[k] * (F(Mu, i, j, k) / dx3[k] + F(Mu, i, j, km) / dx3[km]) * 2.0
                     + 0.25 * (-w6 / dx3[k] + w5 / dx3[km] + 0.5 * dwdz6 + 0.5 * dwdz5);
                mAPK = -invRhocCmu_half / dmx3[k] * F(Mu, i, j, k) / dx3[k] * 2.0 + 0.25 * (w6 / dx3[k] + 0.5 * dwdz6);
                mAMK = -invRhocCmu_half / dmx3[k] * F(Mu, i, j, km) / dx3[km] * 2.0 + 0.25 * (-w5 / dx3[km] + 0.5 * dwdz5);
                rhs = rhs - (mAPI * F(W, ip, j, k) + mACI * F(W, i, j, k) + mAMI * F(W, im, j, k)
                           + mAPJ * F(W, i, jp, k) + mACJ * F(W, i, j, k) + mAMJ * F(W, i, jm, k)
                           + mAPK * F(W, i, j, kp) + mACK * F(W, i, j, k) + mAMK * F(W, i, j, km));
                rhs = rhs - (0.25 * (u2 * dwdx2 + u1 * dwdx1) - invRhocCmu_half / dx1[i] * (mu2 * dudz2 - mu1 * dudz1));
                rhs = rhs - (0.25 * (v3 * (double)jwm * dwdy3 + v4 * (double)jwp * dwdy4)
                           - invRhocCmu_half / dx2[j] * (mu4 * dvdz4 * (double)jwp - mu3 * dvdz3 * (double)jwm));
                rhs = rhs - (0.25 * (ddu2 * dwdx2 + ddu1 * dwdx1) - invRhocCmu_half / dx1[i] * (mu2 * ddudz2 - mu1 * ddudz1));
                rhs = rhs - (0.25 * (ddv3 * (double)jwm * dwdy3 + ddv4 * (double)jwp * dwdy4)
                           - invRhocCmu_half / dx2[j] * (mu4 * ddvdz4 * (double)jwp - mu3 * ddvdz3 * (double)jwm));
                ac[IN(s, i, j, k)] = mACK * dt + 1.0;
                ap[IN(s, i, j, k)] = mAPK * dt;
                am[IN(s, i, j, k)] = mAMK * dt;
                RHS[IN(s, i, j, k)] = rhs * dt;
                if (k == n3m && j == n2m && i == n1m) { mu1_s = mu1; mu2_s = mu2; mu3_s = mu3; mu4_s = mu4; }
            }
        }
    }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHS, n1m * n2m, n3m);

    RHSI = dalloc(nin);
#pragma omp parallel for private(i, j)
    for (k = s->k_indexS; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))] = RHS[IN(s, i, j, k)];
    free(RHS);

    /* stage 2 with stale mu1, mu2 (:1156-1189) */
#pragma omp parallel for private(i, j)
    for (k = s->k_indexS; k <= n3m; k++) {
        const int km = k - 1;
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++) {
                const int ip = i + 1;
                const double mu1 = mu1_s, mu2 = mu2_s;
                double u1 = (dx3[km] * F(U, i, j, k) + dx3[k] * F(U, i, j, km)) / dmx3[k] * 0.5;
                double u2 = (dx3[km] * F(U, ip, j, k) + dx3[k] * F(U, ip, j, km)) / dmx3[k] * 0.5;
                double invRhoc = 0.5 * (dx3[km] * F(invRho, i, j, k) + dx3[k] * F(invRho, i, j, km)) / dmx3[k];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACI = invRhocCmu_half / dx1[i] * (mu2 / dmx1[ip] + mu1 / dmx1[i]) + 0.25 * (-u2 / dmx1[ip] + u1 / dmx1[i]);
                double mAPI = -invRhocCmu_half / dx1[i] * mu2 / dmx1[ip] + 0.25 * (u2 / dmx1[ip]);
                double mAMI = -invRhocCmu_half / dx1[i] * mu1 / dmx1[i] + 0.25 * (-u1 / dmx1[i]);
                size_t o = (size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1));
                ac[o] = mACI * dt + 1.0;
                ap[o] = mAPI * dt;
                am[o] = mAMI * dt;
            }
    }
    tcs_oracle_tdma_many_cycle(am, ac, ap, RHSI, n2m * n3m, n1m);

    RHSJ = dalloc(nin);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))] =
                    RHSI[(size_t)(j - 1) + (size_t)n2m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(i - 1))];
    free(RHSI);

    /* stage 3 with stale km (from stage 2) and stale mu3, mu4 (from stage 1) (:1216-1246) */
#pragma omp parallel for private(i, j)
    for (k = s->k_indexS; k <= n3m; k++)
        for (j = 1; j <= n2m; j++) {
            const int jm = j - 1, jp = j + 1, jwp = s->jC_BC[jp], jwm = s->jC_BC[jm], km = km_s;
            (void)jm;
            for (i = 1; i <= n1m; i++) {
                const double mu3 = mu3_s, mu4 = mu4_s;
                double v3 = (dx3[km] * F(V, i, j, k) + dx3[k] * F(V, i, j, km)) / dmx3[k] * 0.5;
                double v4 = (dx3[km] * F(V, i, jp, k) + dx3[k] * F(V, i, jp, km)) / dmx3[k] * 0.5;
                double invRhoc = 0.5 * (dx3[km] * F(invRho, i, j, k) + dx3[k] * F(invRho, i, j, km)) / dmx3[k];
                double invRhocCmu_half = 0.5 * Cmu * invRhoc;
                double mACJ = invRhocCmu_half / dx2[j] * (mu4 / dmx2[jp] + mu3 / dmx2[j]) + 0.25 * (-v4 / dmx2[jp] + v3 / dmx2[j]);
                double mAPJ = -invRhocCmu_half / dx2[j] * mu4 / dmx2[jp] + 0.25 * (v4 / dmx2[jp]);
                double mAMJ;
                size_t o = (size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1));
                mAPJ = mAPJ * (double)jwp;
                mAMJ = -invRhocCmu_half / dx2[j] * mu3 / dmx2[j] + 0.25 * (-v3 / dmx2[j]);
                mAMJ = mAMJ * (double)jwm;
                ac[o] = mACJ * dt + 1.0;
                ap[o] = mAPJ * dt;
                am[o] = mAMJ * dt;
            }
        }
    tcs_oracle_tdma_many(am, ac, ap, RHSJ, n3m * n1m, n2m);

    memset(s->dW, 0, sizeof(double) * s->NP);
#pragma omp parallel for private(i, j)
    for (k = s->k_indexS; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                F(s->dW, i, j, k) = RHSJ[(size_t)(i - 1) + (size_t)n1m * ((size_t)(k - 1) + (size_t)n3m * (size_t)(j - 1))];
    free(RHSJ); free(am); free(ac); free(ap);
}

/* :1278-1356 */
static void momentum_blockLdV(tcs_oracle *s)
{
    const double *dx2 = s->dx2, *dx3 = s->dx3, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Cmu = s->Cmu, dt = s->dt;
    double *V = s->V, *dV = s->dV, *dW = s->dW, *Mu = s->Mu, *invRho = s->invRho;
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        const int kp = k + 1, km = k - 1;
        for (j = s->j_indexS; j <= s->n2msub; j++) {
            const int jm = j - 1;
            for (i = 1; i <= s->n1msub; i++) {
                double dwm5 = (dx2[jm] * F(dW, i, j, k) + dx2[j] * F(dW, i, jm, k)) / dmx2[j] * 0.5;
                double dwm6 = (dx2[jm] * F(dW, i, j, kp) + dx2[j] * F(dW, i, jm, kp)) / dmx2[j] * 0.5;
                double ddwdy5 = (F(dW, i, j, k) - F(dW, i, jm, k)) / dmx2[j];
                double ddwdy6 = (F(dW, i, j, kp) - F(dW, i, jm, kp)) / dmx2[j];
                double dvdz5 = (F(V, i, j, k) - F(V, i, j, km)) / dmx3[k];
                double dvdz6 = (F(V, i, j, kp) - F(V, i, j, k)) / dmx3[kp];
                double invRhoc = 0.5 * (dx2[jm] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jm, k)) / dmx2[j];
                double mua = 0.5 * (dx2[jm] * F(Mu, i, j, km) + dx2[j] * F(Mu, i, jm, km)) / dmx2[j];
                double muc = 0.5 * (dx2[jm] * F(Mu, i, j, k) + dx2[j] * F(Mu, i, jm, k)) / dmx2[j];
                double mub = 0.5 * (dx2[jm] * F(Mu, i, j, kp) + dx2[j] * F(Mu, i, jm, kp)) / dmx2[j];
                double mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) / dmx3[k];
                double mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) / dmx3[kp];
                F(dV, i, j, k) = F(dV, i, j, k)
                    - dt * (0.25 * (dwm5 * dvdz5 + dwm6 * dvdz6)
                            - 0.5 * Cmu * invRhoc / dx3[k] * (mu6 * ddwdy6 - mu5 * ddwdy5));
            }
        }
    }
}

/* :1362-1460 */
static void momentum_blockLdU(tcs_oracle *s)
{
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double Cmu = s->Cmu, dt = s->dt;
    double *U = s->U, *dU = s->dU, *dV = s->dV, *dW = s->dW, *Mu = s->Mu, *invRho = s->invRho;
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        const int km = k - 1, kp = k + 1;
        for (j = 1; j <= s->n2msub; j++) {
            const int jm = j - 1, jp = j + 1, jum = s->jC_BC[jm], jup = s->jC_BC[jp];
            for (i = 1; i <= s->n1msub; i++) {
                const int im = i - 1;
                double invRhoc = 0.5 * (dx1[im] * F(invRho, i, j, k) + dx1[i] * F(invRho, im, j, k)) / dmx1[i];
                double dvm3 = (dx1[i] * F(dV, im, j, k) + dx1[im] * F(dV, i, j, k)) / dmx1[i] * 0.5 * (double)jum;
                double dvm4 = (dx1[i] * F(dV, im, jp, k) + dx1[im] * F(dV, i, jp, k)) / dmx1[i] * 0.5 * (double)jup;
                double dudy3 = (F(U, i, j, k) - F(U, i, jm, k)) / dmx2[j];
                double dudy4 = (F(U, i, jp, k) - F(U, i, j, k)) / dmx2[jp];
                double dvmdx3 = (F(dV, i, j, k) - F(dV, im, j, k)) / dmx1[i] * (double)jum;
                double dvmdx4 = (F(dV, i, jp, k) - F(dV, im, jp, k)) / dmx1[i] * (double)jup;
                double mua = 0.5 * (dx1[im] * F(Mu, i, jm, k) + dx1[i] * F(Mu, im, jm, k)) / dmx1[i];
                double muc = 0.5 * (dx1[im] * F(Mu, i, j, k) + dx1[i] * F(Mu, im, j, k)) / dmx1[i];
                double mub = 0.5 * (dx1[im] * F(Mu, i, jp, k) + dx1[i] * F(Mu, im, jp, k)) / dmx1[i];
                double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) / dmx2[j];
                double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) / dmx2[jp];
                double dwm5 = (dx1[i] * F(dW, im, j, k) + dx1[im] * F(dW, i, j, k)) / dmx1[i] * 0.5;
                double dwm6 = (dx1[i] * F(dW, im, j, kp) + dx1[im] * F(dW, i, j, kp)) / dmx1[i] * 0.5;
                double dudz5 = (F(U, i, j, k) - F(U, i, j, km)) / dmx3[k];
                double dudz6 = (F(U, i, j, kp) - F(U, i, j, k)) / dmx3[kp];
                double dwmdx5 = (F(dW, i, j, k) - F(dW, im, j, k)) / dmx1[i];
                double dwmdx6 = (F(dW, i, j, kp) - F(dW, im, j, kp)) / dmx1[i];
                double mu5, mu6;
                mua = 0.5 * (dx1[im] * F(Mu, i, j, km) + dx1[i] * F(Mu, im, j, km)) / dmx1[i];
                muc = 0.5 * (dx1[im] * F(Mu, i, j, k) + dx1[i] * F(Mu, im, j, k)) / dmx1[i];
                mub = 0.5 * (dx1[im] * F(Mu, i, j, kp) + dx1[i] * F(Mu, im, j, kp)) / dmx1[i];
                mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) / dmx3[k];
                mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) / dmx3[kp];
                F(dU, i, j, k) = F(dU, i, j, k)
                    - dt * (0.25 * (dvm4 * dudy4 + dvm3 * dudy3) - 0.5 * Cmu * invRhoc / dx2[j] * (mu4 * dvmdx4 - mu3 * dvmdx3))
                    - dt * (0.25 * (dwm6 * dudz6 + dwm5 * dudz5) - 0.5 * Cmu * invRhoc / dx3[k] * (mu6 * dwmdx6 - mu5 * dwmdx5));
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * module_solve_pressure.f90
 * ------------------------------------------------------------------------- */
/* :93-129 */
static void pressure_wave_number(tcs_oracle *s)
{
    const double ddx = s->L1 / (double)s->n1m, ddz = s->L3 / (double)s->n3m;
    const double PI = acos(-1.0);
    int i, k;
    for (k = 1; k <= s->n3m; k++) {
        int km = (k <= s->h3p) ? k - 1 : s->n3m - k + 1;
        s->dzk[k - 1] = 2.0 * (1.0 - cos(2.0 * PI * (double)km * ddz / s->L3)) / (ddz * ddz);
    }
    for (i = 1; i <= s->h1p; i++) {
        int im = i - 1;
        s->dxk2[i - 1] = 2.0 * (1.0 - cos(2.0 * PI * (double)im * ddx / s->L1)) / (ddx * ddx);
    }
}

/* :140-231 */
static void pressure_RHS(tcs_oracle *s)
{
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double dt = s->dt, Cmp = s->Cmp, VBCup = s->Vup, VBCbt = s->Vbt;
    double *U = s->U, *V = s->V, *W = s->W, *dPhat = s->dPhat, *invRho = s->invRho;
    int i, j, k;
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        const int kp = k + 1, km = k - 1;
        for (j = 1; j <= s->n2msub; j++) {
            const int jp = j + 1, jm = j - 1, jvm = s->jC_BC[jm], jvp = s->jC_BC[jp];
            for (i = s->i_indexS; i <= s->n1msub; i++) {
                const int ip = i + 1, im = i - 1;
                double DivUm = (F(U, ip, j, k) - F(U, i, j, k)) / dx1[i]
                             + ((double)jvp * F(V, i, jp, k) - (double)jvm * F(V, i, j, k)) / dx2[j]
                             + (F(W, i, j, kp) - F(W, i, j, k)) / dx3[k];
                double cbc = (double)(1.0 - jvm) * VBCbt / dx2[j] - (double)(1.0 - jvp) * VBCup / dx2[j];
                double ddpdx1 = (F(dPhat, i, j, k) - F(dPhat, im, j, k)) / dmx1[i];
                double ddpdx2 = (F(dPhat, ip, j, k) - F(dPhat, i, j, k)) / dmx1[ip];
                double ddpdy3 = (F(dPhat, i, j, k) - F(dPhat, i, jm, k)) / dmx2[j];
                double ddpdy4 = (F(dPhat, i, jp, k) - F(dPhat, i, j, k)) / dmx2[jp];
                double ddpdz5 = (F(dPhat, i, j, k) - F(dPhat, i, j, km)) / dmx3[k];
                double ddpdz6 = (F(dPhat, i, j, kp) - F(dPhat, i, j, k)) / dmx3[kp];
                double invRho1 = 0.5 / dmx1[i] * (dx1[im] * F(invRho, i, j, k) + dx1[i] * F(invRho, im, j, k));
                double invRho2 = 0.5 / dmx1[ip] * (dx1[ip] * F(invRho, i, j, k) + dx1[i] * F(invRho, ip, j, k));
                double invRho3 = 0.5 / dmx2[j] * (dx2[jm] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jm, k));
                double invRho4 = 0.5 / dmx2[jp] * (dx2[jp] * F(invRho, i, j, k) + dx2[j] * F(invRho, i, jp, k));
                double invRho5 = 0.5 / dmx3[k] * (dx3[km] * F(invRho, i, j, k) + dx3[k] * F(invRho, i, j, km));
                double invRho6 = 0.5 / dmx3[kp] * (dx3[kp] * F(invRho, i, j, k) + dx3[k] * F(invRho, i, j, kp));
                double ExtraTerm = ((1.0 - invRho2) * ddpdx2 - (1.0 - invRho1) * ddpdx1) / dx1[i]
                                 + ((1.0 - invRho4) * ddpdy4 - (1.0 - invRho3) * ddpdy3) / dx2[j]
                                 + ((1.0 - invRho6) * ddpdz6 - (1.0 - invRho5) * ddpdz5) / dx3[k];
                s->PRHS[IN(s, i, j, k)] = (DivUm - cbc) / dt / Cmp + ExtraTerm;
            }
        }
    }
}

/* :489-744 (transpose scheme 2 on one rank: every Alltoallw is a copy) */
static void pressure_poisson(tcs_oracle *s)
{
    const int n1m = s->n1m, n2m = s->n2m, n3m = s->n3m, h1p = s->h1p, h3p = s->h3p;
    const double *dx2 = s->dx2, *dmx2 = s->dmx2;
    const size_t nsys = (size_t)n3m * h1p, nspec = nsys * n2m;
    /* RHSIKhat_Kline(1:n3m, 1:h1p, 1:n2m), interleaved complex */
    double *X = dalloc(2 * nspec);
    double *Am_r = dalloc(nspec), *Ac_r = dalloc(nspec), *Ap_r = dalloc(nspec), *Be_r = dalloc(nspec);
    double *Am_c = dalloc(nspec), *Ac_c = dalloc(nspec), *Ap_c = dalloc(nspec), *Be_c = dalloc(nspec);
    double *tmp, *tw1 = twiddles(n1m), *tw3 = twiddles(n3m);
    double AVERsub, AVERmpi, Pbc_a, Pbc_b;
    int i, j, k;
#define XS(kz, kx, jj) (2 * ((size_t)(kz) + (size_t)n3m * ((size_t)(kx) + (size_t)h1p * (size_t)(jj))))

    /* r2c along x (length n1m) for every (j,k), then c2c forward along z */
#pragma omp parallel for private(k, i)
    for (j = 0; j < n2m; j++) {
        double *line = dalloc(2 * (size_t)(n1m > n3m ? n1m : n3m)), *w1 = dalloc(2 * (size_t)(n1m > n3m ? n1m : n3m)), *w2 = dalloc(2 * (size_t)(n1m > n3m ? n1m : n3m));
        for (k = 0; k < n3m; k++) {
            for (i = 0; i < n1m; i++) { line[2 * i] = s->PRHS[IN(s, i + 1, j + 1, k + 1)]; line[2 * i + 1] = 0.0; }
            fft1(n1m, line, -1, w1, w2, tw1);
            for (i = 0; i < h1p; i++) { X[XS(k, i, j)] = line[2 * i]; X[XS(k, i, j) + 1] = line[2 * i + 1]; }
        }
        for (i = 0; i < h1p; i++) {
            for (k = 0; k < n3m; k++) { line[2 * k] = X[XS(k, i, j)]; line[2 * k + 1] = X[XS(k, i, j) + 1]; }
            fft1(n3m, line, -1, w1, w2, tw3);
            for (k = 0; k < n3m; k++) { X[XS(k, i, j)] = line[2 * k]; X[XS(k, i, j) + 1] = line[2 * k + 1]; }
        }
        free(line); free(w1); free(w2);
    }

    /* y-direction coefficients (:599-626) */
    for (j = 1; j <= n2m; j++) {
        const int jp = j + 1;
        double fft_amj = 1.0 / dx2[j] / dmx2[j];
        double fft_apj = 1.0 / dx2[j] / dmx2[jp];
        double fft_acj;
        if (j == 1) fft_amj = 0.0;
        if (j == n2m) fft_apj = 0.0;
        fft_acj = -fft_amj - fft_apj;
        for (i = 0; i < h1p; i++)
            for (k = 0; k < n3m; k++) {
                size_t o = (size_t)k + (size_t)n3m * ((size_t)i + (size_t)h1p * (size_t)(j - 1));
                Be_r[o] = X[XS(k, i, j - 1)];
                Be_c[o] = X[XS(k, i, j - 1) + 1];
                Am_r[o] = fft_amj;
                Ac_r[o] = fft_acj - s->dxk2[i] - s->dzk[k];
                Ap_r[o] = fft_apj;
                Am_c[o] = fft_amj;
                Ac_c[o] = fft_acj - s->dxk2[i] - s->dzk[k];
                Ap_c[o] = fft_apj;
            }
    }
    Am_r[0] = 0.0; Ac_r[0] = 1.0; Ap_r[0] = 0.0; Be_r[0] = 0.0;   /* :629-634 */
    tcs_oracle_tdma_many(Am_r, Ac_r, Ap_r, Be_r, (int)nsys, n2m);
    tcs_oracle_tdma_many(Am_c, Ac_c, Ap_c, Be_c, (int)nsys, n2m);
    for (j = 0; j < n2m; j++) {   /* :643-652 (h1psub_Ksub_ista == 1 on one rank) */
        Be_c[(size_t)0 + nsys * j] = 0.0;
        Be_c[(size_t)(h3p - 1) + nsys * j] = 0.0;
        for (i = 0; i < h1p; i++)
            for (k = 0; k < n3m; k++) {
                size_t o = (size_t)k + (size_t)n3m * ((size_t)i + (size_t)h1p * (size_t)j);
                X[XS(k, i, j)] = Be_r[o];
                X[XS(k, i, j) + 1] = Be_c[o];
            }
    }
    free(Am_r); free(Ac_r); free(Ap_r); free(Be_r); free(Am_c); free(Ac_c); free(Ap_c); free(Be_c);

    /* c2c backward along z, then c2r along x */
    tmp = dalloc((size_t)n1m * n2m * n3m);
#pragma omp parallel for private(k, i)
    for (j = 0; j < n2m; j++) {
        int nmax = n1m > n3m ? n1m : n3m;
        double *line = dalloc(2 * (size_t)nmax), *w1 = dalloc(2 * (size_t)nmax), *w2 = dalloc(2 * (size_t)nmax);
        for (i = 0; i < h1p; i++) {
            for (k = 0; k < n3m; k++) { line[2 * k] = X[XS(k, i, j)]; line[2 * k + 1] = X[XS(k, i, j) + 1]; }
            fft1(n3m, line, +1, w1, w2, tw3);
            for (k = 0; k < n3m; k++) { X[XS(k, i, j)] = line[2 * k]; X[XS(k, i, j) + 1] = line[2 * k + 1]; }
        }
        for (k = 0; k < n3m; k++) {
            /* c2r: Hermitian extension; imaginary parts of bins 0 and n/2 are ignored */
            for (i = 0; i < h1p; i++) { line[2 * i] = X[XS(k, i, j)]; line[2 * i + 1] = X[XS(k, i, j) + 1]; }
            line[1] = 0.0;
            if (n1m % 2 == 0) line[2 * (n1m / 2) + 1] = 0.0;
            for (i = h1p; i < n1m; i++) { line[2 * i] = line[2 * (n1m - i)]; line[2 * i + 1] = -line[2 * (n1m - i) + 1]; }
            fft1(n1m, line, +1, w1, w2, tw1);
            for (i = 0; i < n1m; i++) tmp[IN(s, i + 1, j + 1, k + 1)] = line[2 * i];
        }
        free(line); free(w1); free(w2);
    }
    free(X); free(tw1); free(tw3);
#undef XS

    /* scale (:694-700), unweighted mean (:703-714) */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                tmp[IN(s, i, j, k)] = tmp[IN(s, i, j, k)] / (double)n1m / (double)n3m;
    AVERsub = 0.0;
    for (k = 1; k <= n3m; k++) {
        double sk = 0.0;
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++) sk += tmp[IN(s, i, j, k)];
        AVERsub = AVERsub + sk;
    }
    AVERmpi = AVERsub / (double)n1m / (double)n2m / (double)n3m;
    memset(s->dP, 0, sizeof(double) * s->NP);   /* freshly allocated in the reference */
#pragma omp parallel for private(i, j)
    for (k = 1; k <= n3m; k++)
        for (j = 1; j <= n2m; j++)
            for (i = 1; i <= n1m; i++)
                F(s->dP, i, j, k) = tmp[IN(s, i, j, k)] - AVERmpi;
    free(tmp);

    /* wall extrapolation (:719-736) for k = 1..n3sub; the k = n3sub plane reads
     * rows that the ghost update overwrites right after. */
    Pbc_a = (dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) / ((dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) - dmx2[1] * dmx2[1]);
    Pbc_b = dmx2[1] * dmx2[1] / ((dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) - dmx2[1] * dmx2[1]);
    for (k = 1; k <= s->n3sub; k++)
        for (i = 1; i <= n1m; i++)
            F(s->dP, i, 0, k) = Pbc_a * F(s->dP, i, 1, k) - Pbc_b * F(s->dP, i, 2, k);
    {
        const int n2sub = s->n2sub, n2msub = s->n2msub;
        Pbc_a = (dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) / ((dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) - dmx2[n2sub] * dmx2[n2sub]);
        Pbc_b = dmx2[n2sub] * dmx2[n2sub] / ((dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) - dmx2[n2sub] * dmx2[n2sub]);
        for (k = 1; k <= s->n3sub; k++)
            for (i = 1; i <= n1m; i++)
                F(s->dP, i, n2sub, k) = Pbc_a * F(s->dP, i, n2msub, k) - Pbc_b * F(s->dP, i, n2sub - 2, k);
    }
    (void)dx2;
}

/* :756-874.  The reference sweeps k, then j = 2..n2m, then the j = 1 row, with
 * i innermost, updating dPhat in place; a cell's x-, y- and z-lower neighbours
 * have therefore already received their new dPhat when they were visited
 * earlier in the sweep.  This restatement keeps the sequential sweep. */
static void pressure_projection(tcs_oracle *s)
{
    const double *dx1 = s->dx1, *dx2 = s->dx2, *dx3 = s->dx3, *dmx1 = s->dmx1, *dmx2 = s->dmx2, *dmx3 = s->dmx3;
    const double dt = s->dt, Cmp = s->Cmp;
    double *U = s->U, *V = s->V, *W = s->W, *P = s->P, *dP = s->dP, *dPhat = s->dPhat, *dP0 = s->dP0, *invRho = s->invRho;
    const int n2sub = s->n2sub, n2msub = s->n2msub;
    int i, j, k;
    for (k = 1; k <= s->n3msub; k++) {
        const int km = k - 1;
        double Pbc_a, Pbc_b;
        for (j = 2; j <= n2msub; j++) {
            const int jm = j - 1;
            for (i = 1; i <= s->n1msub; i++) {
                const int im = i - 1;
                double invRhoc = 0.5 / dmx1[i] * (dx1[i] * F(invRho, im, j, k) + dx1[im] * F(invRho, i, j, k));
                F(U, i, j, k) = F(U, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, im, j, k)) / dmx1[i]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, im, j, k)) / dmx1[i]);
                invRhoc = 0.5 / dmx2[j] * (dx2[j] * F(invRho, i, jm, k) + dx2[jm] * F(invRho, i, j, k));
                F(V, i, j, k) = F(V, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, i, jm, k)) / dmx2[j]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, i, jm, k)) / dmx2[j]);
                invRhoc = 0.5 / dmx3[k] * (dx3[k] * F(invRho, i, j, km) + dx3[km] * F(invRho, i, j, k));
                F(W, i, j, k) = F(W, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, i, j, km)) / dmx3[k]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, i, j, km)) / dmx3[k]);
                F(P, i, j, k) = F(P, i, j, k) + F(dP, i, j, k);
                F(dP0, i, j, k) = (F(dPhat, i, j, k) + F(dP0, i, j, k)) / 2.0;
                F(dPhat, i, j, k) = 2.0 * F(dP, i, j, k) - F(dP0, i, j, k);
            }
        }
        j = 1;
        {
            const int jm = j - 1;
            for (i = 1; i <= s->n1msub; i++) {
                const int im = i - 1;
                double invRhoc = 0.5 / dmx1[i] * (dx1[i] * F(invRho, im, j, k) + dx1[im] * F(invRho, i, j, k));
                F(U, i, j, k) = F(U, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, im, j, k)) / dmx1[i]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, im, j, k)) / dmx1[i]);
                invRhoc = 0.5 / dmx2[j] * (dx2[j] * F(invRho, i, jm, k) + dx2[jm] * F(invRho, i, j, k));
                F(V, i, j, k) = F(V, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, i, jm, k)) / dmx2[j]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, i, jm, k)) / dmx2[j]) * (double)(2 - s->j_indexS);
                invRhoc = 0.5 / dmx3[k] * (dx3[k] * F(invRho, i, j, km) + dx3[km] * F(invRho, i, j, k));
                F(W, i, j, k) = F(W, i, j, k) - dt * Cmp * ((F(dP, i, j, k) - F(dP, i, j, km)) / dmx3[k]
                                + (invRhoc - 1.0) * (F(dPhat, i, j, k) - F(dPhat, i, j, km)) / dmx3[k]);
                F(P, i, j, k) = F(P, i, j, k) + F(dP, i, j, k);
                F(dP0, i, j, k) = (F(dPhat, i, j, k) + F(dP0, i, j, k)) / 2.0;
                F(dPhat, i, j, k) = 2.0 * F(dP, i, j, k) - F(dP0, i, j, k);
            }
        }
        Pbc_a = (dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) / ((dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) - dmx2[1] * dmx2[1]);
        Pbc_b = dmx2[1] * dmx2[1] / ((dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]) - dmx2[1] * dmx2[1]);
        for (i = 1; i <= s->n1sub - 1; i++) F(P, i, 0, k) = Pbc_a * F(P, i, 1, k) - Pbc_b * F(P, i, 2, k);
        Pbc_a = (dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) / ((dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) - dmx2[n2sub] * dmx2[n2sub]);
        Pbc_b = dmx2[n2sub] * dmx2[n2sub] / ((dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]) - dmx2[n2sub] * dmx2[n2sub]);
        for (i = 1; i <= s->n1sub - 1; i++) F(P, i, n2sub, k) = Pbc_a * F(P, i, n2msub, k) - Pbc_b * F(P, i, n2sub - 2, k);
    }
}

/* ---------------------------------------------------------------------------
 * module_post.f90:100-158 (Div), :168-230 (CFL) and the added diagnostics.
 * ------------------------------------------------------------------------- */
static double post_div(tcs_oracle *s)
{
    double mx = -INFINITY;
    int i, j, k;
    double *pk = dalloc((size_t)s->n3msub + 1);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        double m = -INFINITY;
        for (j = 1; j <= s->n2msub; j++)
            for (i = 1; i <= s->n1msub; i++) {
                double d = (F(s->U, i + 1, j, k) - F(s->U, i, j, k)) / s->dx1[i]
                         + (F(s->V, i, j + 1, k) - F(s->V, i, j, k)) / s->dx2[j]
                         + (F(s->W, i, j, k + 1) - F(s->W, i, j, k)) / s->dx3[k];
                if (d > m) m = d;
            }
        pk[k] = m;
    }
    for (k = 1; k <= s->n3msub; k++) if (pk[k] > mx) mx = pk[k];
    free(pk);
    return mx;
}

static void post_cfl(tcs_oracle *s)
{
    double mx = -INFINITY, newdt;
    int i, j, k;
    double *pk = dalloc((size_t)s->n3msub + 1);
#pragma omp parallel for private(i, j)
    for (k = 1; k <= s->n3msub; k++) {
        double m = -INFINITY;
        for (j = 1; j <= s->n2msub; j++)
            for (i = 1; i <= s->n1msub; i++) {
                double c = (fabs(F(s->U, i + 1, j, k) + F(s->U, i, j, k)) / 2.0) / s->dx1[i]
                         + (fabs(F(s->V, i, j + 1, k) + F(s->V, i, j, k)) / 2.0) / s->dx2[j]
                         + (fabs(F(s->W, i, j, k + 1) + F(s->W, i, j, k)) / 2.0) / s->dx3[k];
                if (c > m) m = c;
            }
        pk[k] = m;
    }
    for (k = 1; k <= s->n3msub; k++) if (pk[k] > mx) mx = pk[k];
    free(pk);
    if (s->p.fixed_dt) { s->CFL = s->dt * mx; return; }
    newdt = s->p.MaxCFL / mx;      /* +Inf when the velocity field is zero */
    if (newdt > s->dtMax) newdt = s->dtMax;
    s->dt = newdt;
    s->CFL = newdt * mx;
}

void tcs_oracle_diagnostics(const tcs_oracle *s, double *out)
{
    /* Nusselt numbers from the wall-normal gradient across the first and last
     * half cells, using the wall temperatures; kinetic energy volume average. */
    double nb = 0.0, nt = 0.0, ke = 0.0;
    int i, j, k;
    const double cnt = (double)s->n1m * (double)s->n3m;
    for (k = 1; k <= s->n3msub; k++)
        for (i = 1; i <= s->n1msub; i++) {
            nb += -(F(s->T, i, 1, k) - s->Tbt) / s->dmx2[1];
            nt += -(s->Tup - F(s->T, i, s->n2msub, k)) / s->dmx2[s->n2sub];
        }
    for (k = 1; k <= s->n3msub; k++) {
        double sk = 0.0;
        for (j = 1; j <= s->n2msub; j++)
            for (i = 1; i <= s->n1msub; i++) {
                double u = F(s->U, i, j, k), v = F(s->V, i, j, k), w = F(s->W, i, j, k);
                sk += (u * u + v * v + w * w) * s->dx1[i] * s->dx2[j] * s->dx3[k];
            }
        ke += sk;
    }
    out[0] = nb / cnt;
    out[1] = nt / cnt;
    out[2] = 0.5 * ke / (s->L1 * s->L2 * s->L3);
}

/* ---------------------------------------------------------------------------
 * Setup: main.f90:82-125 with the seeded initial temperature.
 * ------------------------------------------------------------------------- */
static uint64_t splitmix64_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

tcs_oracle *tcs_oracle_create(const tcs_oracle_params *p)
{
    tcs_oracle *s;
    int i, j, k;
    if (!p || p->n1m < 4 || p->n2m < 4 || p->n3m < 4) return NULL;
    s = (tcs_oracle *)calloc(1, sizeof(*s));
    s->p = *p;
    s->top_wall_mode = p->top_wall_mode;
    global_inputpara(s);
    s->n1sub = s->n1m + 1; s->n2sub = s->n2m + 1; s->n3sub = s->n3m + 1;
    s->n1msub = s->n1m; s->n2msub = s->n2m; s->n3msub = s->n3m;
    s->h1p = s->n1m / 2 + 1; s->h3p = s->n3m / 2 + 1;
    s->P1 = (size_t)s->n1sub + 1; s->P2 = (size_t)s->n2sub + 1; s->P3 = (size_t)s->n3sub + 1;
    s->NP = s->P1 * s->P2 * s->P3;
    s->x1 = dalloc(s->P1); s->dx1 = dalloc(s->P1); s->dmx1 = dalloc(s->P1);
    s->x2 = dalloc(s->P2); s->dx2 = dalloc(s->P2); s->dmx2 = dalloc(s->P2);
    s->x3 = dalloc(s->P3); s->dx3 = dalloc(s->P3); s->dmx3 = dalloc(s->P3);
    s->jC_BC = (int *)calloc(s->P2, sizeof(int)); s->jS_BC = (int *)calloc(s->P2, sizeof(int));
    subdomain_mesh(s);
    subdomain_indices(s);
    s->T = dalloc(s->NP); s->U = dalloc(s->NP); s->V = dalloc(s->NP); s->W = dalloc(s->NP); s->P = dalloc(s->NP);
    s->dPhat = dalloc(s->NP); s->dP0 = dalloc(s->NP); s->dU = dalloc(s->NP); s->dV = dalloc(s->NP); s->dW = dalloc(s->NP);
    s->dP = dalloc(s->NP);
    s->KPP = dalloc(s->NP); s->dKPP = dalloc(s->NP); s->invRhoCp = dalloc(s->NP); s->dinvRhoCp = dalloc(s->NP);
    s->Mu = dalloc(s->NP); s->invRho = dalloc(s->NP);
    s->PRHS = dalloc((size_t)s->n1m * s->n2m * s->n3m);
    s->dzk = dalloc((size_t)s->n3m); s->dxk2 = dalloc((size_t)s->h1p);

    /* mpi_thermal_initial / boundary (module_solve_thermal.f90:73-111) */
    for (k = 0; k <= s->n3sub; k++)
        for (i = 0; i <= s->n1sub; i++) {
            F(s->T, i, 0, k) = s->Tbt;
            if (s->top_wall_mode) F(s->T, i, s->n2sub, k) = s->Tup;
        }
    /* seeded interior temperature: conduction profile + uniform noise */
    if (p->init_mode == 0) {
        uint64_t base = splitmix64_mix(p->seed);
        for (k = 1; k <= s->n3m; k++)
            for (j = 1; j <= s->n2m; j++)
                for (i = 1; i <= s->n1m; i++) {
                    uint64_t lin = (uint64_t)IX(s, i, j, k);
                    uint64_t z = splitmix64_mix(base ^ lin);
                    double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
                    double yc = 0.5 * (s->x2[j] + s->x2[j + 1]);
                    F(s->T, i, j, k) = 0.5 - yc + p->noise_amp * (2.0 * u - 1.0);
                }
    }
    /* velocity/pressure zero (module_solve_momentum.f90:84-140), dPhat = dP0 = 0 */
    s->time = p->tStart;
    s->dt = p->dtStart;
    s->CFL = p->MaxCFL;
    pressure_wave_number(s);
    ghostcell_update(s, s->T);
    ghostcell_update(s, s->U);
    ghostcell_update(s, s->V);
    ghostcell_update(s, s->W);
    ghostcell_update(s, s->P);
    return s;
}

void tcs_oracle_destroy(tcs_oracle *s)
{
    if (!s) return;
    free(s->x1); free(s->dx1); free(s->dmx1); free(s->x2); free(s->dx2); free(s->dmx2);
    free(s->x3); free(s->dx3); free(s->dmx3); free(s->jC_BC); free(s->jS_BC);
    free(s->T); free(s->U); free(s->V); free(s->W); free(s->P); free(s->dPhat); free(s->dP0);
    free(s->dU); free(s->dV); free(s->dW); free(s->dP);
    free(s->KPP); free(s->dKPP); free(s->invRhoCp); free(s->dinvRhoCp); free(s->Mu); free(s->invRho);
    free(s->PRHS); free(s->dzk); free(s->dxk2);
    free(s);
}

int tcs_oracle_dims(const tcs_oracle *s, int *d)
{
    d[0] = (int)s->P1; d[1] = (int)s->P2; d[2] = (int)s->P3;
    return 0;
}

static double *field_ptr(const tcs_oracle *s, int which)
{
    switch (which) {
    case TCS_O_T: return s->T; case TCS_O_U: return s->U; case TCS_O_V: return s->V;
    case TCS_O_W: return s->W; case TCS_O_P: return s->P; case TCS_O_DPHAT: return s->dPhat;
    case TCS_O_DP0: return s->dP0; case TCS_O_DU: return s->dU; case TCS_O_DV: return s->dV;
    case TCS_O_DW: return s->dW; case TCS_O_DP: return s->dP; case TCS_O_MU: return s->Mu;
    case TCS_O_INVRHO: return s->invRho;
    default: return NULL;
    }
}

int tcs_oracle_get_field(const tcs_oracle *s, int which, double *out)
{
    double *a = field_ptr(s, which);
    if (!a) return -1;
    memcpy(out, a, sizeof(double) * s->NP);
    return 0;
}

int tcs_oracle_set_field(tcs_oracle *s, int which, const double *in)
{
    double *a = field_ptr(s, which);
    if (!a) return -1;
    memcpy(a, in, sizeof(double) * s->NP);
    return 0;
}

int tcs_oracle_get_metric(const tcs_oracle *s, int which, double *out)
{
    const double *src[9] = {s->x1, s->dx1, s->dmx1, s->x2, s->dx2, s->dmx2, s->x3, s->dx3, s->dmx3};
    size_t n[9] = {s->P1, s->P1, s->P1, s->P2, s->P2, s->P2, s->P3, s->P3, s->P3};
    if (which < 0 || which > 8) return -1;
    memcpy(out, src[which], sizeof(double) * n[which]);
    return 0;
}

void tcs_oracle_scalars(const tcs_oracle *s, double *out)
{
    out[0] = s->time; out[1] = s->dt; out[2] = s->CFL; out[3] = s->maxDivU;
    out[4] = s->Cmu; out[5] = s->Ct; out[6] = s->dtMax;
}

int tcs_oracle_get_prhs(const tcs_oracle *s, double *out)
{
    memcpy(out, s->PRHS, sizeof(double) * (size_t)s->n1m * s->n2m * s->n3m);
    return 0;
}

int tcs_oracle_set_prhs(tcs_oracle *s, const double *in)
{
    memcpy(s->PRHS, in, sizeof(double) * (size_t)s->n1m * s->n2m * s->n3m);
    return 0;
}

int tcs_oracle_set_dt(tcs_oracle *s, double dt)
{
    s->dt = dt;
    return 0;
}

int tcs_oracle_run_stage(tcs_oracle *s, int stage)
{
    switch (stage) {
    case TCS_O_S_THERMAL: thermal_coeffi(s); thermal_solver(s); break;
    case TCS_O_S_GHOST_T: ghostcell_update(s, s->T); break;
    case TCS_O_S_MOM_COEFFI: momentum_coeffi(s); break;
    case TCS_O_S_DU: momentum_solvedU(s); ghostcell_update(s, s->dU); break;
    case TCS_O_S_DV: momentum_solvedV(s); ghostcell_update(s, s->dV); break;
    case TCS_O_S_DW: momentum_solvedW(s); ghostcell_update(s, s->dW); break;
    case TCS_O_S_BLOCKLDV: momentum_blockLdV(s); ghostcell_update(s, s->dV); break;
    case TCS_O_S_BLOCKLDU: momentum_blockLdU(s); break;
    case TCS_O_S_PSEUDO:
        momentum_pseudoupdate(s);
        ghostcell_update(s, s->U); ghostcell_update(s, s->V); ghostcell_update(s, s->W);
        break;
    case TCS_O_S_PRHS: pressure_RHS(s); break;
    case TCS_O_S_POISSON: pressure_poisson(s); ghostcell_update(s, s->dP); break;
    case TCS_O_S_PROJECT:
        pressure_projection(s);
        ghostcell_update(s, s->U); ghostcell_update(s, s->V); ghostcell_update(s, s->W);
        ghostcell_update(s, s->P); ghostcell_update(s, s->dPhat);
        break;
    case TCS_O_S_POST:
        s->maxDivU = post_div(s);
        post_cfl(s);
        s->time = s->time + s->dt;
        break;
    default: return -1;
    }
    return 0;
}

/* main.f90:129-223, one iteration per step. */
int tcs_oracle_step(tcs_oracle *s, int nsteps, double *diag)
{
    int n, st;
    for (n = 0; n < nsteps; n++) {
        double dt_used = s->dt, d3[3];
        for (st = 0; st < TCS_O_S_POST; st++) tcs_oracle_run_stage(s, st);
        s->maxDivU = post_div(s);
        if (s->maxDivU >= 1.0e-3) return -(n + 1);   /* BLOW UP (main.f90:208-212) */
        post_cfl(s);
        /* time advances by the dt set for the next step (main.f90:218-221) */
        s->time = s->time + s->dt;
        if (diag) {
            tcs_oracle_diagnostics(s, d3);
            diag[n * TCS_O_D_N + TCS_O_D_DT] = dt_used;
            diag[n * TCS_O_D_N + TCS_O_D_TIME] = s->time;
            diag[n * TCS_O_D_N + TCS_O_D_MAXDIV] = s->maxDivU;
            diag[n * TCS_O_D_N + TCS_O_D_CFL] = s->CFL;
            diag[n * TCS_O_D_N + TCS_O_D_NUBOT] = d3[0];
            diag[n * TCS_O_D_N + TCS_O_D_NUTOP] = d3[1];
            diag[n * TCS_O_D_N + TCS_O_D_KE] = d3[2];
        }
    }
    return nsteps;
}
