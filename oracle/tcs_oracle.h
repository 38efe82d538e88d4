/*
 * tcs_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (C99, FP64, one rank, OpenMP over independent planes) of the
 * PaScaL_TCS per-timestep path: main.f90:82-223 and every routine it calls on
 * one MPI rank.  It is the test oracle for the CUDA library in pascal_tcs_b200/:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and never as the product path.
 *
 * Parity status: UNPINNED against the reference itself.  The reference is
 * Fortran 90 + MPI + FFTW (MKL) and none of those toolchains exist here; the
 * reference ships no golden vectors or tests.  The restatement is pinned
 * component-wise by mathematical known-answer tests instead (dense solves for
 * the tridiagonal routines, an O(n^2) DFT for the FFT, the discrete Poisson
 * residual, the post-projection divergence).
 */
#ifndef TCS_ORACLE_H
#define TCS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Run parameters: the PARA_INPUT.dat namelists (module_global.f90:83-105)
 * plus the additions the seeded benchmark cases need. */
typedef struct {
    int n1m, n2m, n3m;               /* &meshes */
    int uniform1, uniform2, uniform3;/* &uniform_mesh */
    double gamma1, gamma2, gamma3;   /* &mesh_stretch */
    double aspect1, H, aspect3;      /* &aspect_ratio */
    double Ra, Pr, DeltaT, MaxCFL;   /* &sim_parameter */
    double dtStart, tStart;          /* &sim_control */
    int property_set;                /* 0 constant (active in the reference), 1 water, 2 glycerol */
    int fixed_dt;                    /* 0: CFL-adaptive dt every step (reference); 1: keep dtStart */
    uint64_t seed;                   /* seeded initial temperature noise */
    double noise_amp;                /* 0.01 in the benchmark cases; 0 = reference's T=0 start */
    int init_mode;                   /* 0: conduction profile + noise; 1: reference (T=0 interior) */
    int top_wall_mode;               /* 0: one-rank reference (top ghost row of T stays 0);
                                        1: top ghost row = Tup, as on a y decomposition of >= 2 ranks */
} tcs_oracle_params;

/* Field identifiers for get/set (padded arrays, Fortran order, i fastest). */
enum {
    TCS_O_T = 0, TCS_O_U, TCS_O_V, TCS_O_W, TCS_O_P,
    TCS_O_DPHAT, TCS_O_DP0, TCS_O_DU, TCS_O_DV, TCS_O_DW, TCS_O_DP,
    TCS_O_MU, TCS_O_INVRHO, TCS_O_NFIELDS
};

/* Metric identifiers (arrays of length n+2, index 0..nsub). */
enum {
    TCS_O_X1 = 0, TCS_O_DX1, TCS_O_DMX1,
    TCS_O_X2, TCS_O_DX2, TCS_O_DMX2,
    TCS_O_X3, TCS_O_DX3, TCS_O_DMX3
};

/* Per-step diagnostics written by tcs_oracle_step (7 doubles per step). */
enum {
    TCS_O_D_DT = 0,     /* dt used by this step */
    TCS_O_D_TIME,       /* time after the step */
    TCS_O_D_MAXDIV,     /* signed max divergence (module_post.f90:100-158) */
    TCS_O_D_CFL,        /* CFL after the step's CFL update */
    TCS_O_D_NUBOT,      /* bottom-wall Nusselt number */
    TCS_O_D_NUTOP,      /* top-wall Nusselt number */
    TCS_O_D_KE,         /* volume-averaged kinetic energy */
    TCS_O_D_N
};

/* Stage identifiers for tcs_oracle_run_stage: the calls of main.f90:133-219 in order. */
enum {
    TCS_O_S_THERMAL = 0,   /* coeffi + solver + coeffi_clean (main.f90:133-139) */
    TCS_O_S_GHOST_T,       /* main.f90:142 */
    TCS_O_S_MOM_COEFFI,    /* main.f90:145 */
    TCS_O_S_DU,            /* solvedU + ghost(dU)  (main.f90:148-151) */
    TCS_O_S_DV,            /* solvedV + ghost(dV)  (main.f90:154-157) */
    TCS_O_S_DW,            /* solvedW + ghost(dW)  (main.f90:160-163) */
    TCS_O_S_BLOCKLDV,      /* blockLdV + ghost(dV) (main.f90:166-169) */
    TCS_O_S_BLOCKLDU,      /* main.f90:172 */
    TCS_O_S_PSEUDO,        /* pseudoupdate + ghost(U,V,W) (main.f90:175-180) */
    TCS_O_S_PRHS,          /* main.f90:183 */
    TCS_O_S_POISSON,       /* Poisson_FFT2 + ghost(dP) (main.f90:186-189) */
    TCS_O_S_PROJECT,       /* projection + ghost(U,V,W,P,dPhat) (main.f90:192-199) */
    TCS_O_S_POST,          /* Div, CFL, time update (main.f90:205-221) */
    TCS_O_S_N
};

typedef struct tcs_oracle tcs_oracle;

tcs_oracle *tcs_oracle_create(const tcs_oracle_params *p);
void tcs_oracle_destroy(tcs_oracle *s);
int  tcs_oracle_dims(const tcs_oracle *s, int *dims3);           /* padded (N1+2, N2+2, N3+2) */
int  tcs_oracle_get_field(const tcs_oracle *s, int which, double *out);
int  tcs_oracle_set_field(tcs_oracle *s, int which, const double *in);
int  tcs_oracle_get_metric(const tcs_oracle *s, int which, double *out);
int  tcs_oracle_step(tcs_oracle *s, int nsteps, double *diag);   /* diag: nsteps x TCS_O_D_N, may be NULL */
int  tcs_oracle_run_stage(tcs_oracle *s, int stage);
int  tcs_oracle_get_prhs(const tcs_oracle *s, double *out);       /* (n1m, n2m, n3m) interior, i fastest */
int  tcs_oracle_set_prhs(tcs_oracle *s, const double *in);
int  tcs_oracle_set_dt(tcs_oracle *s, double dt);
void tcs_oracle_scalars(const tcs_oracle *s, double *out);       /* time, dt, CFL, maxDivU, Cmu, Ct, dtMax */
void tcs_oracle_diagnostics(const tcs_oracle *s, double *out);   /* Nu_bot, Nu_top, KE */
int  tcs_oracle_set_threads(int nthreads);

/* PaScaL_TDMA one-rank restatements (pascal_tdma.f90:487-578, 715-806 with
 * tdmas.f90:113-212).  A,B,C,D are (n_sys, n_row), system index fastest;
 * D is overwritten by the solution, A and C are clobbered. */
void tcs_oracle_tdma_many(double *A, double *B, double *C, double *D, int n_sys, int n_row);
void tcs_oracle_tdma_many_cycle(double *A, double *B, double *C, double *D, int n_sys, int n_row);

/* Mixed-radix complex FFT (unnormalised, sign -1 forward, +1 backward),
 * interleaved re/im, `howmany` contiguous transforms of length n. */
int tcs_oracle_fft_c2c(int n, int howmany, double *data, int sign);

#ifdef __cplusplus
}
#endif
#endif
