/*
 * tcs.h -- C ABI of libtcs: the PaScaL_TCS per-timestep path on one B200.
 *
 * Every entry point takes plain pointers, sizes and a context handle, returns
 * an int status (TCS_OK = 0), and never blocks the host except where a scalar
 * or a host buffer is returned.  All names mirror the reference routine they
 * replace; the citation after each declaration is the reference interface
 * (path:line within the PaScaL_TCS source tree).
 *
 * Fields are the reference's padded arrays (0:n1sub, 0:n2sub, 0:n3sub),
 * n_sub = n_m + 1, Fortran order (i fastest), FP64.  They live on the device;
 * host arrays cross only through tcs_upload_field / tcs_download_field (the
 * continue-file reader and writer, and the instantaneous-field dump, are the
 * only reference call sites that need host data: main.f90:121-125, 209, 226-228).
 */
#ifndef TCS_H
#define TCS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define TCS_OK              0
#define TCS_ERR_ARG         1   /* bad argument, shape or handle */
#define TCS_ERR_CUDA        2   /* a CUDA call failed (see tcs_last_error) */
#define TCS_ERR_UNSUPPORTED 3   /* size or option outside what the kernels support */
#define TCS_ERR_BLOWUP      4   /* max divergence >= 1e-3 (main.f90:208-212) */
#define TCS_ERR_NOMEM       5   /* device allocation failed */
#define TCS_ERR_NONFINITE   6   /* a returned scalar is NaN or Inf */

/* Run configuration: the PARA_INPUT.dat namelists (module_global.f90:83-105)
 * plus the options of the seeded benchmark cases.  The layout of the leading
 * members is shared with the test oracle's parameter block. */
typedef struct tcs_config {
    int n1m, n2m, n3m;                /* &meshes */
    int uniform1, uniform2, uniform3; /* &uniform_mesh (x and z must be periodic) */
    double gamma1, gamma2, gamma3;    /* &mesh_stretch */
    double aspect1, H, aspect3;       /* &aspect_ratio */
    double Ra, Pr, DeltaT, MaxCFL;    /* &sim_parameter */
    double dtStart, tStart;           /* &sim_control */
    int property_set;                 /* 0 constant (module_global.f90:117-120), 1 water (:113-116), 2 glycerol (:129-132) */
    int fixed_dt;                     /* 0: dt = min(MaxCFL / max|u|/dx, dtMax) after every step (module_post.f90:222-226); 1: keep dtStart */
    uint64_t seed;                    /* initial temperature noise seed */
    double noise_amp;                 /* noise amplitude (0.01 in the benchmark cases) */
    int init_mode;                    /* 0: T = 0.5 - y + noise; 1: T = 0 interior (mpi_thermal_initial) */
    int top_wall_mode;                /* 0: top ghost row of T stays 0 as on one y rank (module_solve_thermal.f90:102-110); 1: = Tup */
    int device;                       /* CUDA device ordinal */
    int precision;                    /* TCS_PREC_FP64 (the reference's arithmetic) or TCS_PREC_FP32_MIXED */
} tcs_config;

/* numerical forms (tcs_config.precision).  FP32_MIXED stores the fields in FP32
 * and runs stencils, ADI sweeps and FFTs in FP32 with one FP64-residual
 * refinement pass per tridiagonal system; the modal pressure solves, the
 * pressure right-hand side, the projection and every reduction compute in
 * FP64.  The host interface moves FP64 arrays in both forms. */
enum { TCS_PREC_FP64 = 0, TCS_PREC_FP32_MIXED = 1 };

/* field identifiers */
enum {
    TCS_F_T = 0, TCS_F_U, TCS_F_V, TCS_F_W, TCS_F_P, TCS_F_DPHAT, TCS_F_DP0,
    TCS_F_DU, TCS_F_DV, TCS_F_DW, TCS_F_DP, TCS_F_MU, TCS_F_INVRHO, TCS_F_COUNT
};

/* device scalars returned by tcs_get_scalars */
enum {
    TCS_S_DT = 0, TCS_S_TIME, TCS_S_CFL, TCS_S_MAXDIV, TCS_S_NUBOT, TCS_S_NUTOP, TCS_S_KE,
    TCS_S_BLOWUP, TCS_S_AVER, TCS_S_STEP, TCS_S_FIXED_DT, TCS_S_COUNT
};

typedef struct tcs_ctx tcs_ctx;
typedef struct tcs_tdma_plan tcs_tdma_plan;

/* ---- set-up: main.f90:82-125 ------------------------------------------- */
/* global_inputpara + mpi_subdomain_make/mesh/indices + *_allocation/initial/boundary +
 * mpi_pressure_wave_number + the initial ghost updates (main.f90:82-109). */
int tcs_create(const tcs_config *cfg, tcs_ctx **out);
int tcs_destroy(tcs_ctx *ctx);                                     /* *_clean (main.f90:234-241) */
int tcs_set_stream(tcs_ctx *ctx, void *cuda_stream);               /* NULL: library-owned stream */
void *tcs_get_stream(tcs_ctx *ctx);
int tcs_dims(const tcs_ctx *ctx, int *padded3);                    /* (n1m+2, n2m+2, n3m+2) */
int tcs_upload_field(tcs_ctx *ctx, int field, const double *host); /* blocking copy of a padded host array */
int tcs_download_field(tcs_ctx *ctx, int field, double *host);
int tcs_upload_field_async(tcs_ctx *ctx, int field, const double *pinned_host);   /* on the context stream */
int tcs_download_field_async(tcs_ctx *ctx, int field, double *pinned_host);
int tcs_field_device_ptr(tcs_ctx *ctx, int field, void **dev);     /* current device buffer: double (FP64) or float (FP32_MIXED) */
int tcs_precision(const tcs_ctx *ctx);                             /* tcs_config.precision of the context */
int tcs_synchronize(tcs_ctx *ctx);
int tcs_set_dt(tcs_ctx *ctx, double dt);
int tcs_get_metric(const tcs_ctx *ctx, int which, double *out);    /* x1,dx1,dmx1,x2,...,dmx3 (0..8) */

/* ---- one time step, reference order (main.f90:133-221) ---------------- */
int tcs_thermal_coeffi(tcs_ctx *ctx);                  /* module_solve_thermal.f90:116  (fused: no work) */
int tcs_thermal_solver(tcs_ctx *ctx);                  /* module_solve_thermal.f90:175  (U,V,W are the context's) */
int tcs_thermal_coeffi_clean(tcs_ctx *ctx);            /* module_solve_thermal.f90:161  (no work) */
int tcs_subdomain_ghostcell_update(tcs_ctx *ctx, int field); /* module_mpi_subdomain.f90:758 */
int tcs_momentum_coeffi(tcs_ctx *ctx);                 /* module_solve_momentum.f90:145 */
int tcs_momentum_solvedU(tcs_ctx *ctx);                /* module_solve_momentum.f90:225 */
int tcs_momentum_solvedV(tcs_ctx *ctx);                /* module_solve_momentum.f90:569 */
int tcs_momentum_solvedW(tcs_ctx *ctx);                /* module_solve_momentum.f90:930 */
int tcs_momentum_blockLdV(tcs_ctx *ctx);               /* module_solve_momentum.f90:1278 */
int tcs_momentum_blockLdU(tcs_ctx *ctx);               /* module_solve_momentum.f90:1362 */
int tcs_momentum_pseudoupdateUVW(tcs_ctx *ctx);        /* module_solve_momentum.f90:178 */
int tcs_momentum_coeffi_clean(tcs_ctx *ctx);           /* module_solve_momentum.f90:213 (no work) */
int tcs_pressure_RHS(tcs_ctx *ctx);                    /* module_solve_pressure.f90:140 */
int tcs_pressure_Poisson_FFT2(tcs_ctx *ctx);           /* module_solve_pressure.f90:489 */
int tcs_pressure_Poisson_FFT1(tcs_ctx *ctx);           /* module_solve_pressure.f90:238 (transpose scheme 1: on one
                                                          GPU the same arithmetic and kernels as FFT2) */
int tcs_pressure_Projection(tcs_ctx *ctx);             /* module_solve_pressure.f90:756 */
int tcs_post_div(tcs_ctx *ctx, double *maxDivU);       /* module_post.f90:100 (also computes CFL, Nu, KE) */
int tcs_post_cfl(tcs_ctx *ctx, double *CFL, double *dt); /* module_post.f90:168 */

/* Whole steps (main.f90:129-223) replayed from a CUDA graph; stops early on
 * blow-up.  *done receives the number of completed steps. */
int tcs_step(tcs_ctx *ctx, int nsteps, int *done);
int tcs_get_scalars(tcs_ctx *ctx, double *out);        /* TCS_S_COUNT doubles */
/* On-device checkpoint of the step state (T, U, V, W, P, dPhat, dP0, scalars) and
 * its restore: the continue-file write/read of module_post.f90:1264-1454 without
 * leaving the device (and, unlike those files, including dPhat and dP0). */
int tcs_snapshot(tcs_ctx *ctx);
int tcs_restore(tcs_ctx *ctx);
/* Per-step series recorded by tcs_step: 7 doubles per step
 * (dt used, time, max divergence, CFL, Nu bottom, Nu top, kinetic energy). */
int tcs_get_history(tcs_ctx *ctx, int first, int count, double *out);

/* ---- PaScaL_TDMA many-systems interface (pascal_tdma.f90) ------------- */
/* pascal_tdma.f90:185 PaScaL_TDMA_plan_many_create(plan, n_sys, myrank, nprocs, mpi_world).
 * Only nprocs == 1 exists on one GPU; other values return TCS_ERR_UNSUPPORTED. */
int tcs_tdma_plan_many_create(tcs_tdma_plan **plan, int n_sys, int myrank, int nprocs);
/* pascal_tdma.f90:272 PaScaL_TDMA_plan_many_destroy(plan, nprocs) */
int tcs_tdma_plan_many_destroy(tcs_tdma_plan *plan);
/* pascal_tdma.f90:487 PaScaL_TDMA_many_solve(plan, A, B, C, D, n_sys, n_row): A,B,C,D are
 * (n_sys, n_row), system index fastest, host or device pointers; D := solution,
 * A and C are clobbered. */
int tcs_tdma_many_solve(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_sys, int n_row);
/* pascal_tdma.f90:715 PaScaL_TDMA_many_solve_cycle(plan, A, B, C, D, n_sys, n_row) */
int tcs_tdma_many_solve_cycle(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_sys, int n_row);
/* PaScaL_TDMA_plan_single_create/destroy, _single_solve(_cycle) (pascal_tdma.f90:139-175, 301-475) and
 * _many_solve(_cycle)_nonblocking (:590-703, 818-930): on one rank the same kernel as the many solve */
int tcs_tdma_plan_single_create(tcs_tdma_plan **plan, int myrank, int nprocs, int gather_rank);
int tcs_tdma_plan_single_destroy(tcs_tdma_plan *plan);
int tcs_tdma_single_solve(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_row);
int tcs_tdma_single_solve_cycle(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_row);
int tcs_tdma_many_solve_nonblocking(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_sys, int n_row);
int tcs_tdma_many_solve_cycle_nonblocking(tcs_tdma_plan *plan, double *A, double *B, double *C, double *D, int n_sys, int n_row);

/* No counterpart in the reference.  The PaScaL_TDMA many-systems solve
 * (cyclic != 0: the _cycle form) for callers that cannot allocate device
 * memory when they solve: host arrays A, B, C, D (n_sys, n_row) are staged
 * through a fixed device array compiled into the library, with no plan, no
 * cudaMalloc and no cudaFree.  n_sys * n_row must not exceed
 * TCS_TDMA_NOALLOC_MAX_ELEMS (TCS_ERR_UNSUPPORTED otherwise).  The array costs
 * 4 * TCS_TDMA_NOALLOC_MAX_ELEMS doubles (8 MiB) on every GPU that loads the
 * library, for the life of the process.  The first call on a device looks up
 * the array's address, and so does the first call after that device's
 * context was reset (cudaDeviceReset); make those calls before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race.
 * Blocking; runs on the legacy default stream of the current device. */
#define TCS_TDMA_NOALLOC_MAX_ELEMS (1 << 18)
int tcs_tdma_many_solve_noalloc(double *A, double *B, double *C, double *D, int n_sys, int n_row, int cyclic);

/* ---- measurement --------------------------------------------------------- */
int tcs_kernel_count(void);
/* Restart files and planes (module_post.f90): the continue files of
 * :1264-1454 (cont_time.bin = time, dt; cont_U/V/W/P/THETA.bin = the n1m*n2m*n3m
 * interior, i fastest, FP64; the reader also takes cont_T.bin for T when
 * cont_THETA.bin is absent) written and read by k-slabs straight from the
 * device, plus cont_dPhat.bin and cont_dP0.bin so that a resumed run continues
 * bit for bit (*with_pressure_history = 0 when those two are absent).  After a
 * read the periodic ghosts are refreshed before the next stage.
 * tcs_extract_plane copies one padded plane (axis 1: i = index over (j,k),
 * 2: j = index over (i,k), 3: k = index over (i,j); first index fastest) of
 * nfields fields into out, field after field: the instant-field planes of
 * :270-361 without downloading whole fields. */
int tcs_write_continue(tcs_ctx *ctx, const char *dir);
int tcs_read_continue(tcs_ctx *ctx, const char *dir, int *with_pressure_history);
int tcs_extract_plane(tcs_ctx *ctx, int axis, int index, int nfields, const int *fields, double *out);

/* Ensembles (no counterpart in the reference, which runs one case per MPI job):
 * independent cases on one device advanced together.  Every tcs_ensemble_step
 * replays one CUDA graph per step, in one of two forms:
 *   batched (1): each line sweep (thermal, solvedU/V/W, the modal Poisson
 *     solves) is ONE launch over all cases (up to a parameter block's worth of
 *     cases per launch), a persistent grid whose blocks pull (case, block)
 *     work items; the kernels between the sweeps run as one branch per case;
 *   branch per case (0): every case's whole step is its own graph branch.
 * Both give results bit-identical to stepping each case alone.  The default,
 * auto (-1), runs the first 8 steps (real steps) 4 in each form, times the
 * last 2 of each and keeps the faster form; tcs_ensemble_form reports the
 * form in use (-1 while still measuring) and the measured ms per step of each.
 * Cases keep their own state and entry points; tcs_ensemble_destroy does not
 * destroy them.  Probes must be off. */
typedef struct tcs_ensemble tcs_ensemble;
int tcs_ensemble_create(tcs_ctx *const *cases, int n, tcs_ensemble **out);
int tcs_ensemble_destroy(tcs_ensemble *ens);
int tcs_ensemble_step(tcs_ensemble *ens, int nsteps, int *nblown);   /* *nblown: cases that have blown up */
int tcs_ensemble_size(const tcs_ensemble *ens);
int tcs_ensemble_set_batched(tcs_ensemble *ens, int mode);             /* 1, 0 or -1 (auto, the default) */
int tcs_ensemble_form(const tcs_ensemble *ens, int *form, float *ms_branches, float *ms_batched);

unsigned long long tcs_launch_count(void);           /* kernels this library has launched so far */
/* The device's FP64 FMA throughput in TFLOP/s, measured (no counterpart in the
 * reference): the denominator of the line kernels' FP64-pipe roofline. */
int tcs_measure_fp64_peak(int device, double *tflops);
/* The largest error, in ulps of the correctly rounded 1/b, of the line solver's
 * reciprocal (FP64, or FP32 when fp32 != 0) over n values b = +-10^x, x in
 * [-6, 6] (no counterpart in the reference: a check of this library's
 * arithmetic). */
int tcs_check_reciprocal(int n, int fp32, double *max_ulp);
const char *tcs_kernel_name(int kernel_id);
/* Record a CUDA event pair around every launch of the kernels in mask (bit =
 * kernel id) on the launching stream; tcs_probe_read returns their summed
 * device time.  Probed steps run without the CUDA graph. */
int tcs_probe_enable(tcs_ctx *ctx, uint64_t mask);
int tcs_probe_read(tcs_ctx *ctx, int kernel_id, double *total_ms, int *launches);
int tcs_probe_reset(tcs_ctx *ctx);
/* The reference's stage timers (main.f90:55-72, timer.f90): the timer (1..18)
 * whose work a kernel does, 0 for kernels outside the time loop, -1 for a bad
 * id; and a timer's label as the reference prints it (NULL outside 1..18).
 * Summing probed kernel times per timer gives the reference's stage split. */
int tcs_timer_of_kernel(int kernel_id);
const char *tcs_timer_name(int timer);
/* Bounds-check build (no reference counterpart; the reference's debug builds
 * use the compiler's array checks, Makefile.inc:6-11): libtcs_bc.so, compiled
 * with -DTCS_BOUNDS_CHECK, checks every field, table, spectrum and
 * shared-memory row index the kernels form; an index out of range is counted
 * and its access redirected to a valid cell, never made.  tcs_bounds_checked
 * says whether the loaded library has the checks; tcs_bounds_violations
 * returns the case's count so far (always 0 in the normal build). */
int tcs_bounds_checked(void);
int tcs_bounds_violations(tcs_ctx *ctx, double *count);
int tcs_set_use_graph(tcs_ctx *ctx, int on);
/* launch-shape knobs (powers of two): lines per thread block of the strided
 * (y, z), contiguous (x) and modal line solvers and of the x and z FFTs, and
 * the most lanes (partitions) a tridiagonal line is split over.  A line-solver
 * value is an upper bound: each launch runs the largest power of two up to it
 * whose blocks fit the SM's shared memory at the family's blocks per SM; a
 * value no single block could hold is refused (TCS_ERR_ARG).
 * TCS_TUNE_LONG_LINES picks where long strided lines run as one block per SM
 * (the same warps, lines fitted to 132 KiB of shared memory so that L1 keeps
 * 124 KiB) when the usual blocks would leave under 60 KiB of L1 or halve
 * their lines: 1 never, 2 the z sweeps (default), 4 the z and y sweeps.
 * TCS_TUNE_Y_SOLVER picks the tridiagonal solver of the non-cyclic strided
 * lines: 1 the partitioned solver that every sweep uses (default: modified
 * Thomas per lane with a parallel reduced-system solve, pascal_tdma.f90:
 * 487-578; in the FP32-mixed form FP32 elimination with one FP64-residual
 * refinement pass); 2 the plain Thomas elimination with one line per thread
 * (tdmas.f90:27-50) in FP64 for the y sweeps (rows built in the field type);
 * 4 the same for the modal pressure solves too.  2 and 4 keep c' and d' in a
 * scratch buffer that setting the knob allocates ((1 + right-hand sides) x
 * rows x lines doubles: 2.1 GB for the y sweeps and 2.4 GB for the modal
 * solves at 512^3) and setting 1 frees.  Measured on B200: the one-line form
 * is faster for the y sweeps at 512^3 and slower at 256^3, where 65536 lines
 * leave the SMs short of threads; for the modal solves it is slower at both
 * sizes (its scratch traffic is 1.5x the spectrum's).
 * TCS_TUNE_IFFT_LINES_X: lines per block of the inverse x transform
 * (TCS_TUNE_FFT_LINES_X sets those of the pressure right-hand side and its
 * forward x transform).
 * TCS_TUNE_MIXED_ROWS (FP32-mixed form; no effect in the FP64 form): 1 the x
 * and z sweeps eliminate their FP32 rows in FP32 with one FP64-residual
 * refinement pass (default); 2 the x sweeps eliminate their FP32-built rows
 * in FP64 instead (no refinement pass; the solution is rounded once to FP32);
 * 4 the x and z sweeps; 8 the same with the z sweeps at three blocks per SM
 * (shared-memory elimination; faster at 256^3, slower at 512^3).
 * TCS_TUNE_Z_STAGING (FP64 form): 1 the z sweep of solvedW reads its stencil
 * inputs from global memory (default); 2 it stages them into shared memory with
 * tensor-memory-accelerator (TMA) box copies one pass of 64 k-planes ahead
 * (same arithmetic, same results; refused, TCS_ERR_ARG, unless the form is
 * FP64, N3 a multiple of 64 and N1 even). */
enum { TCS_TUNE_TL_STRIDED = 0, TCS_TUNE_TL_CONTIG, TCS_TUNE_TL_MODAL, TCS_TUNE_FFT_LINES_X, TCS_TUNE_FFT_LINES_Z,
       TCS_TUNE_LANES, TCS_TUNE_LONG_LINES, TCS_TUNE_Y_SOLVER, TCS_TUNE_IFFT_LINES_X, TCS_TUNE_MIXED_ROWS,
       TCS_TUNE_Z_STAGING, TCS_TUNE_COUNT };
int tcs_set_tuning(tcs_ctx *ctx, int knob, int value);
int tcs_get_tuning(tcs_ctx *ctx, int knob, int *value);
/* Autotuner (no reference counterpart): coordinate descent over every knob,
 * each candidate timed with CUDA events over trial_steps steps replayed from
 * the same state, which is restored afterwards (through tcs_snapshot, whose
 * earlier snapshot it replaces).  The winner is cached per (n1m, n2m, n3m,
 * precision) for the process and appended to cache_path when given (NULL: no
 * file); a cached shape is applied without timing and sets *from_cache. */
int tcs_autotune(tcs_ctx *ctx, int trial_steps, const char *cache_path, int *from_cache);
const char *tcs_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
