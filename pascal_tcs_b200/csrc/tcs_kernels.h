// tcs_kernels.h -- host-side view of one case (Ctx), kernel identifiers and
// the launch helpers shared by the stage files.
#pragma once

#include "tcs_fields.cuh"

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

namespace tcs {

// Every kernel the time step launches, in launch order.
enum KernelId : int {
    K_THERMAL_Z = 0, K_THERMAL_X, K_THERMAL_Y, K_MOM_COEFFI,
    K_DU_Z, K_DU_X, K_DU_Y, K_DV_Z, K_DV_X, K_DV_Y, K_DW_Z, K_DW_X, K_DW_Y,
    K_BLOCKLDV, K_BLOCKLDU, K_PSEUDO, K_PRHS_FFTX, K_FFTZ_FWD, K_MODAL, K_MEAN,
    K_FFTZ_INV, K_IFFTX, K_DP_WALL, K_PROJECT, K_P_WALL, K_POST, K_FINAL, K_TDMA_API,
    K_COUNT
};

const char *kernel_name(int kid);

struct FFTPlan {
    int n, npass;
    int radix[24];
};

struct ProbeState;   // CUDA-event probes (tcs_capi.cu)

struct Ctx {
    Grid g;
    Fields f;
    int tl_strided, tl_contig, tl_modal;
    int fft_lines_x, fft_lines_z;
    FFTPlan fp1, fp3;
    int h1p;
    double wall_ab, wall_bb, wall_at, wall_bt;   // Pbc_a, Pbc_b of the two walls
    ProbeState *probe;
};

LinePlan make_line_plan(int n, bool cyclic, int TL);
bool make_fft_plan(int n, FFTPlan &fp);
void probe_begin(const Ctx &cx, int kid, cudaStream_t s);
void probe_end(const Ctx &cx, int kid, cudaStream_t s);
int record_launch_error(const char *what);
int set_error(int code, const std::string &msg);

template <class Prob>
inline void launch_lines(const Prob &p, const LinePlan &lp, dim3 grid, cudaStream_t s, int kid, const Ctx &cx)
{
    const size_t smem = (size_t)(2 + Prob::NRHS) * lp.TL * lp.LS * sizeof(double) + (size_t)lp.n * sizeof(int);
    static size_t configured = 0;
    if (smem > configured) {
        cudaFuncSetAttribute(line_solve_kernel<Prob>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = smem;
    }
    probe_begin(cx, kid, s);
    line_solve_kernel<Prob><<<grid, 256, smem, s>>>(p, lp);
    probe_end(cx, kid, s);
    record_launch_error(kernel_name(kid));
}

// Stage launchers (one per reference routine or fused group).
void launch_thermal(const Ctx &cx, cudaStream_t s);
void launch_momentum_coeffi(const Ctx &cx, cudaStream_t s);
void launch_solve_du(const Ctx &cx, cudaStream_t s);
void launch_solve_dv(const Ctx &cx, cudaStream_t s);
void launch_solve_dw(const Ctx &cx, cudaStream_t s);
void launch_blockld_v(const Ctx &cx, cudaStream_t s);
void launch_blockld_u(const Ctx &cx, cudaStream_t s);
void launch_pseudo_update(const Ctx &cx, cudaStream_t s);           // standalone (Un = U + dU, ...)
void launch_pseudo_prhs_fftx(const Ctx &cx, cudaStream_t s, bool with_pseudo);
void launch_poisson_rest(const Ctx &cx, cudaStream_t s);
void launch_projection(const Ctx &cx, cudaStream_t s);
void launch_post(const Ctx &cx, cudaStream_t s, int record_hist);
void launch_ghost(const Ctx &cx, double *a, cudaStream_t s);
void launch_set_fields_walls(const Ctx &cx, cudaStream_t s);

} // namespace tcs
