// tcs_tdma.cu -- the PaScaL_TDMA many-systems interface on one GPU:
// PaScaL_TDMA_many_solve and PaScaL_TDMA_many_solve_cycle
// (pascal_tdma.f90:487-578, 715-806) for one rank, with the reduced 2-row
// systems of tdma_many / tdma_cycl_many (tdmas.f90:113-146, 159-212).
//
// Arrays are the reference's (n_sys, n_row) with the system index fastest,
// so one thread per system reads and writes fully coalesced rows.  The
// arithmetic is the reference's, operation for operation, with explicit
// round-to-nearest intrinsics so that no multiply-add is fused: the results
// are bit-identical to a strict IEEE evaluation of the Fortran expressions
// (including the one-rank cyclic closure, where e(2) = -a(2) is overwritten by
// e(n2) = -c(2)).  D receives the solution; A and C are clobbered as in the
// reference.
#include "tcs_kernels.h"
#include "tcs.h"

#include <mutex>

namespace tcs {

#define MUL(a, b) __dmul_rn((a), (b))
#define SUB(a, b) __dsub_rn((a), (b))
#define ADD(a, b) __dadd_rn((a), (b))
#define DIV(a, b) __ddiv_rn((a), (b))

__global__ void tdma_many_kernel(double *__restrict__ A, const double *__restrict__ B, double *__restrict__ C,
                                 double *__restrict__ D, int n_sys, int n_row, int cyclic)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sys) return;
    const size_t s = (size_t)n_sys;
#define a(j) A[(size_t)i + s * (size_t)(j)]
#define b(j) B[(size_t)i + s * (size_t)(j)]
#define c(j) C[(size_t)i + s * (size_t)(j)]
#define d(j) D[(size_t)i + s * (size_t)(j)]
    double r;
    a(0) = DIV(a(0), b(0)); d(0) = DIV(d(0), b(0)); c(0) = DIV(c(0), b(0));
    a(1) = DIV(a(1), b(1)); d(1) = DIV(d(1), b(1)); c(1) = DIV(c(1), b(1));
    double am1 = a(1), cm1 = c(1), dm1 = d(1);
    for (int j = 2; j < n_row; j++) {
        const double aj = a(j);
        r = DIV(1.0, SUB(b(j), MUL(aj, cm1)));
        dm1 = MUL(r, SUB(d(j), MUL(aj, dm1))); d(j) = dm1;
        cm1 = MUL(r, c(j)); c(j) = cm1;
        am1 = MUL(MUL(-r, aj), am1); a(j) = am1;
    }
    if (n_row >= 3) {
        double ap1 = a(n_row - 2), cp1 = c(n_row - 2), dp1 = d(n_row - 2);
        for (int j = n_row - 3; j >= 1; j--) {
            const double cj = c(j);
            dp1 = SUB(d(j), MUL(cj, dp1)); d(j) = dp1;
            ap1 = SUB(a(j), MUL(cj, ap1)); a(j) = ap1;
            cp1 = MUL(-cj, cp1); c(j) = cp1;
        }
    }
    r = DIV(1.0, SUB(1.0, MUL(a(1), c(0))));
    d(0) = MUL(r, SUB(d(0), MUL(c(0), d(1))));
    a(0) = MUL(r, a(0));
    c(0) = MUL(MUL(-r, c(0)), c(1));
    const double A1 = a(0), C1 = c(0), D1 = d(0);
    const double A2 = a(n_row - 1), C2 = c(n_row - 1), D2 = d(n_row - 1);
    double x1, x2;
    if (cyclic) {
        const double e2 = -C2;
        x1 = DIV(SUB(SUB(D1, MUL(A1, D2)), MUL(C1, D2)), ADD(ADD(1.0, MUL(A1, e2)), MUL(C1, e2)));
        x2 = ADD(D2, MUL(x1, e2));
    } else {
        r = DIV(1.0, SUB(1.0, MUL(A2, C1)));
        x2 = MUL(r, SUB(D2, MUL(A2, D1)));
        x1 = SUB(D1, MUL(C1, x2));
    }
    d(0) = x1;
    d(n_row - 1) = x2;
    for (int j = 1; j < n_row - 1; j++) d(j) = SUB(SUB(d(j), MUL(a(j), x1)), MUL(c(j), x2));
#undef a
#undef b
#undef c
#undef d
}

#undef MUL
#undef SUB
#undef ADD
#undef DIV

void launch_tdma_many(double *A, const double *B, double *C, double *D, int n_sys, int n_row, int cyclic, cudaStream_t s)
{
    tdma_many_kernel<<<(n_sys + 127) / 128, 128, 0, s>>>(A, B, C, D, n_sys, n_row, cyclic);
    record_launch_error("tdma_many");
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the many-systems solve.
//
// Some callers cannot allocate device memory at the point where they solve:
// code that runs while a memory budget forbids further cudaMalloc after
// start-up (a solver embedded in a host application that owns the device
// memory pool), callers on a path where a cudaMalloc/cudaFree would
// synchronise the device and stall other work, and Fortran drivers that only
// hand over host arrays and must not create per-call plans.  They stage their
// systems through this file-scope device array instead.  It is statically
// sized, so every GPU that loads the library holds TCS_TDMA_NOALLOC_MAX_ELEMS
// x 4 doubles (8 MiB) until the process exits.  All calls share it and it
// keeps the last call's contents; calls that overlap on the GPU (other host
// threads, other streams) race on it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_tdma_noalloc[4 * TCS_TDMA_NOALLOC_MAX_ELEMS];

// Host code needs the array's device address (the symbol's name is only a
// host-side stand-in).  It is looked up once per device context: the slot
// remembers the unique id of the context it was taken in, so after a
// cudaDeviceReset (a new primary context, in which the library's module is
// loaded again) the next call looks it up afresh instead of using the dead
// address.  The context id comes from the driver (cuCtxGetCurrent, cuCtxGetId)
// through the runtime's entry-point query; without it every call looks up.
struct NoallocSlot { double *ptr; unsigned long long ctx_id; bool have_id; };
static std::mutex g_noalloc_mu;
static NoallocSlot g_noalloc_slot[64] = {};

typedef int (*PfnCtxGetCurrent)(void **ctx);
typedef int (*PfnCtxGetId)(void *ctx, unsigned long long *id);
static PfnCtxGetCurrent g_ctx_get_current = nullptr;
static PfnCtxGetId g_ctx_get_id = nullptr;
static std::once_flag g_ctx_fn_once;

static bool current_ctx_id(unsigned long long *id)
{
    std::call_once(g_ctx_fn_once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = (PfnCtxGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = (PfnCtxGetId)f;
        cudaGetLastError();
    });
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    void *ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0 || !ctx) return false;
    return g_ctx_get_id(ctx, id) == 0;
}

// The array's address on the current device (set-up on a device's first call,
// and again after its context was reset).
static int noalloc_base(int dev, double **out)
{
    unsigned long long id = 0;
    bool have = current_ctx_id(&id);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocSlot &sl = g_noalloc_slot[dev];
    if (!sl.ptr || !have || !sl.have_id || id != sl.ctx_id) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_tdma_noalloc);
        if (e != cudaSuccess) return set_error(TCS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        have = current_ctx_id(&id);        // the lookup makes the primary context current
        sl.ptr = (double *)p;
        sl.ctx_id = id;
        sl.have_id = have;
    }
    *out = sl.ptr;
    return TCS_OK;
}

} // namespace tcs

extern "C" int tcs_tdma_many_solve_noalloc(double *A, double *B, double *C, double *D, int n_sys, int n_row, int cyclic)
{
    using namespace tcs;
    if (!A || !B || !C || !D) return set_error(TCS_ERR_ARG, "null argument");
    if (n_sys < 1 || n_row < 2) return set_error(TCS_ERR_ARG, "n_sys >= 1 and n_row >= 2 required");
    const size_t n = (size_t)n_sys * (size_t)n_row;
    if (n > (size_t)TCS_TDMA_NOALLOC_MAX_ELEMS)
        return set_error(TCS_ERR_UNSUPPORTED, "n_sys * n_row exceeds TCS_TDMA_NOALLOC_MAX_ELEMS");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(TCS_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return set_error(TCS_ERR_UNSUPPORTED, "device ordinal >= 64");
    double *base = nullptr;
    const int r = noalloc_base(dev, &base);
    if (r) return r;
    double *dA = base, *dB = base + n, *dC = base + 2 * n, *dD = base + 3 * n;
    const size_t bytes = n * sizeof(double);
    // Every element the kernel reads is copied in first, so nothing needs clearing.
    if ((e = cudaMemcpy(dA, A, bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dB, B, bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dC, C, bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dD, D, bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
        return set_error(TCS_ERR_CUDA, std::string("cudaMemcpy to the static scratch: ") + cudaGetErrorString(e));
    tdma_many_kernel<<<(n_sys + 127) / 128, 128, 0, 0>>>(dA, dB, dC, dD, n_sys, n_row, cyclic ? 1 : 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_error(TCS_ERR_CUDA, std::string("tdma_many launch: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpy(A, dA, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(C, dC, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(D, dD, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return set_error(TCS_ERR_CUDA, std::string("cudaMemcpy from the static scratch: ") + cudaGetErrorString(e));
    return TCS_OK;
}
