// tcs_capi.cu -- host runtime and C ABI of libtcs (declared in include/tcs.h).
//
// Owns one case: the host-side mesh (mpi_subdomain_mesh), the device fields,
// the stage sequence of main.f90:129-223, CUDA-graph replay of whole steps,
// CUDA-event probes and the PaScaL_TDMA many-systems plans.
#include "tcs_kernels.h"
#include "tcs.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace tcs {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local int g_launch_err = 0;
static std::atomic<unsigned long long> g_launches{0};   // kernels launched by this library (graph replays included)

static int set_err(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int record_launch_error(const char *what)
{
    g_launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_launch_err = 1;
        g_err = std::string("launch of ") + what + " failed: " + cudaGetErrorString(e);
    }
    return e == cudaSuccess ? 0 : 1;
}

int set_error(int code, const std::string &msg) { return set_err(code, msg); }

static int take_launch_error()
{
    const int e = g_launch_err;
    g_launch_err = 0;
    return e ? TCS_ERR_CUDA : TCS_OK;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_err(TCS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

static const char *const k_names[K_COUNT] = {
    "thermal_z", "thermal_x", "thermal_y", "momentum_coeffi",
    "du_z", "du_x", "du_y", "dv_z", "dv_x", "dv_y", "dw_z", "dw_x", "dw_y",
    "blockld_v", "blockld_u", "pseudo_update", "prhs_fftx", "fftz_fwd", "modal_tdma", "mean",
    "fftz_inv", "ifftx", "dp_wall", "projection", "p_wall", "post", "finalize", "tdma_api"};

const char *kernel_name(int kid) { return (kid >= 0 && kid < K_COUNT) ? k_names[kid] : "?"; }

// The reference's stage timers (main.f90:55-72: timer_str(1..18), stamped
// after every call of the time loop, :129-221) and the timer each kernel's
// work falls under.  The property evaluation of mpi_thermal_coeffi (1) is
// fused into the thermal sweeps (2), the pseudo-update (9) into the pressure
// right-hand side (10), the ghost-cell updates (13) into the stores of the
// producing kernels, and mpi_Post_CFL (16) into the diagnostics kernel (15),
// so those timers count no kernels; 0 marks kernels outside the time loop.
static const char *const k_timer_names[19] = {
    "", "[Main] Thermal coeff", "[Main] Thermal solve", "[Main] Momentum coeff", "[Main] Momentum solvedU",
    "[Main] Momentum solvedV", "[Main] Momentum solvedW", "[Main] Momentum blockLdV", "[Main] Momentum blockLdU",
    "[Main] Momentum updatePseudoUVW", "[Main] Pressure RHS", "[Main] Pressure PoissonSolve",
    "[Main] Pressure projection", "[Main] Update GhostCell", "[Main] Clean coeff", "[Main] Post div",
    "[Main] Post CFL", "[Main] Misc operation", "[Main] File write"};
static const int k_timer_of[K_COUNT] = {
    2, 2, 2, 3,                       // thermal_z, thermal_x, thermal_y, momentum_coeffi
    4, 4, 4, 5, 5, 5, 6, 6, 6,        // du_*, dv_*, dw_*
    7, 8, 9, 10, 11, 11, 11,          // blockld_v, blockld_u, pseudo_update, prhs_fftx, fftz_fwd, modal_tdma, mean
    11, 11, 11, 12, 12, 15, 15, 0};   // fftz_inv, ifftx, dp_wall, projection, p_wall, post, finalize, tdma_api
static_assert(sizeof(k_timer_of) / sizeof(int) == K_COUNT, "one timer per kernel");

// ---------------------------------------------------------------------------
// probes: CUDA event pairs on the launching stream
// ---------------------------------------------------------------------------
struct ProbeState {
    uint64_t mask = 0;
    std::vector<cudaEvent_t> pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> rec[K_COUNT];
    cudaEvent_t pending[K_COUNT] = {};
    cudaEvent_t take()
    {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
};

void probe_begin(const Shapes &cx, int kid, cudaStream_t s)
{
    ProbeState *p = cx.probe;
    if (!p || !(p->mask & (1ull << kid))) return;
    p->pending[kid] = p->take();
    cudaEventRecord(p->pending[kid], s);
}

void probe_end(const Shapes &cx, int kid, cudaStream_t s)
{
    ProbeState *p = cx.probe;
    if (!p || !(p->mask & (1ull << kid)) || !p->pending[kid]) return;
    cudaEvent_t e = p->take();
    cudaEventRecord(e, s);
    p->rec[kid].push_back({p->pending[kid], e});
    p->pending[kid] = nullptr;
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------
LinePlan make_line_plan(int n, bool cyclic, int TL, int pmax)
{
    LinePlan lp;
    int P;
    if (pmax > 32) pmax = 32;
    if (cyclic) { P = 1; while (P * 2 <= pmax && n / (P * 2) >= 2) P *= 2; }
    else { P = n / 2; if (P > pmax) P = pmax; if (P < 1) P = 1; }
    lp.n = n; lp.P = P; lp.m0 = n / P; lp.rem = n % P;
    const int mmax = lp.m0 + (lp.rem > 0 ? 1 : 0);
    lp.PS = mmax | 1;
    lp.LS = (P * lp.PS) | 1;
    lp.TL = TL;
    lp.cyclic = cyclic ? 1 : 0;
    return lp;
}

// Shared-memory bytes per row of a line-solver block: A, C, D[nrhs] of the
// row type, plus the kept rows A0, B0, C0, D0[nrhs] when FP32 rows are refined.
static size_t row_bytes(int nrhs, bool fp32_refined)
{
    return fp32_refined ? (size_t)(5 + 2 * nrhs) * sizeof(float) : (size_t)(2 + nrhs) * sizeof(double);
}

static int choose_tl(int n, bool cyclic, size_t rowb, int want)
{
    LinePlan lp = make_line_plan(n, cyclic, want);
    int tl = want;
    while (tl > 2 && rowb * tl * lp.LS + (size_t)n * sizeof(int) > 112 * 1024) tl /= 2;
    return tl;
}

bool make_fft_plan(int n, FFTPlan &fp, int maxr)
{
    fp.n = n; fp.npass = 0;
    int m = n;
    // a power of 4 that is no power of 8 takes radix 4 throughout (one radix in
    // every pass allows the z transform's one-buffer form), else radix 8 first
    int p8 = n;
    while (p8 % 8 == 0) p8 /= 8;
    int p4 = n;
    while (p4 % 4 == 0) p4 /= 4;
    const bool only4 = p8 != 1 && p4 == 1;
    while (maxr >= 8 && !only4 && m % 8 == 0 && fp.npass < 24) { fp.radix[fp.npass++] = 8; m /= 8; }
    while (m % 4 == 0 && fp.npass < 24) { fp.radix[fp.npass++] = 4; m /= 4; }
    while (m % 2 == 0 && fp.npass < 24) { fp.radix[fp.npass++] = 2; m /= 2; }
    while (m % 3 == 0 && fp.npass < 24) { fp.radix[fp.npass++] = 3; m /= 3; }
    while (m % 5 == 0 && fp.npass < 24) { fp.radix[fp.npass++] = 5; m /= 5; }
    int Ns = 1;
    for (int p = 0; p < fp.npass; p++) {
        fp.dnb[p] = make_fastdiv((unsigned)(n / fp.radix[p]));
        fp.dns[p] = make_fastdiv((unsigned)Ns);
        Ns *= fp.radix[p];
    }
    fp.dn = make_fastdiv((unsigned)n);
    fp.dh = make_fastdiv((unsigned)(n / 2 + 1));
    return m == 1;
}

} // namespace tcs

using namespace tcs;

// ---------------------------------------------------------------------------
// the context
// ---------------------------------------------------------------------------
struct tcs_ctx {
    tcs_config cfg;
    bool fp32 = false;                   // TCS_PREC_FP32_MIXED
    // The grid, scalars, history and launch shapes live in cx in both forms;
    // the fields are allocated in the context of the active form only.
    Ctx<double> cx;
    Ctx<float> cf;
    double *stage = nullptr;             // FP64 staging copy of one field (FP32 form)
    double *io_dev = nullptr, *io_host = nullptr;   // file IO chunk: device staging and pinned host copy
    size_t io_cap = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<double> hm[9];           // x1, dx1, dmx1, x2, dx2, dmx2, x3, dx3, dmx3
    std::vector<void *> allocs;
    uint32_t ghost_ok = 0;               // bit per field id: periodic ghosts are current
    bool pending_pseudo = false;
    bool use_graph = true;
    struct GraphEntry { const void *T, *U, *dPhat; cudaGraphExec_t exec; unsigned long long kernels; };
    std::vector<GraphEntry> graphs;
    ProbeState probe;
    int partials = 0;
    void *snap[10] = {};                 // on-device copy of T, U, V, W, P, dPhat, dP0 (+ U, V, W low words)
    double snap_scal[S_NSCAL] = {};
    bool have_snap = false;
};

// Run fn on the context of the active form.
template <class Fn>
static auto on_ctx(tcs_ctx *c, Fn &&fn) -> decltype(fn(c->cx))
{
    if (c->fp32) return fn(c->cf);
    return fn(c->cx);
}

// The shapes are decided once on cx; the FP32 context runs with the same ones.
static void sync_shapes(tcs_ctx *c)
{
    static_cast<Shapes &>(c->cf) = static_cast<const Shapes &>(c->cx);
}

static size_t esize(const tcs_ctx *c) { return c->fp32 ? sizeof(float) : sizeof(double); }

namespace tcs {
int post_partial_count();
void launch_tdma_many(double *A, const double *B, double *C, double *D, int n_sys, int n_row, int cyclic, cudaStream_t s);
} // namespace tcs

static void mesh_periodic(int uniform, double L, double gamma, int nm, std::vector<double> &x, std::vector<double> &dx, std::vector<double> &dmx)
{
    // mpi_subdomain_mesh for a periodic direction on one rank (module_mpi_subdomain.f90:167-209)
    const int nsub = nm + 1;
    x.assign(nsub + 1, 0.0); dx.assign(nsub + 1, 0.0); dmx.assign(nsub + 1, 0.0);
    for (int i = 0; i <= nsub; i++) {
        if (uniform == 1) x[i] = (double)(i - 1) * L / (double)nm + 0.0;
        else x[i] = L * 0.5 * (1.0 + std::tanh(0.5 * gamma * (2.0 * (double)(i - 1) / (double)nm - 1.0)) / std::tanh(gamma * 0.5)) + 0.0;
    }
    for (int i = 1; i <= nsub - 1; i++) dx[i] = x[i + 1] - x[i];
    dx[0] = dx[nsub - 1]; dx[nsub] = dx[1];
    for (int i = 1; i <= nsub - 1; i++) dmx[i] = 0.5 * (dx[i - 1] + dx[i]);
    dmx[0] = dmx[nsub - 1]; dmx[nsub] = dmx[1];
}

static void mesh_wall(int uniform, double L, double gamma, int nm, std::vector<double> &x, std::vector<double> &dx, std::vector<double> &dmx)
{
    // the wall-bounded y direction (module_mpi_subdomain.f90:211-253)
    const int nsub = nm + 1;
    x.assign(nsub + 1, 0.0); dx.assign(nsub + 1, 0.0); dmx.assign(nsub + 1, 0.0);
    for (int j = 0; j <= nsub; j++) {
        if (uniform == 1) x[j] = (double)(j - 1) * L / (double)nm + 0.0;
        else x[j] = L * 0.5 * (1. + std::tanh(0.5 * gamma * (2. * (double)(j - 1) / (double)nm - 1.0)) / std::tanh(gamma * 0.5)) + 0.0;
    }
    x[0] = x[1];
    for (int j = 1; j <= nsub - 1; j++) dx[j] = x[j + 1] - x[j];
    dx[0] = 0.0; dx[nsub] = 0.0;
    for (int j = 1; j <= nsub - 1; j++) dmx[j] = 0.5 * (dx[j - 1] + dx[j]);
    dmx[0] = 0.0;
    dmx[nsub] = 0.5 * (dx[nsub - 1] + dx[nsub]);
}

static void set_properties(const tcs_config &c, Phys &p)
{
    // module_global.f90:107-141
    p.Uup = p.Ubt = p.Vup = p.Vbt = p.Wup = p.Wbt = 0.0;
    p.Tup = -0.5; p.Tbt = 0.5;
    if (c.property_set == 1) {
        p.a10 = 0.9922e+3; p.a11 = -3.736e-4; p.a12 = -3.98e-6; p.a13 = 0.; p.a14 = 0.; p.a15 = 0.;
        p.b10 = 4.1690e+3; p.b11 = 0.084e-4; p.b12 = 4.60e-6; p.b13 = 0.; p.b14 = 0.; p.b15 = 0.;
        p.c10 = (double)0.6297f; p.c11 = 21.99e-4; p.c12 = -17.8e-6; p.c13 = 0.; p.c14 = 0.; p.c15 = 0.;
        p.d10 = 0.6690e-6; p.d11 = -175.9e-4; p.d12 = 295.8e-6; p.d13 = -460.e-8; p.d14 = 0.; p.d15 = 0.;
    } else if (c.property_set == 2) {
        p.a10 = 1.2477e+3; p.a11 = -4.789e-4; p.a12 = -0.3795e-6; p.a13 = 0.; p.a14 = 0.; p.a15 = 0.;
        p.b10 = 2.5108e+3; p.b11 = 22.511e-4; p.b12 = 0.; p.b13 = 0.; p.b14 = 0.; p.b15 = 0.;
        p.c10 = 2.9351e-3; p.c11 = 3.863e-4; p.c12 = 0.; p.c13 = 0.; p.c14 = 0.; p.c15 = 0.;
        p.d10 = 238.71e-6; p.d11 = -702.83e-4; p.d12 = 2393.1e-6; p.d13 = -6923.0e-8; p.d14 = 33131.3e-10; p.d15 = -71517.5e-12;
    } else {
        p.a10 = 1.0; p.a11 = 0.0; p.a12 = 0.0; p.a13 = 0.0; p.a14 = 0.; p.a15 = 0.;
        p.b10 = 1.0; p.b11 = 0.0; p.b12 = 0.0; p.b13 = 0.0; p.b14 = 0.; p.b15 = 0.;
        p.c10 = 1.0; p.c11 = 0.0; p.c12 = 0.0; p.c13 = 0.0; p.c14 = 0.; p.c15 = 0.;
        p.d10 = 1.0; p.d11 = 0.0; p.d12 = 0.0; p.d13 = 0.0; p.d14 = 0.; p.d15 = 0.;
    }
    p.a12pera11 = (p.a12 < 1.0e-14) ? 0.0 : p.a12 / p.a11;
    p.Rho0 = p.a10; p.Cp0 = p.b10; p.KPP0 = p.c10; p.Mu0 = p.a10 * p.d10;
    p.cK = p.c10 / p.KPP0;
    p.cRC = p.Rho0 * p.Cp0 / (p.a10 * p.b10);
    p.k2 = 2.0 * p.c12; p.k3 = 3.0 * p.c13; p.k4 = 4.0 * p.c14; p.k5 = 5.0 * p.c15;
    // numerator of d(invRhoCp)/dT (module_solve_thermal.f90:144-148) in powers of t
    p.n0 = p.a11 + p.b11;
    p.n1 = 2.0 * p.a11 * p.b11 + 2.0 * p.b12 + 2.0 * p.a12;
    p.n2 = 3.0 * p.a12 * p.b11 + 3.0 * p.a11 * p.b12 + 3.0 * (p.a13 + p.b13);
    p.n3 = 4.0 * p.a13 * p.b11 + 4.0 * p.a11 * p.b13 + 4.0 * p.a12 * p.b12;
    p.n4 = 5.0 * p.a13 * p.b12 + 5.0 * p.a12 * p.b13;
    p.n5 = 6.0 * p.a13 * p.b13;
    p.Cmu = std::sqrt(c.Pr / c.Ra); p.Cmt = 1.0; p.Ct = 1.0 / std::sqrt(c.Ra * c.Pr); p.Cmp = 1.0;
    p.DeltaT = c.DeltaT; p.MaxCFL = c.MaxCFL;
    p.L1 = c.H * c.aspect1; p.L2 = c.H; p.L3 = c.H * c.aspect3;
    const double t1 = p.L1 / (double)c.n1m, t2 = p.L2 / (double)c.n2m, t3 = p.L3 / (double)c.n3m;
    double mn = t1; if (t2 < mn) mn = t2; if (t3 < mn) mn = t3;
    p.dtMax = mn * 100;
}

static uint64_t splitmix64_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

template <class T>
static int dalloc(tcs_ctx *c, T **p, size_t n)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) ? n * sizeof(T) : 16);
    if (e != cudaSuccess) return set_err(TCS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->allocs.push_back(q);
    cudaMemsetAsync(q, 0, n * sizeof(T), c->stream);
    *p = (T *)q;
    return TCS_OK;
}

template <class T>
static int upload_vec(tcs_ctx *c, const std::vector<T> &v, const T **out)
{
    T *d;
    int r = dalloc(c, &d, v.size());
    if (r) return r;
    CK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    *out = d;
    return TCS_OK;
}

static void host_ghost(std::vector<double> &a, int N1, int N2, int N3)
{
    const size_t P1 = N1 + 2, P2 = N2 + 2;
    auto I = [&](int i, int j, int k) { return (size_t)i + P1 * ((size_t)j + P2 * (size_t)k); };
    for (int k = 0; k <= N3 + 1; k++)
        for (int j = 0; j <= N2 + 1; j++) { a[I(0, j, k)] = a[I(N1, j, k)]; a[I(N1 + 1, j, k)] = a[I(1, j, k)]; }
    for (int j = 0; j <= N2 + 1; j++)
        for (int i = 0; i <= N1 + 1; i++) { a[I(i, j, 0)] = a[I(i, j, N3)]; a[I(i, j, N3 + 1)] = a[I(i, j, 1)]; }
}

template <class R>
static R *field_ptr_t(FieldsT<R> &F, int f)
{
    switch (f) {
    case TCS_F_T: return F.T; case TCS_F_U: return F.U; case TCS_F_V: return F.V; case TCS_F_W: return F.W;
    case TCS_F_P: return F.P; case TCS_F_DPHAT: return F.dPhat; case TCS_F_DP0: return F.dP0;
    case TCS_F_DU: return F.dU; case TCS_F_DV: return F.dV; case TCS_F_DW: return F.dW; case TCS_F_DP: return F.dP;
    default: return nullptr;
    }
}

static void *field_ptr(tcs_ctx *c, int f)
{
    return on_ctx(c, [&](auto &x) -> void * { return field_ptr_t(x.f, f); });
}

template <class R> static void swap_T(Ctx<R> &x) { std::swap(x.f.T, x.f.Tn); }
template <class R> static void swap_UVW(Ctx<R> &x)
{
    std::swap(x.f.U, x.f.Un); std::swap(x.f.V, x.f.Vn); std::swap(x.f.W, x.f.Wn);
    std::swap(x.f.Ulo, x.f.Unlo); std::swap(x.f.Vlo, x.f.Vnlo); std::swap(x.f.Wlo, x.f.Wnlo);
}

// The low word of a velocity field (FP32 form), else null.
template <class R>
static R *lo_ptr_t(FieldsT<R> &F, int f)
{
    switch (f) {
    case TCS_F_U: return F.Ulo; case TCS_F_V: return F.Vlo; case TCS_F_W: return F.Wlo;
    default: return nullptr;
    }
}
template <class R> static void swap_phat(Ctx<R> &x) { std::swap(x.f.dPhat, x.f.dPhatn); std::swap(x.f.dP0, x.f.dP0n); }

static int flush_pending(tcs_ctx *c)
{
    if (!c->pending_pseudo) return TCS_OK;
    on_ctx(c, [&](auto &x) { launch_pseudo_update(x, c->stream); swap_UVW(x); });
    c->pending_pseudo = false;
    return take_launch_error();
}

extern "C" {

const char *tcs_last_error(void) { return g_err.c_str(); }
int tcs_kernel_count(void) { return K_COUNT; }
unsigned long long tcs_launch_count(void) { return g_launches; }
const char *tcs_kernel_name(int kid) { return kernel_name(kid); }
int tcs_bounds_checked(void)
{
#ifdef TCS_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

int tcs_bounds_violations(tcs_ctx *c, double *count)
{
    if (!c || !count) return set_err(TCS_ERR_ARG, "null argument");
    cudaSetDevice(c->cfg.device);
    CK(cudaMemcpyAsync(count, c->cx.g.scal + S_OOB, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

int tcs_timer_of_kernel(int kid) { return (kid >= 0 && kid < K_COUNT) ? k_timer_of[kid] : -1; }
const char *tcs_timer_name(int timer) { return (timer >= 1 && timer <= 18) ? k_timer_names[timer] : nullptr; }

int tcs_create(const tcs_config *cfg, tcs_ctx **out)
{
    if (!cfg || !out) return set_err(TCS_ERR_ARG, "null argument");
    *out = nullptr;
    if (cfg->n1m < 4 || cfg->n2m < 4 || cfg->n3m < 4) return set_err(TCS_ERR_ARG, "every n_m must be >= 4");
    if ((long long)(cfg->n1m + 2) * (cfg->n2m + 2) * (cfg->n3m + 2) > (1ll << 31))
        return set_err(TCS_ERR_UNSUPPORTED, "padded grid exceeds 2^31 cells");
    if (cfg->n1m > 4096 || cfg->n3m > 4096 || cfg->n2m > 4096) return set_err(TCS_ERR_UNSUPPORTED, "an axis exceeds 4096 cells");
    FFTPlan fp1, fp3, fp1u;
    // the x transforms share their kernels with the right-hand side and the
    // inverse scaling, which keep their registers for that work: radix <= 4
    // (a radix-8 butterfly took the right-hand side from 64 to 88 registers)
    if (!make_fft_plan(cfg->n1m, fp1, 4) || !make_fft_plan(cfg->n3m, fp3, 8) || !make_fft_plan(cfg->n1m, fp1u, 8))
        return set_err(TCS_ERR_UNSUPPORTED, "n1m and n3m must factor into 2, 3 and 5 (FFT radices)");
    if (cfg->precision != TCS_PREC_FP64 && cfg->precision != TCS_PREC_FP32_MIXED)
        return set_err(TCS_ERR_ARG, "precision must be TCS_PREC_FP64 or TCS_PREC_FP32_MIXED");
    CK(cudaSetDevice(cfg->device));
    tcs_ctx *c = new tcs_ctx();
    c->cfg = *cfg;
    c->fp32 = cfg->precision == TCS_PREC_FP32_MIXED;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return set_err(TCS_ERR_CUDA, "stream"); }
    c->own_stream = true;
    const int N1 = cfg->n1m, N2 = cfg->n2m, N3 = cfg->n3m;
    GridT<double> &g = c->cx.g;
    g.N1 = N1; g.N2 = N2; g.N3 = N3; g.P1 = N1 + 2; g.P2 = N2 + 2;
    g.NP = (long long)(N1 + 2) * (N2 + 2) * (N3 + 2);
    set_properties(*cfg, g.ph);
    g.phd = g.ph;
    g.kdeg2 = (g.ph.c13 == 0.0 && g.ph.c14 == 0.0 && g.ph.c15 == 0.0) ? 1 : 0;
    mesh_periodic(cfg->uniform1, g.ph.L1, cfg->gamma1, N1, c->hm[0], c->hm[1], c->hm[2]);
    mesh_wall(cfg->uniform2, g.ph.L2, cfg->gamma2, N2, c->hm[3], c->hm[4], c->hm[5]);
    mesh_periodic(cfg->uniform3, g.ph.L3, cfg->gamma3, N3, c->hm[6], c->hm[7], c->hm[8]);
    // fix dtMax with the reference formula on n - 1 = n_m (module_global.f90:161-165)
    int r = TCS_OK;
    MetricT<double> *ms[3] = {&g.m1, &g.m2, &g.m3};
    MetricT<float> *mf[3] = {&c->cf.g.m1, &c->cf.g.m2, &c->cf.g.m3};
    auto to_f = [](const std::vector<double> &v) { return std::vector<float>(v.begin(), v.end()); };
    for (int d = 0; d < 3 && !r; d++) {
        const std::vector<double> &dx = c->hm[3 * d + 1], &dmx = c->hm[3 * d + 2];
        std::vector<double> rdx(dx.size()), rdmx(dmx.size());
        for (size_t q = 0; q < dx.size(); q++) { rdx[q] = dx[q] != 0.0 ? 1.0 / dx[q] : 0.0; rdmx[q] = dmx[q] != 0.0 ? 1.0 / dmx[q] : 0.0; }
        r = r ? r : upload_vec(c, dx, &ms[d]->dx);
        r = r ? r : upload_vec(c, dmx, &ms[d]->dmx);
        r = r ? r : upload_vec(c, rdx, &ms[d]->rdx);
        r = r ? r : upload_vec(c, rdmx, &ms[d]->rdmx);
        if (c->fp32) {   // the same tables rounded once to FP32
            r = r ? r : upload_vec(c, to_f(dx), &mf[d]->dx);
            r = r ? r : upload_vec(c, to_f(dmx), &mf[d]->dmx);
            r = r ? r : upload_vec(c, to_f(rdx), &mf[d]->rdx);
            r = r ? r : upload_vec(c, to_f(rdmx), &mf[d]->rdmx);
        }
    }
    g.d1 = g.m1; g.d2 = g.m2; g.d3 = g.m3;
    const size_t NP = (size_t)g.NP;
    c->cx.h1p = N1 / 2 + 1;
    if (!r) r = dalloc(c, &g.scal, (size_t)S_NALLOC);
    c->partials = post_partial_count();
    if (!r) r = dalloc(c, &c->cx.f.part, (size_t)c->partials);
    c->cx.f.hist_cap = 100000;
    if (!r) r = dalloc(c, &c->cx.f.hist, (size_t)c->cx.f.hist_cap * 7);
    // the fields of the active form
    auto alloc_fields = [&](auto &x) {
        auto &F = x.f;
        using R = std::remove_pointer_t<decltype(F.T)>;
        R **fl[] = {&F.T, &F.U, &F.V, &F.W, &F.P, &F.dPhat, &F.dP0, &F.Tn, &F.Un, &F.Vn, &F.Wn, &F.dPhatn, &F.dP0n,
                    &F.dU, &F.dV, &F.dW, &F.dP, &F.scr};
        for (R **p : fl) if (!r) r = dalloc(c, p, NP);
        if (!r) r = dalloc(c, &F.Mu2, (size_t)(N2 + 2) * (N3 + 2));
        if (!r) r = dalloc(c, &F.iR2, (size_t)(N2 + 2) * (N3 + 2));
        if (HasLo<R>::on) {
            if (!r) r = dalloc(c, &F.iR2d, (size_t)(N2 + 2) * (N3 + 2));
        } else {
            F.iR2d = (double *)F.iR2;
        }
        if (!r) r = dalloc(c, &F.S, (size_t)c->cx.h1p * N2 * N3);
        if (HasLo<R>::on) {
            R **lo[] = {&F.Ulo, &F.Vlo, &F.Wlo, &F.Unlo, &F.Vnlo, &F.Wnlo};
            for (R **p : lo) if (!r) r = dalloc(c, p, NP);
        }
    };
    on_ctx(c, alloc_fields);
    if (c->fp32 && !r) r = dalloc(c, &c->stage, NP);
    if (r) { tcs_destroy(c); return r; }
    // the split form of the pressure right-hand side keeps it in a free FP64
    // array: scr (free between the momentum sweeps and the next step's thermal
    // sweeps) in the FP64 form, the host-transfer staging array in the FP32 form
    c->cx.f.prhs = c->fp32 ? nullptr : (double *)c->cx.f.scr;
    c->cf.f.prhs = c->fp32 ? c->stage : nullptr;
    auto &F = c->cx.f;

    // wavenumbers (module_solve_pressure.f90:93-129) and modal y coefficients (:599-609)
    const double PI = std::acos(-1.0), ddx = g.ph.L1 / (double)N1, ddz = g.ph.L3 / (double)N3;
    const int h3p = N3 / 2 + 1;
    std::vector<double> dzk(N3), dxk2(c->cx.h1p), fam(N2 + 2, 0.0), fap(N2 + 2, 0.0);
    for (int k = 1; k <= N3; k++) {
        const int km = (k <= h3p) ? k - 1 : N3 - k + 1;
        dzk[k - 1] = 2.0 * (1.0 - std::cos(2.0 * PI * (double)km * ddz / g.ph.L3)) / (ddz * ddz);
    }
    for (int i = 1; i <= c->cx.h1p; i++) dxk2[i - 1] = 2.0 * (1.0 - std::cos(2.0 * PI * (double)(i - 1) * ddx / g.ph.L1)) / (ddx * ddx);
    const std::vector<double> &dx2 = c->hm[4], &dmx2 = c->hm[5];
    for (int j = 1; j <= N2; j++) {
        fam[j] = (j == 1) ? 0.0 : 1.0 / dx2[j] / dmx2[j];
        fap[j] = (j == N2) ? 0.0 : 1.0 / dx2[j] / dmx2[j + 1];
    }
    r = r ? r : upload_vec(c, dzk, &F.dzk);
    r = r ? r : upload_vec(c, dxk2, &F.dxk2);
    r = r ? r : upload_vec(c, fam, &F.fam);
    r = r ? r : upload_vec(c, fap, &F.fap);
    auto twid = [](int n) {
        std::vector<double2> w(n);
        for (int e = 0; e < n; e++) w[e] = make_double2(std::cos(2.0 * M_PI * (double)e / (double)n), -std::sin(2.0 * M_PI * (double)e / (double)n));
        return w;
    };
    r = r ? r : upload_vec(c, twid(N1), &F.tw1);
    r = r ? r : upload_vec(c, twid(N3), &F.tw3);
    {   // Pbc_a, Pbc_b (module_solve_pressure.f90:720-730)
        const int n2sub = N2 + 1, n2msub = N2;
        const double s1 = (dmx2[1] + dmx2[2]) * (dmx2[1] + dmx2[2]);
        c->cx.wall_ab = s1 / (s1 - dmx2[1] * dmx2[1]);
        c->cx.wall_bb = dmx2[1] * dmx2[1] / (s1 - dmx2[1] * dmx2[1]);
        const double s2 = (dmx2[n2sub] + dmx2[n2msub]) * (dmx2[n2sub] + dmx2[n2msub]);
        c->cx.wall_at = s2 / (s2 - dmx2[n2sub] * dmx2[n2sub]);
        c->cx.wall_bt = dmx2[n2sub] * dmx2[n2sub] / (s2 - dmx2[n2sub] * dmx2[n2sub]);
    }
    c->cx.fp1 = fp1; c->cx.fp3 = fp3; c->cx.fp1u = fp1u;
    const size_t rb1 = row_bytes(1, c->fp32);
    c->cx.tl_contig = choose_tl(N1, true, rb1, 8);
    c->cx.tl_modal = choose_tl(N2, false, row_bytes(2, false), 8);   // modal rows are FP64 in both forms
    {
        const int tz = choose_tl(N3, true, rb1, 8), ty = choose_tl(N2, false, rb1, 8);
        c->cx.tl_strided = tz < ty ? tz : ty;
    }
    // measured on B200 at 256^3: 4 lines per block beats 1, 2, 8 and 16 for both FFT kernels
    c->cx.fft_lines_x = N1 <= 256 ? 4 : (N1 <= 512 ? 2 : 1);
    // z transforms: 16 lines in the one-radix form (256-byte rows), else 4 (2 or 1 for long lines)
    c->cx.fft_lines_z = fftz_form(fp3, 16) == 1 ? 16 : (N3 <= 256 ? 4 : (N3 <= 512 ? 2 : 1));
    // inverse x transform, measured on B200: the one-radix form runs best with 2
    // lines per block (64 or 128 threads; 256^3 and 512^3), the general form with 8
    c->cx.ifft_lines_x = ifftx_form(fp1u, 2) == 1 ? 2 : (ifftx_form(fp1u, 8) ? 8 : 1);
    c->cx.lanes = 32;
    c->cx.long_lines = 2;
    c->cx.y_solver = 1;
    c->cx.thomas_scr = nullptr;
    c->cx.mixed_rows = 1;
    c->cx.z_staging = 1;
    c->cx.probe = &c->probe;
    sync_shapes(c);
    {   // the FP32 context shares the grid, constants, scalars, tables and history
        GridT<float> &gf = c->cf.g;
        gf.N1 = g.N1; gf.N2 = g.N2; gf.N3 = g.N3; gf.P1 = g.P1; gf.P2 = g.P2; gf.NP = g.NP;
        gf.d1 = g.d1; gf.d2 = g.d2; gf.d3 = g.d3;
        gf.ph = phys_cast<float>(g.ph); gf.phd = g.ph;
        gf.scal = g.scal; gf.kdeg2 = g.kdeg2;
        FieldsT<float> &ff = c->cf.f;
        ff.dxk2 = F.dxk2; ff.dzk = F.dzk; ff.fam = F.fam; ff.fap = F.fap;
        ff.tw1 = F.tw1; ff.tw3 = F.tw3;
        ff.part = F.part; ff.hist = F.hist; ff.hist_cap = F.hist_cap;
    }

    // initial fields: mpi_thermal_initial/boundary, mpi_momentum_initial/boundary,
    // mpi_pressure_initial, then ghost(T,U,V,W,P) (main.f90:92-109)
    std::vector<double> T(NP, 0.0);
    const size_t P1 = N1 + 2, P2 = N2 + 2;
    auto I = [&](int i, int j, int k) { return (size_t)i + P1 * ((size_t)j + P2 * (size_t)k); };
    for (int k = 0; k <= N3 + 1; k++)
        for (int i = 0; i <= N1 + 1; i++) {
            T[I(i, 0, k)] = g.ph.Tbt;
            if (cfg->top_wall_mode) T[I(i, N2 + 1, k)] = g.ph.Tup;
        }
    if (cfg->init_mode == 0) {
        const uint64_t base = splitmix64_mix(cfg->seed);
        const std::vector<double> &x2 = c->hm[3];
        for (int k = 1; k <= N3; k++)
            for (int j = 1; j <= N2; j++) {
                const double yc = 0.5 * (x2[j] + x2[j + 1]);
                for (int i = 1; i <= N1; i++) {
                    const uint64_t z = splitmix64_mix(base ^ (uint64_t)I(i, j, k));
                    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
                    T[I(i, j, k)] = 0.5 - yc + cfg->noise_amp * (2.0 * u - 1.0);
                }
            }
    }
    host_ghost(T, N1, N2, N3);
    if (!r) {
        if (c->fp32) {
            const std::vector<float> Tf(T.begin(), T.end());
            cudaMemcpyAsync(c->cf.f.T, Tf.data(), NP * sizeof(float), cudaMemcpyHostToDevice, c->stream);
            cudaMemcpyAsync(c->cf.f.Tn, Tf.data(), NP * sizeof(float), cudaMemcpyHostToDevice, c->stream);
            cudaStreamSynchronize(c->stream);   // Tf is a local
        } else {
            cudaMemcpyAsync(F.T, T.data(), NP * sizeof(double), cudaMemcpyHostToDevice, c->stream);
            cudaMemcpyAsync(F.Tn, T.data(), NP * sizeof(double), cudaMemcpyHostToDevice, c->stream);
        }
        double sc[S_NSCAL] = {0};
        sc[S_DT] = cfg->dtStart; sc[S_TIME] = cfg->tStart; sc[S_CFL] = cfg->MaxCFL;
        sc[S_FIXED_DT] = cfg->fixed_dt ? 1.0 : 0.0;
        cudaMemcpyAsync(g.scal, sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) r = set_err(TCS_ERR_CUDA, "initial upload");
    }
    if (r) { tcs_destroy(c); return r; }
    c->ghost_ok = 0xffffffffu;
    *out = c;
    return TCS_OK;
}

int tcs_destroy(tcs_ctx *c)
{
    if (!c) return TCS_ERR_ARG;
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &ge : c->graphs) cudaGraphExecDestroy(ge.exec);
    for (void *p : c->allocs) cudaFree(p);
    if (c->cx.thomas_scr) cudaFree(c->cx.thomas_scr);
    if (c->io_host) cudaFreeHost(c->io_host);
    for (auto &v : c->probe.rec) for (auto &pr : v) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    for (cudaEvent_t e : c->probe.pool) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return TCS_OK;
}

int tcs_set_stream(tcs_ctx *c, void *s)
{
    if (!c) return set_err(TCS_ERR_ARG, "null context");
    CK(cudaStreamSynchronize(c->stream));
    if (c->own_stream) cudaStreamDestroy(c->stream);
    if (s) { c->stream = (cudaStream_t)s; c->own_stream = false; }
    else { CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)); c->own_stream = true; }
    for (auto &ge : c->graphs) cudaGraphExecDestroy(ge.exec);
    c->graphs.clear();
    return TCS_OK;
}

void *tcs_get_stream(tcs_ctx *c) { return c ? (void *)c->stream : nullptr; }

int tcs_dims(const tcs_ctx *c, int *d)
{
    if (!c || !d) return set_err(TCS_ERR_ARG, "null argument");
    d[0] = c->cx.g.N1 + 2; d[1] = c->cx.g.N2 + 2; d[2] = c->cx.g.N3 + 2;
    return TCS_OK;
}

int tcs_get_metric(const tcs_ctx *c, int which, double *out)
{
    if (!c || !out || which < 0 || which > 8) return set_err(TCS_ERR_ARG, "bad metric");
    std::memcpy(out, c->hm[which].data(), c->hm[which].size() * sizeof(double));
    return TCS_OK;
}

static int copy_field(tcs_ctx *c, int f, double *host, bool up, bool async)
{
    if (!c || !host) return set_err(TCS_ERR_ARG, "null argument");
    cudaSetDevice(c->cfg.device);
    int r = flush_pending(c);
    if (r) return r;
    const size_t NP = (size_t)c->cx.g.NP;
    const GridT<double> &g = c->cx.g;
    if (f == TCS_F_MU || f == TCS_F_INVRHO) {
        if (up) return set_err(TCS_ERR_ARG, "Mu and invRho are derived from T");
        std::vector<double> t((size_t)(g.N2 + 2) * (g.N3 + 2));
        if (c->fp32 && f == TCS_F_MU) {
            std::vector<float> tf(t.size());
            CK(cudaMemcpyAsync(tf.data(), c->cf.f.Mu2, tf.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (size_t q = 0; q < t.size(); q++) t[q] = tf[q];
        } else {   // FP64: Mu, and invRho in both forms
            const double *tab = f == TCS_F_MU ? c->cx.f.Mu2 : (c->fp32 ? c->cf.f.iR2d : c->cx.f.iR2d);
            CK(cudaMemcpyAsync(t.data(), tab, t.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        }
        CK(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < g.N3 + 2; k++)
            for (int j = 0; j < g.N2 + 2; j++)
                for (int i = 0; i < g.N1 + 2; i++) host[(size_t)i + (size_t)g.P1 * ((size_t)j + (size_t)g.P2 * k)] = t[j + (size_t)g.P2 * k];
        return TCS_OK;
    }
    void *d = field_ptr(c, f);
    if (!d) return set_err(TCS_ERR_ARG, "unknown field");
    if (c->fp32) {   // FP64 host arrays pass through the FP64 staging buffer
        float *df = (float *)d, *lo = lo_ptr_t(c->cf.f, f);
        if (up) {
            CK(cudaMemcpyAsync(c->stage, host, NP * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            if (lo) launch_split(c->stage, df, lo, (long long)NP, c->stream);
            else launch_convert_in<float>(c->stage, df, (long long)NP, c->stream);
            if (f == TCS_F_T) launch_convert_in<float>(c->stage, c->cf.f.Tn, (long long)NP, c->stream);
            c->ghost_ok &= ~(1u << f);
        } else {
            if (lo) launch_join(df, lo, c->stage, (long long)NP, c->stream);
            else launch_convert<float>(df, c->stage, (long long)NP, c->stream);
            CK(cudaMemcpyAsync(host, c->stage, NP * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        }
        if ((r = take_launch_error())) return r;
    } else if (up) {
        CK(cudaMemcpyAsync(d, host, NP * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (f == TCS_F_T) CK(cudaMemcpyAsync(c->cx.f.Tn, host, NP * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        c->ghost_ok &= ~(1u << f);
    } else {
        CK(cudaMemcpyAsync(host, d, NP * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (!async) CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

int tcs_upload_field(tcs_ctx *c, int f, const double *h) { return copy_field(c, f, (double *)h, true, false); }
int tcs_download_field(tcs_ctx *c, int f, double *h) { return copy_field(c, f, h, false, false); }
int tcs_upload_field_async(tcs_ctx *c, int f, const double *h) { return copy_field(c, f, (double *)h, true, true); }
int tcs_download_field_async(tcs_ctx *c, int f, double *h) { return copy_field(c, f, h, false, true); }

int tcs_precision(const tcs_ctx *c) { return c ? c->cfg.precision : -1; }

int tcs_field_device_ptr(tcs_ctx *c, int f, void **dev)
{
    if (!c || !dev) return set_err(TCS_ERR_ARG, "null argument");
    int r = flush_pending(c);
    if (r) return r;
    *dev = field_ptr(c, f);
    return *dev ? TCS_OK : set_err(TCS_ERR_ARG, "unknown field");
}

int tcs_synchronize(tcs_ctx *c)
{
    if (!c) return set_err(TCS_ERR_ARG, "null context");
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

int tcs_set_dt(tcs_ctx *c, double dt)
{
    if (!c || !(dt > 0.0)) return set_err(TCS_ERR_ARG, "dt must be positive");
    CK(cudaMemcpyAsync(c->cx.g.scal + S_DT, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

// ---- stages ---------------------------------------------------------------
#define ENTER(c)                                                   \
    if (!(c)) return set_err(TCS_ERR_ARG, "null context");        \
    cudaSetDevice((c)->cfg.device);

int tcs_thermal_coeffi(tcs_ctx *c) { ENTER(c); return TCS_OK; }
int tcs_thermal_coeffi_clean(tcs_ctx *c) { ENTER(c); return TCS_OK; }
int tcs_momentum_coeffi_clean(tcs_ctx *c) { ENTER(c); return TCS_OK; }

static void ensure_ghosts(tcs_ctx *c, int f)
{
    if (c->ghost_ok & (1u << f)) return;
    on_ctx(c, [&](auto &x) {
        launch_ghost(x, field_ptr_t(x.f, f), c->stream);
        if (auto *lo = lo_ptr_t(x.f, f)) launch_ghost(x, lo, c->stream);
    });
    c->ghost_ok |= (1u << f);
}

int tcs_subdomain_ghostcell_update(tcs_ctx *c, int f)
{
    ENTER(c);
    if (f < 0 || f >= TCS_F_MU) return set_err(TCS_ERR_ARG, "unknown field");
    // while the pseudo-update is deferred into the pressure RHS, U/V/W ghosts
    // are written by that fused kernel
    if (c->pending_pseudo && (f == TCS_F_U || f == TCS_F_V || f == TCS_F_W)) return TCS_OK;
    int r = flush_pending(c);
    if (r) return r;
    ensure_ghosts(c, f);
    return take_launch_error();
}

int tcs_thermal_solver(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    ensure_ghosts(c, TCS_F_T); ensure_ghosts(c, TCS_F_U); ensure_ghosts(c, TCS_F_V); ensure_ghosts(c, TCS_F_W);
    on_ctx(c, [&](auto &x) { launch_thermal(x, c->stream); swap_T(x); });
    return take_launch_error();
}

int tcs_momentum_coeffi(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    ensure_ghosts(c, TCS_F_T);
    on_ctx(c, [&](auto &x) { launch_momentum_coeffi(x, c->stream); });
    return take_launch_error();
}

#define SIMPLE_STAGE(name, launcher, outfield)                  \
    int name(tcs_ctx *c)                                        \
    {                                                           \
        ENTER(c);                                               \
        int r = flush_pending(c);                               \
        if (r) return r;                                        \
        on_ctx(c, [&](auto &x) { launcher(x, c->stream); });    \
        if ((outfield) >= 0) c->ghost_ok |= (1u << (outfield)); \
        return take_launch_error();                             \
    }
SIMPLE_STAGE(tcs_momentum_solvedU, launch_solve_du, TCS_F_DU)
SIMPLE_STAGE(tcs_momentum_solvedV, launch_solve_dv, TCS_F_DV)
SIMPLE_STAGE(tcs_momentum_solvedW, launch_solve_dw, TCS_F_DW)
SIMPLE_STAGE(tcs_momentum_blockLdV, launch_blockld_v, TCS_F_DV)
#undef SIMPLE_STAGE

int tcs_momentum_blockLdU(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    on_ctx(c, [&](auto &x) { launch_blockld_u(x, c->stream); });
    c->ghost_ok &= ~(1u << TCS_F_DU);   // the reference leaves dU's ghosts stale here
    return take_launch_error();
}

int tcs_momentum_pseudoupdateUVW(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    c->pending_pseudo = true;          // executed inside tcs_pressure_RHS
    c->ghost_ok |= (1u << TCS_F_U) | (1u << TCS_F_V) | (1u << TCS_F_W);
    return TCS_OK;
}

int tcs_pressure_RHS(tcs_ctx *c)
{
    ENTER(c);
    ensure_ghosts(c, TCS_F_DPHAT);
    if (c->pending_pseudo) {
        on_ctx(c, [&](auto &x) { launch_pseudo_prhs_fftx(x, c->stream, true); swap_UVW(x); });
        c->pending_pseudo = false;
    } else {
        ensure_ghosts(c, TCS_F_U); ensure_ghosts(c, TCS_F_V); ensure_ghosts(c, TCS_F_W);
        on_ctx(c, [&](auto &x) { launch_pseudo_prhs_fftx(x, c->stream, false); });
    }
    return take_launch_error();
}

int tcs_pressure_Poisson_FFT2(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    on_ctx(c, [&](auto &x) { launch_poisson_rest(x, c->stream); });
    c->ghost_ok |= (1u << TCS_F_DP);
    return take_launch_error();
}

// Transpose scheme 1 (module_solve_pressure.f90:238-482).  On one rank its
// arithmetic is scheme 2's: the same r2c x and c2c z transforms in the same
// order, dxk1 = dxk2 (both span the whole half spectrum, :118-127), the same
// pin of mode (0,0), the same zeroing of the imaginary (0,0) and (0,h3p)
// modes, scaling, mean removal and wall extrapolation.  With no transposes to
// choose between on one GPU, both entry points run the same kernels.
int tcs_pressure_Poisson_FFT1(tcs_ctx *c) { return tcs_pressure_Poisson_FFT2(c); }

int tcs_pressure_Projection(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    ensure_ghosts(c, TCS_F_DPHAT);
    on_ctx(c, [&](auto &x) { launch_projection(x, c->stream); swap_phat(x); });
    c->ghost_ok |= (1u << TCS_F_U) | (1u << TCS_F_V) | (1u << TCS_F_W) | (1u << TCS_F_P) | (1u << TCS_F_DPHAT);
    return take_launch_error();
}

int tcs_post_div(tcs_ctx *c, double *maxDivU)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    on_ctx(c, [&](auto &x) { launch_post(x, c->stream, 1); });
    if ((r = take_launch_error())) return r;
    double sc[S_NSCAL];
    CK(cudaMemcpyAsync(sc, c->cx.g.scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (maxDivU) *maxDivU = sc[S_MAXDIV];
    return sc[S_BLOWUP] != 0.0 ? set_err(TCS_ERR_BLOWUP, "BLOW UP: max divergence >= 1e-3") : TCS_OK;
}

int tcs_post_cfl(tcs_ctx *c, double *CFL, double *dt)
{
    ENTER(c);
    double sc[S_NSCAL];
    CK(cudaMemcpyAsync(sc, c->cx.g.scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (CFL) *CFL = sc[S_CFL];
    if (dt) *dt = sc[S_DT];
    return std::isfinite(sc[S_DT]) ? TCS_OK : set_err(TCS_ERR_NONFINITE, "dt is not finite");
}

} // extern "C"

template <class R>
static void launch_step_t(Ctx<R> &cx, cudaStream_t s)
{
    launch_thermal(cx, s);
    swap_T(cx);
    launch_momentum_coeffi(cx, s);
    launch_solve_du(cx, s);
    launch_solve_dv(cx, s);
    launch_solve_dw(cx, s);
    launch_blockld_v(cx, s);
    launch_blockld_u(cx, s);
    launch_pseudo_prhs_fftx(cx, s, true);
    swap_UVW(cx);
    launch_poisson_rest(cx, s);
    launch_projection(cx, s);
    swap_phat(cx);
    launch_post(cx, s, 1);
}

static void launch_step(tcs_ctx *c)
{
    on_ctx(c, [&](auto &x) { launch_step_t(x, c->stream); });
}

extern "C" {

// Launch-shape knobs (lines per block of the line-solver families and of the
// FFT kernels).  A line-solver value is the most lines per block: every
// launch fits it down (fit_tl halves it until the family's blocks per SM fit
// the SM's shared memory), so the value that runs is the largest power of two
// up to it that fits.  Values are refused only where one block of the
// family's largest row type could not hold them at all (227 KB per block);
// the bound takes the bank-padded line stride of the non-cyclic strided
// problems (at most one bank row, 32 words, above the odd stride).
static bool lines_fit_one_block(size_t rowb, int value, int LS, int n)
{
    return rowb * (size_t)value * (size_t)(LS + 32) + (size_t)n * sizeof(int) <= (size_t)227 * 1024;
}

int tcs_set_tuning(tcs_ctx *c, int knob, int value)
{
    ENTER(c);
    if (value < 1 || value > 64 || (value & (value - 1))) return set_err(TCS_ERR_ARG, "tuning value must be a power of two in 1..64");
    Ctx<double> &x = c->cx;
    const GridT<double> &g = x.g;
    const size_t rb1 = row_bytes(1, c->fp32);
    switch (knob) {
    case TCS_TUNE_TL_STRIDED: {
        LinePlan a = make_line_plan(g.N3, true, value), b = make_line_plan(g.N2, false, value);
        if (!lines_fit_one_block(rb1, value, std::max(a.LS, b.LS), std::max(g.N2, g.N3)))
            return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.tl_strided = value; break; }
    case TCS_TUNE_TL_CONTIG: {
        LinePlan a = make_line_plan(g.N1, true, value);
        if (!lines_fit_one_block(rb1, value, a.LS, g.N1)) return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.tl_contig = value; break; }
    case TCS_TUNE_TL_MODAL: {
        LinePlan a = make_line_plan(g.N2, false, value);
        if (!lines_fit_one_block(row_bytes(2, false), value, a.LS, g.N2)) return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.tl_modal = value; break; }
    case TCS_TUNE_FFT_LINES_X:
        if ((size_t)value * g.N1 * (32 + esize(c)) > 200 * 1024) return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.fft_lines_x = value; break;
    case TCS_TUNE_FFT_LINES_Z:
        if (!fftz_form(x.fp3, value)) return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.fft_lines_z = value; break;
    case TCS_TUNE_IFFT_LINES_X:
        if (!ifftx_form(x.fp1u, value)) return set_err(TCS_ERR_ARG, "too many lines for shared memory");
        x.ifft_lines_x = value; break;
    case TCS_TUNE_MIXED_ROWS:
        if (value > 8) return set_err(TCS_ERR_ARG, "mixed rows: 1 FP32 elimination, 2 FP64 rows in the x sweeps, 4 x and z sweeps, 8 z at 3 blocks per SM");
        x.mixed_rows = value; break;
    case TCS_TUNE_Z_STAGING:
        if (value > 2) return set_err(TCS_ERR_ARG, "z staging: 1 global loads, 2 TMA-staged inputs for dw_z");
        if (value == 2 && (c->fp32 || !dwz_staging_possible(x)))
            return set_err(TCS_ERR_ARG, "z staging needs the FP64 form, N3 a multiple of 64 and an even N1");
        x.z_staging = value; break;
    case TCS_TUNE_LANES:
        if (value < 2 || value > 32) return set_err(TCS_ERR_ARG, "lanes per line must be 2..32");
        x.lanes = value; break;
    case TCS_TUNE_LONG_LINES:
        if (value > 4) return set_err(TCS_ERR_ARG, "long-line form: 1 never, 2 z sweeps, 4 z and y sweeps");
        x.long_lines = value; break;
    case TCS_TUNE_Y_SOLVER: {
        if (value > 4) return set_err(TCS_ERR_ARG, "y solver: 1 partitioned, 2 one line per thread (y sweeps), 4 also the modal solves");
        // c', d' of every line of the largest one-line-per-thread launch: the y
        // sweeps (one right-hand side) and, with 4, the modal solves (two)
        const size_t ny = value >= 2 ? thomas_words(g.N2, g.N1, g.N3, 1) : 0;
        const size_t words = std::max(ny, value == 4 ? thomas_words(g.N2, x.h1p, g.N3, 2) : (size_t)0);
        if (x.thomas_scr) {
            cudaStreamSynchronize(c->stream);
            cudaFree(x.thomas_scr);
            x.thomas_scr = nullptr;
        }
        if (words) {
            void *q = nullptr;
            const cudaError_t ce = cudaMalloc(&q, words * sizeof(double));
            if (ce != cudaSuccess) {
                cudaGetLastError();
                x.y_solver = 1;
                sync_shapes(c);
                return set_err(TCS_ERR_NOMEM, std::string("y solver scratch: ") + cudaGetErrorString(ce));
            }
            x.thomas_scr = (double *)q;
        }
        x.y_solver = value; break; }
    default: return set_err(TCS_ERR_ARG, "unknown tuning knob");
    }
    sync_shapes(c);
    for (auto &ge : c->graphs) cudaGraphExecDestroy(ge.exec);
    c->graphs.clear();
    return TCS_OK;
}

int tcs_get_tuning(tcs_ctx *c, int knob, int *value)
{
    ENTER(c);
    if (!value) return set_err(TCS_ERR_ARG, "null argument");
    const Ctx<double> &x = c->cx;
    switch (knob) {
    case TCS_TUNE_TL_STRIDED: *value = x.tl_strided; break;
    case TCS_TUNE_TL_CONTIG: *value = x.tl_contig; break;
    case TCS_TUNE_TL_MODAL: *value = x.tl_modal; break;
    case TCS_TUNE_FFT_LINES_X: *value = x.fft_lines_x; break;
    case TCS_TUNE_FFT_LINES_Z: *value = x.fft_lines_z; break;
    case TCS_TUNE_LANES: *value = x.lanes; break;
    case TCS_TUNE_LONG_LINES: *value = x.long_lines; break;
    case TCS_TUNE_Y_SOLVER: *value = x.y_solver; break;
    case TCS_TUNE_IFFT_LINES_X: *value = x.ifft_lines_x; break;
    case TCS_TUNE_MIXED_ROWS: *value = x.mixed_rows; break;
    case TCS_TUNE_Z_STAGING: *value = x.z_staging; break;
    default: return set_err(TCS_ERR_ARG, "unknown tuning knob");
    }
    return TCS_OK;
}

int tcs_set_use_graph(tcs_ctx *c, int on)
{
    ENTER(c);
    c->use_graph = on != 0;
    return TCS_OK;
}

int tcs_step(tcs_ctx *c, int nsteps, int *done)
{
    ENTER(c);
    if (done) *done = 0;
    if (nsteps < 0) return set_err(TCS_ERR_ARG, "nsteps < 0");
    int r = flush_pending(c);
    if (r) return r;
    const int fl[] = {TCS_F_T, TCS_F_U, TCS_F_V, TCS_F_W, TCS_F_P, TCS_F_DPHAT};
    for (int f : fl) ensure_ghosts(c, f);
    if ((r = take_launch_error())) return r;
    double sc0[S_NSCAL];
    CK(cudaMemcpyAsync(sc0, c->cx.g.scal, sizeof(sc0), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (sc0[S_BLOWUP] != 0.0) return set_err(TCS_ERR_BLOWUP, "the case has already blown up");
    const bool graph = c->use_graph && c->probe.mask == 0;
    for (int n = 0; n < nsteps; n++) {
        if (!graph) {
            launch_step(c);
            if ((r = take_launch_error())) return r;
            continue;
        }
        const void *T0 = field_ptr(c, TCS_F_T), *U0 = field_ptr(c, TCS_F_U), *P0 = field_ptr(c, TCS_F_DPHAT);
        cudaGraphExec_t exec = nullptr;
        unsigned long long kernels_this = 0;
        for (auto &ge : c->graphs) if (ge.T == T0 && ge.U == U0 && ge.dPhat == P0) { exec = ge.exec; kernels_this = ge.kernels; break; }
        if (!exec) {
            cudaGraph_t gr;
            const unsigned long long before = g_launches;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            launch_step(c);
            const unsigned long long nk = g_launches - before;
            g_launches = before;
            cudaError_t ec = cudaStreamEndCapture(c->stream, &gr);
            if (ec != cudaSuccess || take_launch_error()) return set_err(TCS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
            CK(cudaGraphInstantiate(&exec, gr, 0));
            cudaGraphDestroy(gr);
            c->graphs.push_back({T0, U0, P0, exec, nk});
            kernels_this = nk;
            // capture swapped the buffers already; the launch below performs that step
        } else {
            on_ctx(c, [&](auto &x) { swap_T(x); swap_UVW(x); swap_phat(x); });
        }
        CK(cudaGraphLaunch(exec, c->stream));
        g_launches += kernels_this;
    }
    double sc[S_NSCAL];
    CK(cudaMemcpyAsync(sc, c->cx.g.scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->ghost_ok |= (1u << TCS_F_T) | (1u << TCS_F_U) | (1u << TCS_F_V) | (1u << TCS_F_W) | (1u << TCS_F_P) | (1u << TCS_F_DPHAT) | (1u << TCS_F_DP);
    const int steps_now = (int)sc[S_STEP] - (int)sc0[S_STEP];
    if (done) *done = steps_now;
    if (sc[S_BLOWUP] != 0.0) return set_err(TCS_ERR_BLOWUP, "BLOW UP: max divergence >= 1e-3");
    return TCS_OK;
}

// The buffers a snapshot holds: T, U, V, W, P, dPhat, dP0 and, in the FP32
// form, the low words of U, V, W.
static int snap_buffers(tcs_ctx *c, void **b)
{
    const int fl[7] = {TCS_F_T, TCS_F_U, TCS_F_V, TCS_F_W, TCS_F_P, TCS_F_DPHAT, TCS_F_DP0};
    for (int q = 0; q < 7; q++) b[q] = field_ptr(c, fl[q]);
    if (!c->fp32) return 7;
    b[7] = c->cf.f.Ulo; b[8] = c->cf.f.Vlo; b[9] = c->cf.f.Wlo;
    return 10;
}

// On-device checkpoint of the state a time step reads (T, U, V, W, P, dPhat,
// dP0 and the scalars): a restart that needs no host round trip.
int tcs_snapshot(tcs_ctx *c)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    const size_t bytes = (size_t)c->cx.g.NP * esize(c);
    void *src[10];
    const int n = snap_buffers(c, src);
    for (int q = 0; q < n; q++) {
        unsigned char *sp = (unsigned char *)c->snap[q];
        if (!sp && (r = dalloc(c, &sp, bytes))) return r;
        c->snap[q] = sp;
        CK(cudaMemcpyAsync(c->snap[q], src[q], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaMemcpyAsync(c->snap_scal, c->cx.g.scal, sizeof(c->snap_scal), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->have_snap = true;
    return TCS_OK;
}

int tcs_restore(tcs_ctx *c)
{
    ENTER(c);
    if (!c->have_snap) return set_err(TCS_ERR_ARG, "no snapshot");
    int r = flush_pending(c);
    if (r) return r;
    const size_t bytes = (size_t)c->cx.g.NP * esize(c);
    void *dst[10];
    const int n = snap_buffers(c, dst);
    for (int q = 0; q < n; q++)
        CK(cudaMemcpyAsync(dst[q], c->snap[q], bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->cx.g.scal, c->snap_scal, sizeof(c->snap_scal), cudaMemcpyHostToDevice, c->stream));
    c->ghost_ok |= (1u << TCS_F_T) | (1u << TCS_F_U) | (1u << TCS_F_V) | (1u << TCS_F_W) | (1u << TCS_F_P) | (1u << TCS_F_DPHAT);
    return TCS_OK;
}

int tcs_get_scalars(tcs_ctx *c, double *out)
{
    ENTER(c);
    if (!out) return set_err(TCS_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(out, c->cx.g.scal, sizeof(double) * S_NSCAL, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

int tcs_get_history(tcs_ctx *c, int first, int count, double *out)
{
    ENTER(c);
    if (!out || first < 0 || count < 0 || first + count > c->cx.f.hist_cap) return set_err(TCS_ERR_ARG, "history range");
    CK(cudaMemcpyAsync(out, c->cx.f.hist + (size_t)first * 7, sizeof(double) * 7 * (size_t)count, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

// ---- probes ---------------------------------------------------------------
int tcs_probe_enable(tcs_ctx *c, uint64_t mask)
{
    ENTER(c);
    c->probe.mask = mask;
    return TCS_OK;
}

int tcs_probe_read(tcs_ctx *c, int kid, double *total_ms, int *launches)
{
    ENTER(c);
    if (kid < 0 || kid >= K_COUNT) return set_err(TCS_ERR_ARG, "kernel id");
    CK(cudaStreamSynchronize(c->stream));
    double t = 0.0;
    for (auto &pr : c->probe.rec[kid]) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        t += ms;
    }
    if (total_ms) *total_ms = t;
    if (launches) *launches = (int)c->probe.rec[kid].size();
    return TCS_OK;
}

int tcs_probe_reset(tcs_ctx *c)
{
    ENTER(c);
    CK(cudaStreamSynchronize(c->stream));
    for (auto &v : c->probe.rec) {
        for (auto &pr : v) { c->probe.pool.push_back(pr.first); c->probe.pool.push_back(pr.second); }
        v.clear();
    }
    return TCS_OK;
}

// ---- PaScaL_TDMA ------------------------------------------------------------
} // extern "C"

// A plan borrows a (stream, device staging buffer) slot from a per-process
// pool and returns it when destroyed.  The reference creates and destroys a
// plan around every sweep (module_solve_thermal.f90:364-366 and every solve of
// module_solve_momentum.f90 and module_solve_pressure.f90), so a caller that
// keeps the reference's solvers and swaps in only PaScaL_TDMA would otherwise
// pay a stream creation, a cudaMalloc and a cudaFree per sweep; with the pool
// the staging grows to the largest system seen on the device and stays.
// Slots are per device; a slot is used by one plan at a time, so plans alive
// at the same time (other host threads) stage through different buffers.
struct TdmaSlot {
    int device;
    cudaStream_t stream;
    double *buf;
    size_t cap;
    bool busy;
};
static std::mutex g_tdma_mu;
static std::vector<TdmaSlot *> g_tdma_slots;

struct tcs_tdma_plan {
    int n_sys;
    TdmaSlot *slot;
};

extern "C" {

int tcs_tdma_plan_many_create(tcs_tdma_plan **plan, int n_sys, int myrank, int nprocs)
{
    if (!plan || n_sys < 1) return set_err(TCS_ERR_ARG, "bad plan arguments");
    if (nprocs != 1 || myrank != 0) return set_err(TCS_ERR_UNSUPPORTED, "one GPU holds the whole line: nprocs must be 1");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    TdmaSlot *sl = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_tdma_mu);
        for (TdmaSlot *t : g_tdma_slots)
            if (!t->busy && t->device == dev) { sl = t; break; }
        if (!sl) {
            sl = new TdmaSlot{dev, nullptr, nullptr, 0, false};
            if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess) {
                delete sl;
                return set_err(TCS_ERR_CUDA, "stream");
            }
            g_tdma_slots.push_back(sl);
        }
        sl->busy = true;
    }
    tcs_tdma_plan *p = new tcs_tdma_plan();
    p->n_sys = n_sys;
    p->slot = sl;
    *plan = p;
    return TCS_OK;
}

int tcs_tdma_plan_many_destroy(tcs_tdma_plan *p)
{
    if (!p) return set_err(TCS_ERR_ARG, "null plan");
    cudaStreamSynchronize(p->slot->stream);
    {
        std::lock_guard<std::mutex> lk(g_tdma_mu);
        p->slot->busy = false;
    }
    delete p;
    return TCS_OK;
}

static int tdma_solve(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_sys, int n_row, int cyclic)
{
    if (!p || !A || !B || !C || !D) return set_err(TCS_ERR_ARG, "null argument");
    if (n_sys != p->n_sys || n_row < 2) return set_err(TCS_ERR_ARG, "n_sys must match the plan and n_row >= 2");
    TdmaSlot *sl = p->slot;
    cudaSetDevice(sl->device);
    cudaPointerAttributes at;
    bool dev = cudaPointerGetAttributes(&at, D) == cudaSuccess && at.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    const size_t n = (size_t)n_sys * n_row;
    if (dev) {
        launch_tdma_many(A, B, C, D, n_sys, n_row, cyclic, sl->stream);
        if (take_launch_error()) return TCS_ERR_CUDA;
        CK(cudaStreamSynchronize(sl->stream));
        return TCS_OK;
    }
    if (sl->cap < 4 * n) {
        if (sl->buf) cudaFree(sl->buf);
        sl->buf = nullptr; sl->cap = 0;
        CK(cudaMalloc(&sl->buf, 4 * n * sizeof(double)));
        sl->cap = 4 * n;
    }
    double *dA = sl->buf, *dB = dA + n, *dC = dB + n, *dD = dC + n;
    CK(cudaMemcpyAsync(dA, A, n * sizeof(double), cudaMemcpyHostToDevice, sl->stream));
    CK(cudaMemcpyAsync(dB, B, n * sizeof(double), cudaMemcpyHostToDevice, sl->stream));
    CK(cudaMemcpyAsync(dC, C, n * sizeof(double), cudaMemcpyHostToDevice, sl->stream));
    CK(cudaMemcpyAsync(dD, D, n * sizeof(double), cudaMemcpyHostToDevice, sl->stream));
    launch_tdma_many(dA, dB, dC, dD, n_sys, n_row, cyclic, sl->stream);
    if (take_launch_error()) return TCS_ERR_CUDA;
    CK(cudaMemcpyAsync(A, dA, n * sizeof(double), cudaMemcpyDeviceToHost, sl->stream));
    CK(cudaMemcpyAsync(C, dC, n * sizeof(double), cudaMemcpyDeviceToHost, sl->stream));
    CK(cudaMemcpyAsync(D, dD, n * sizeof(double), cudaMemcpyDeviceToHost, sl->stream));
    CK(cudaStreamSynchronize(sl->stream));
    return TCS_OK;
}

int tcs_tdma_many_solve(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    return tdma_solve(p, A, B, C, D, n_sys, n_row, 0);
}

int tcs_tdma_many_solve_cycle(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    return tdma_solve(p, A, B, C, D, n_sys, n_row, 1);
}

} // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: many independent cases on one GPU advanced together.  One step
// of every case is captured into a single CUDA graph, each case on its own
// branch forked from a root stream, so one graph launch advances the whole
// ensemble and the GPU runs the cases' kernels concurrently (small grids do
// not fill 148 SMs on their own).  Graphs are cached per buffer state, as in
// tcs_step.
// ---------------------------------------------------------------------------
struct tcs_ensemble {
    std::vector<tcs_ctx *> cases;
    int device = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr, fork2 = nullptr;
    std::vector<cudaEvent_t> join, join2;
    // the form of a step: 1 = batched (a line sweep is one multi-case launch),
    // 0 = one graph branch per case, -1 = auto (measure both, keep the faster)
    int mode = -1;
    int chosen = -1;          // auto: the form picked, -1 while measuring
    int tune_step = 0;        // auto: steps of the measurement taken so far (of 8)
    float tune_ms[2] = {-1.f, -1.f};
    cudaEvent_t tev[2][2] = {};
    struct Entry {
        std::vector<const void *> key;
        bool batched;
        cudaGraphExec_t exec;
        unsigned long long kernels;
        void *arena;
    };
    std::vector<Entry> graphs;
};

static void ensemble_drop_graphs(tcs_ensemble *e)
{
    for (auto &g : e->graphs) {
        cudaGraphExecDestroy(g.exec);
        if (g.arena) cudaFree(g.arena);
    }
    e->graphs.clear();
}

// One step of every case in the batched form.  The line sweeps (thermal,
// solvedU/V/W, the modal Poisson solves) run as one line_solve_multi launch
// per sweep on the root stream; the kernels between them run as one branch
// per case (forked from and joined back to the root).  In planning mode
// nothing is launched: the multi-case launches append their work lists to
// the arena and the host-side buffer swaps are applied as the step makes them.
static void ensemble_sequence(tcs_ensemble *e, MultiArena &A)
{
    const bool plan = A.planning;
    std::vector<Ctx<double> *> d;
    std::vector<Ctx<float> *> f;
    for (tcs_ctx *c : e->cases) {
        if (c->fp32) f.push_back(&c->cf);
        else d.push_back(&c->cx);
    }
    auto branches = [&](auto &&body) {
        if (!plan) cudaEventRecord(e->fork, e->root);
        for (size_t i = 0; i < e->cases.size(); i++) {
            tcs_ctx *c = e->cases[i];
            if (!plan) cudaStreamWaitEvent(c->stream, e->fork, 0);
            on_ctx(c, [&](auto &x) { body(x, c->stream); });
            if (!plan) {
                cudaEventRecord(e->join[i], c->stream);
                cudaStreamWaitEvent(e->root, e->join[i], 0);
            }
        }
    };
    launch_thermal_multi(d, A, e->root);
    launch_thermal_multi(f, A, e->root);
    branches([&](auto &x, cudaStream_t s) {
        swap_T(x);
        if (!plan) launch_momentum_coeffi(x, s);
    });
    launch_momentum_multi(d, A, e->root);
    launch_momentum_multi(f, A, e->root);
    branches([&](auto &x, cudaStream_t s) {
        if (!plan) {
            launch_blockld_v(x, s);
            launch_blockld_u(x, s);
            launch_pseudo_prhs_fftx(x, s, true);
        }
        swap_UVW(x);
        if (!plan) launch_poisson_fwd(x, s);
    });
    launch_modal_multi(d, A, e->root);
    launch_modal_multi(f, A, e->root);
    branches([&](auto &x, cudaStream_t s) {
        if (!plan) {
            launch_poisson_back(x, s);
            launch_projection(x, s);
        }
        swap_phat(x);
        if (!plan) launch_post(x, s, 1);
    });
}

// Capture one step of every case into a graph (the buffers swap as the step
// swaps them).  Batched: plan the multi-case launches, put the buffer state
// back, upload the work lists once, then capture; the graph keeps the upload.
static int ensemble_capture(tcs_ensemble *e, bool batched, cudaGraphExec_t *exec, unsigned long long *nk, void **arena)
{
    *exec = nullptr;
    *arena = nullptr;
    MultiArena A;
    if (batched) {
        ensemble_sequence(e, A);
        for (tcs_ctx *c : e->cases) on_ctx(c, [&](auto &x) { swap_T(x); swap_UVW(x); swap_phat(x); });
        CK(cudaMalloc(&A.dev, std::max<size_t>(A.host.size(), 16)));
        *arena = A.dev;
        CK(cudaMemcpy(A.dev, A.host.data(), A.host.size(), cudaMemcpyHostToDevice));
        A.planning = false;
        A.cursor = 0;
        // a stage's later launches run on the case streams (idle while the root runs a stage)
        A.fork = e->fork2;
        for (size_t i = 0; i < e->cases.size(); i++) {
            A.aux.push_back(e->cases[i]->stream);
            A.join.push_back(e->join2[i]);
        }
    }
    cudaGraph_t gr;
    const unsigned long long before = g_launches;
    CK(cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal));
    if (batched) {
        ensemble_sequence(e, A);
    } else {
        cudaEventRecord(e->fork, e->root);
        for (size_t i = 0; i < e->cases.size(); i++) {
            tcs_ctx *c = e->cases[i];
            cudaStreamWaitEvent(c->stream, e->fork, 0);
            launch_step(c);
            cudaEventRecord(e->join[i], c->stream);
            cudaStreamWaitEvent(e->root, e->join[i], 0);
        }
    }
    *nk = g_launches - before;
    g_launches = before;
    cudaError_t ec = cudaStreamEndCapture(e->root, &gr);
    if (ec != cudaSuccess || take_launch_error())
        return set_err(TCS_ERR_CUDA, std::string("ensemble graph capture: ") + cudaGetErrorString(ec));
    if (batched && A.cursor != A.host.size()) {
        cudaGraphDestroy(gr);
        return set_err(TCS_ERR_CUDA, "ensemble work lists do not match the captured step");
    }
    ec = cudaGraphInstantiate(exec, gr, 0);
    cudaGraphDestroy(gr);
    if (ec != cudaSuccess) return set_err(TCS_ERR_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(ec));
    return TCS_OK;
}

static std::vector<const void *> ensemble_key(tcs_ensemble *e)
{
    std::vector<const void *> k;
    for (tcs_ctx *c : e->cases) {
        k.push_back(field_ptr(c, TCS_F_T));
        k.push_back(field_ptr(c, TCS_F_U));
        k.push_back(field_ptr(c, TCS_F_DPHAT));
    }
    return k;
}

extern "C" {

int tcs_ensemble_create(tcs_ctx *const *cases, int n, tcs_ensemble **out)
{
    if (!cases || !out || n < 1) return set_err(TCS_ERR_ARG, "need at least one case");
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!cases[i]) return set_err(TCS_ERR_ARG, "null case");
        if (cases[i]->cfg.device != cases[0]->cfg.device) return set_err(TCS_ERR_ARG, "all cases must be on one device");
        if (cases[i]->probe.mask) return set_err(TCS_ERR_ARG, "disable the probes of every case first");
        for (int j = 0; j < i; j++)
            if (cases[j] == cases[i] || cases[j]->stream == cases[i]->stream)
                return set_err(TCS_ERR_ARG, "cases must be distinct and on distinct streams");
    }
    CK(cudaSetDevice(cases[0]->cfg.device));
    tcs_ensemble *e = new tcs_ensemble();
    e->cases.assign(cases, cases + n);
    e->device = cases[0]->cfg.device;
    bool ok = cudaStreamCreateWithFlags(&e->root, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork2, cudaEventDisableTiming) == cudaSuccess;
    for (int f = 0; f < 2 && ok; f++)
        for (int q = 0; q < 2 && ok; q++) ok = cudaEventCreate(&e->tev[f][q]) == cudaSuccess;
    e->join.assign(n, nullptr);
    e->join2.assign(n, nullptr);
    for (int i = 0; i < n && ok; i++)
        ok = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->join2[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { tcs_ensemble_destroy(e); return set_err(TCS_ERR_CUDA, "ensemble streams/events"); }
    *out = e;
    return TCS_OK;
}

int tcs_ensemble_destroy(tcs_ensemble *e)
{
    if (!e) return TCS_ERR_ARG;
    cudaSetDevice(e->device);
    if (e->root) cudaStreamSynchronize(e->root);
    ensemble_drop_graphs(e);
    for (cudaEvent_t ev : e->join) if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : e->join2) if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->fork2) cudaEventDestroy(e->fork2);
    for (auto &tf : e->tev)
        for (cudaEvent_t ev : tf) if (ev) cudaEventDestroy(ev);
    if (e->root) cudaStreamDestroy(e->root);
    delete e;
    return TCS_OK;
}

// nsteps whole steps of every case; *nblown receives how many cases have
// blown up (their fields stay at the step that blew up, as in tcs_step).
int tcs_ensemble_step(tcs_ensemble *e, int nsteps, int *nblown)
{
    if (!e || nsteps < 0) return set_err(TCS_ERR_ARG, "bad ensemble arguments");
    CK(cudaSetDevice(e->device));
    int r;
    const int fl[] = {TCS_F_T, TCS_F_U, TCS_F_V, TCS_F_W, TCS_F_P, TCS_F_DPHAT};
    for (tcs_ctx *c : e->cases) {
        if ((r = flush_pending(c))) return r;
        for (int f : fl) ensure_ghosts(c, f);
        if ((r = take_launch_error())) return r;
        CK(cudaStreamSynchronize(c->stream));
    }
    for (int s = 0; s < nsteps; s++) {
        // auto: steps 0-3 run one branch per case, 4-7 batched; steps 2-3 and 6-7 are timed
        bool form;
        int tstep = -1;
        if (e->mode >= 0) form = e->mode == 1;
        else if (e->chosen >= 0) form = e->chosen == 1;
        else {
            tstep = e->tune_step;
            form = tstep >= 4;
        }
        const std::vector<const void *> key = ensemble_key(e);
        cudaGraphExec_t exec = nullptr;
        unsigned long long kernels = 0;
        for (auto &g : e->graphs)
            if (g.key == key && g.batched == form) { exec = g.exec; kernels = g.kernels; break; }
        if (!exec) {
            void *arena = nullptr;
            const int rc = ensemble_capture(e, form, &exec, &kernels, &arena);
            if (rc) {
                if (arena) cudaFree(arena);
                return rc;
            }
            e->graphs.push_back({key, form, exec, kernels, arena});
            // the capture swapped every case's buffers already
        } else {
            for (tcs_ctx *c : e->cases) on_ctx(c, [&](auto &x) { swap_T(x); swap_UVW(x); swap_phat(x); });
        }
        if (tstep >= 0 && (tstep & 3) == 2) CK(cudaEventRecord(e->tev[form][0], e->root));
        CK(cudaGraphLaunch(exec, e->root));
        g_launches += kernels;
        if (tstep >= 0 && (tstep & 3) == 3) CK(cudaEventRecord(e->tev[form][1], e->root));
        if (tstep >= 0 && ++e->tune_step == 8) {
            CK(cudaStreamSynchronize(e->root));
            for (int f = 0; f < 2; f++) {
                CK(cudaEventElapsedTime(&e->tune_ms[f], e->tev[f][0], e->tev[f][1]));
                e->tune_ms[f] *= 0.5f;
            }
            e->chosen = e->tune_ms[1] < e->tune_ms[0] ? 1 : 0;
        }
    }
    CK(cudaStreamSynchronize(e->root));
    int blown = 0;
    for (tcs_ctx *c : e->cases) {
        double sc[S_NSCAL];
        CK(cudaMemcpy(sc, c->cx.g.scal, sizeof(sc), cudaMemcpyDeviceToHost));
        if (sc[S_BLOWUP] != 0.0) blown++;
        c->ghost_ok |= (1u << TCS_F_T) | (1u << TCS_F_U) | (1u << TCS_F_V) | (1u << TCS_F_W) | (1u << TCS_F_P) |
                       (1u << TCS_F_DPHAT) | (1u << TCS_F_DP);
    }
    if (nblown) *nblown = blown;
    return TCS_OK;
}

int tcs_ensemble_size(const tcs_ensemble *e) { return e ? (int)e->cases.size() : 0; }

int tcs_ensemble_set_batched(tcs_ensemble *e, int mode)
{
    if (!e || mode < -1 || mode > 1) return set_err(TCS_ERR_ARG, "mode must be 1 (batched), 0 (branch per case) or -1 (auto)");
    e->mode = mode;
    return TCS_OK;
}

int tcs_ensemble_form(const tcs_ensemble *e, int *form, float *ms_branches, float *ms_batched)
{
    if (!e) return set_err(TCS_ERR_ARG, "null ensemble");
    if (form) *form = e->mode >= 0 ? e->mode : e->chosen;
    if (ms_branches) *ms_branches = e->tune_ms[0];
    if (ms_batched) *ms_batched = e->tune_ms[1];
    return TCS_OK;
}
} // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: coordinate descent over the launch-shape knobs, each candidate
// timed with CUDA events over a few graph-replayed steps from the same state.
// Results are cached per (grid shape, precision) for the process and, when a
// path is given, in a text file of lines "n1 n2 n3 precision k0 .. k5".
// ---------------------------------------------------------------------------
namespace {
struct TuneKey {
    int n1, n2, n3, prec;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(n1, n2, n3, prec) < std::tie(o.n1, o.n2, o.n3, o.prec);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::vector<int>> g_tune;
std::map<std::string, bool> g_tune_files;

void tune_load(const std::string &path)
{
    if (path.empty() || g_tune_files[path]) return;
    g_tune_files[path] = true;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        TuneKey k;
        std::vector<int> v(TCS_TUNE_COUNT, 0);
        if (!(ss >> k.n1 >> k.n2 >> k.n3 >> k.prec)) continue;
        int got = 0;
        while (got < TCS_TUNE_COUNT && (ss >> v[got])) got++;
        // lines written before the later knobs existed leave those knobs as they are (0)
        if (got >= TCS_TUNE_LONG_LINES + 1) g_tune[k] = v;
    }
}
} // namespace

static int tune_trial(tcs_ctx *c, int steps, float *ms)
{
    int r, done = 0;
    if ((r = tcs_restore(c))) return r;
    if ((r = tcs_step(c, 1, &done)) && r != TCS_ERR_BLOWUP) return r;     // captures this shape's graph
    if ((r = tcs_restore(c))) return r;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return set_err(TCS_ERR_CUDA, "tuning events");
    }
    cudaEventRecord(e0, c->stream);
    r = tcs_step(c, steps, &done);
    cudaEventRecord(e1, c->stream);
    const bool ok = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(ms, e0, e1) == cudaSuccess;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r == TCS_ERR_BLOWUP) r = TCS_OK;
    return (r == TCS_OK && !ok) ? set_err(TCS_ERR_CUDA, "tuning trial timing") : r;
}

extern "C" int tcs_autotune(tcs_ctx *c, int trial_steps, const char *cache_path, int *from_cache)
{
    if (!c) return set_err(TCS_ERR_ARG, "null context");
    if (trial_steps < 1) return set_err(TCS_ERR_ARG, "trial_steps must be >= 1");
    cudaSetDevice(c->cfg.device);
    if (from_cache) *from_cache = 0;
    const TuneKey key{c->cfg.n1m, c->cfg.n2m, c->cfg.n3m, c->cfg.precision};
    const std::string path = cache_path ? cache_path : "";
    std::vector<int> best;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_load(path);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) best = it->second;
    }
    int r;
    if (!best.empty()) {
        for (int k = 0; k < TCS_TUNE_COUNT; k++)
            if (best[k] && (r = tcs_set_tuning(c, k, best[k]))) return r;
        if (from_cache) *from_cache = 1;
        return TCS_OK;
    }
    if (c->probe.mask) return set_err(TCS_ERR_ARG, "disable the probes before tuning");
    if ((r = tcs_snapshot(c))) return r;
    best.resize(TCS_TUNE_COUNT);
    for (int k = 0; k < TCS_TUNE_COUNT; k++) tcs_get_tuning(c, k, &best[k]);
    float best_ms = 0.0f;
    if ((r = tune_trial(c, trial_steps, &best_ms))) return r;
    static const int cand[] = {1, 2, 4, 8, 16, 32};
    for (int k = 0; k < TCS_TUNE_COUNT; k++) {
        for (int v : cand) {
            if (v == best[k]) continue;
            if (tcs_set_tuning(c, k, v) != TCS_OK) continue;          // not valid for this shape
            float ms = 0.0f;
            if ((r = tune_trial(c, trial_steps, &ms))) return r;
            if (ms < best_ms) { best_ms = ms; best[k] = v; }
        }
        if ((r = tcs_set_tuning(c, k, best[k]))) return r;
    }
    if ((r = tcs_restore(c))) return r;
    CK(cudaStreamSynchronize(c->stream));
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    if (!path.empty()) {
        std::ofstream out(path, std::ios::app);
        out << key.n1 << ' ' << key.n2 << ' ' << key.n3 << ' ' << key.prec;
        for (int v : best) out << ' ' << v;
        out << '\n';
    }
    return TCS_OK;
}

// ---------------------------------------------------------------------------
// PaScaL_TDMA single-system and nonblocking entry points
// (pascal_tdma.f90:139-175, 301-475, 590-703, 818-930).  On one rank the
// single-system solve is the many-system solve with n_sys = 1 (tdma_single
// and tdma_cycl_single of tdmas.f90:27-100 do the many versions' arithmetic
// on the 2-row reduced system), and the nonblocking variants differ only in
// their MPI calls, so all of them run the same kernel.
// ---------------------------------------------------------------------------
extern "C" {

int tcs_tdma_plan_single_create(tcs_tdma_plan **plan, int myrank, int nprocs, int gather_rank)
{
    if (gather_rank != 0) return set_err(TCS_ERR_UNSUPPORTED, "one GPU holds the whole line: gather_rank must be 0");
    return tcs_tdma_plan_many_create(plan, 1, myrank, nprocs);
}

int tcs_tdma_plan_single_destroy(tcs_tdma_plan *p) { return tcs_tdma_plan_many_destroy(p); }

int tcs_tdma_single_solve(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_row)
{
    return tdma_solve(p, A, B, C, D, 1, n_row, 0);
}

int tcs_tdma_single_solve_cycle(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_row)
{
    return tdma_solve(p, A, B, C, D, 1, n_row, 1);
}

int tcs_tdma_many_solve_nonblocking(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    return tdma_solve(p, A, B, C, D, n_sys, n_row, 0);
}

int tcs_tdma_many_solve_cycle_nonblocking(tcs_tdma_plan *p, double *A, double *B, double *C, double *D, int n_sys, int n_row)
{
    return tdma_solve(p, A, B, C, D, n_sys, n_row, 1);
}

} // extern "C"

// ---------------------------------------------------------------------------
// Restart files and planes from the device.
//
// tcs_write_continue / tcs_read_continue write and read the reference's
// continue files (module_post.f90:1264-1454: cont_time.bin = time, dt;
// cont_U/V/W/P/THETA.bin = the n1m x n2m x n3m interior, i fastest, FP64,
// the names the reference's writer and reader use, :1336 and :1443) by
// k-slabs through one device staging chunk and one pinned host chunk, and add
// cont_dPhat.bin and cont_dP0.bin, which the reference does not save, so that
// a resumed run continues bit for bit.  tcs_extract_plane copies one padded
// plane of chosen fields to the host (the instant-field planes of
// module_post.f90:270-361) without moving the rest of the field.
// ---------------------------------------------------------------------------
static int io_chunk(tcs_ctx *c, size_t n)
{
    if (n <= c->io_cap) return TCS_OK;
    if (c->io_host) { cudaFreeHost(c->io_host); c->io_host = nullptr; }
    int r = dalloc(c, &c->io_dev, n);
    if (r) return r;
    if (cudaMallocHost(&c->io_host, n * sizeof(double)) != cudaSuccess) return set_err(TCS_ERR_NOMEM, "pinned IO buffer");
    c->io_cap = n;
    return TCS_OK;
}

static const struct { int field; const char *name; } k_cont[] = {
    {TCS_F_U, "cont_U.bin"}, {TCS_F_V, "cont_V.bin"}, {TCS_F_W, "cont_W.bin"}, {TCS_F_P, "cont_P.bin"},
    {TCS_F_T, "cont_THETA.bin"}, {TCS_F_DPHAT, "cont_dPhat.bin"}, {TCS_F_DP0, "cont_dP0.bin"}};
// Temperature files written by earlier versions of this library, read when
// cont_THETA.bin is absent.
static const char *const k_cont_T_legacy = "cont_T.bin";

static std::string join_path(const char *dir, const char *name)
{
    std::string d = dir ? dir : "";
    if (!d.empty() && d.back() != '/') d += '/';
    return d + name;
}

extern "C" {

int tcs_write_continue(tcs_ctx *c, const char *dir)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    const GridT<double> &g = c->cx.g;
    const int ks = std::max(1, (int)((size_t)(4u << 20) / ((size_t)g.N1 * g.N2)));
    if ((r = io_chunk(c, (size_t)g.N1 * g.N2 * ks))) return r;
    double sc[S_NSCAL];
    CK(cudaMemcpyAsync(sc, g.scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    {
        FILE *fp = std::fopen(join_path(dir, "cont_time.bin").c_str(), "wb");
        if (!fp) return set_err(TCS_ERR_ARG, "cannot open cont_time.bin for writing");
        const double td[2] = {sc[S_TIME], sc[S_DT]};
        const bool ok = std::fwrite(td, sizeof(double), 2, fp) == 2;
        std::fclose(fp);
        if (!ok) return set_err(TCS_ERR_ARG, "short write of cont_time.bin");
    }
    for (const auto &cf : k_cont) {
        FILE *fp = std::fopen(join_path(dir, cf.name).c_str(), "wb");
        if (!fp) return set_err(TCS_ERR_ARG, std::string("cannot open ") + cf.name + " for writing");
        bool ok = true;
        for (int k0 = 1; k0 <= g.N3 && ok; k0 += ks) {
            const int nk = std::min(ks, g.N3 - k0 + 1);
            const size_t n = (size_t)g.N1 * g.N2 * nk;
            on_ctx(c, [&](auto &x) { launch_pack(x, field_ptr_t(x.f, cf.field), lo_ptr_t(x.f, cf.field), c->io_dev, k0, nk, c->stream); });
            if ((r = take_launch_error())) { std::fclose(fp); return r; }
            if (cudaMemcpyAsync(c->io_host, c->io_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess) { std::fclose(fp); return set_err(TCS_ERR_CUDA, "continue-file copy"); }
            ok = std::fwrite(c->io_host, sizeof(double), n, fp) == n;
        }
        std::fclose(fp);
        if (!ok) return set_err(TCS_ERR_ARG, std::string("short write of ") + cf.name);
    }
    return TCS_OK;
}

int tcs_read_continue(tcs_ctx *c, const char *dir, int *with_pressure_history)
{
    ENTER(c);
    int r = flush_pending(c);
    if (r) return r;
    const GridT<double> &g = c->cx.g;
    const int ks = std::max(1, (int)((size_t)(4u << 20) / ((size_t)g.N1 * g.N2)));
    if ((r = io_chunk(c, (size_t)g.N1 * g.N2 * ks))) return r;
    double td[2];
    {
        FILE *fp = std::fopen(join_path(dir, "cont_time.bin").c_str(), "rb");
        if (!fp) return set_err(TCS_ERR_ARG, "cannot open cont_time.bin");
        const bool ok = std::fread(td, sizeof(double), 2, fp) == 2;
        std::fclose(fp);
        if (!ok) return set_err(TCS_ERR_ARG, "cont_time.bin is short");
    }
    int history = 1;
    const size_t want = (size_t)g.N1 * g.N2 * g.N3;
    for (const auto &cf : k_cont) {
        FILE *fp = std::fopen(join_path(dir, cf.name).c_str(), "rb");
        if (!fp && cf.field == TCS_F_T) fp = std::fopen(join_path(dir, k_cont_T_legacy).c_str(), "rb");
        const bool optional = cf.field == TCS_F_DPHAT || cf.field == TCS_F_DP0;
        if (!fp) {
            if (optional) { history = 0; continue; }
            return set_err(TCS_ERR_ARG, std::string("cannot open ") + cf.name);
        }
        std::fseek(fp, 0, SEEK_END);
        const long sz = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        if (sz != (long)(want * sizeof(double))) { std::fclose(fp); return set_err(TCS_ERR_ARG, std::string(cf.name) + " does not hold n1m*n2m*n3m doubles"); }
        for (int k0 = 1; k0 <= g.N3; k0 += ks) {
            const int nk = std::min(ks, g.N3 - k0 + 1);
            const size_t n = (size_t)g.N1 * g.N2 * nk;
            if (std::fread(c->io_host, sizeof(double), n, fp) != n) { std::fclose(fp); return set_err(TCS_ERR_ARG, std::string("short read of ") + cf.name); }
            if (cudaMemcpyAsync(c->io_dev, c->io_host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
                std::fclose(fp); return set_err(TCS_ERR_CUDA, "continue-file copy");
            }
            on_ctx(c, [&](auto &x) {
                auto *d2 = cf.field == TCS_F_T ? x.f.Tn : nullptr;
                launch_unpack(x, c->io_dev, field_ptr_t(x.f, cf.field), d2, lo_ptr_t(x.f, cf.field), k0, nk, c->stream);
            });
            if ((r = take_launch_error())) { std::fclose(fp); return r; }
            CK(cudaStreamSynchronize(c->stream));     // the pinned chunk is refilled next
        }
        std::fclose(fp);
        c->ghost_ok &= ~(1u << cf.field);
    }
    CK(cudaMemcpyAsync(g.scal + S_TIME, &td[0], sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(g.scal + S_DT, &td[1], sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (with_pressure_history) *with_pressure_history = history;
    return TCS_OK;
}

int tcs_extract_plane(tcs_ctx *c, int axis, int index, int nfields, const int *fields, double *out)
{
    ENTER(c);
    if (axis < 1 || axis > 3 || nfields < 1 || !fields || !out) return set_err(TCS_ERR_ARG, "bad plane arguments");
    const GridT<double> &g = c->cx.g;
    const int P3 = g.N3 + 2, lim = axis == 1 ? g.P1 : (axis == 2 ? g.P2 : P3);
    if (index < 0 || index >= lim) return set_err(TCS_ERR_ARG, "plane index outside the padded range");
    int r = flush_pending(c);
    if (r) return r;
    const size_t n = (size_t)(axis == 1 ? g.P2 : g.P1) * (axis == 3 ? g.P2 : P3);
    if ((r = io_chunk(c, n))) return r;
    for (int q = 0; q < nfields; q++) {
        if (fields[q] < 0 || fields[q] >= TCS_F_MU) return set_err(TCS_ERR_ARG, "unknown field");
        on_ctx(c, [&](auto &x) { launch_plane(x, field_ptr_t(x.f, fields[q]), lo_ptr_t(x.f, fields[q]), c->io_dev, axis, index, c->stream); });
        if ((r = take_launch_error())) return r;
        CK(cudaMemcpyAsync(out + q * n, c->io_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return TCS_OK;
}

} // extern "C"
