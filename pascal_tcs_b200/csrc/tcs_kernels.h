// tcs_kernels.h -- host-side view of one case (Ctx), kernel identifiers and
// the launch helpers shared by the stage files.
#pragma once

#include "tcs_fields.cuh"

#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

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
    FastDiv dnb[24], dns[24];   // per pass: n / radix and the span Ns
    FastDiv dn, dh;             // n and n/2 + 1
};

// A block's z-FFT lines in shared memory: element (line l, row q) of NL lines at
// (q + q/8) NL + l -- lines fastest, so that the threads of a warp, which take
// consecutive lines and then consecutive butterflies, touch consecutive
// words; the pad row after every 8 rows spreads the strided writes of a pass
// with span 1 over the banks.
__host__ __device__ __forceinline__ int frow(int q) { return q + (q >> 3); }
__host__ __device__ __forceinline__ size_t fft_buf_elems(int NL, int n) { return (size_t)NL * (size_t)frow(n); }

// The form of a z transform of NL lines per block: 1 the one-radix form (every
// pass of radix 4 or 8, one butterfly per thread: NL n / radix <= 1024 threads,
// one buffer), 2 the general form (256 threads, two buffers), 0 neither fits
// the 227 KB a block may take.
inline size_t fftz_smem(const FFTPlan &fp, int NL, int form) { return (size_t)form * fft_buf_elems(NL, fp.n) * 16; }
inline int fftz_form(const FFTPlan &fp, int NL)
{
    bool uni = fp.npass >= 1 && (fp.radix[0] == 8 || fp.radix[0] == 4);
    for (int p = 1; p < fp.npass; p++) uni = uni && fp.radix[p] == fp.radix[0];
    if (uni && (long long)NL * (fp.n / fp.radix[0]) <= 1024 && fftz_smem(fp, NL, 1) <= 227 * 1024) return 1;
    return fftz_smem(fp, NL, 2) <= 227 * 1024 ? 2 : 0;
}

// The form of the inverse x transform of NL lines per block: 1 the one-radix
// form (fpu of one radix 4 or 8, packed lines x N1 / radix <= 512 threads, one
// line-major buffer), 2 the general form (256 threads, two buffers, the
// radix-4 plan), 0 neither fits.
inline size_t ifftx_smem(const FFTPlan &fpu, int NL, int form)
{
    const size_t nfl = (size_t)((NL + 1) / 2);
    return form == 1 ? nfl * (size_t)frow(fpu.n) * 16 : nfl * (size_t)fpu.n * 2 * 16;
}
inline int ifftx_form(const FFTPlan &fpu, int NL)
{
    bool uni = fpu.npass >= 1 && (fpu.radix[0] == 8 || fpu.radix[0] == 4);
    for (int p = 1; p < fpu.npass; p++) uni = uni && fpu.radix[p] == fpu.radix[0];
    if (uni && (long long)((NL + 1) / 2) * (fpu.n / fpu.radix[0]) <= 512 && ifftx_smem(fpu, NL, 1) <= 227 * 1024) return 1;
    return ifftx_smem(fpu, NL, 2) <= 227 * 1024 ? 2 : 0;
}

struct ProbeState;   // CUDA-event probes (tcs_capi.cu)

// Launch shapes shared by both forms.
struct Shapes {
    int tl_strided, tl_contig, tl_modal;
    int fft_lines_x, fft_lines_z;
    int ifft_lines_x;                            // lines per block of the inverse x transform
    int lanes;                                   // at most this many partitions (lanes) per line
    int long_lines;                              // one-block-per-SM form of long lines: 1 never, 2 z sweeps, 4 z and y sweeps
    int y_solver;                                // y lines: 1 partitioned (line_block), 2 one line per thread for the y sweeps, 4 also the modal solves
    double *thomas_scr;                          // c', d' of the one-line-per-thread solver (null unless y_solver asks for it)
    int mixed_rows;                              // FP32-mixed form: 1 FP32 elimination + refinement, 2 FP64 rows in the x sweeps, 4 x and z sweeps, 8 z at 3 blocks/SM
    int z_staging;                               // FP64 dw_z: 1 loads from global memory, 2 inputs staged by TMA
    FFTPlan fp1, fp3;
    FFTPlan fp1u;                                // N1 with radices up to 8 (the inverse x transform's one-radix form)
    int h1p;
    double wall_ab, wall_bb, wall_at, wall_bt;   // Pbc_a, Pbc_b of the two walls
    ProbeState *probe;
};

template <class R>
struct Ctx : Shapes {
    GridT<R> g;
    FieldsT<R> f;
};

LinePlan make_line_plan(int n, bool cyclic, int TL, int pmax = 32);
bool make_fft_plan(int n, FFTPlan &fp, int maxr);   // radices 2, 3, 4, 5 and (maxr >= 8) 8
void probe_begin(const Shapes &cx, int kid, cudaStream_t s);
void probe_end(const Shapes &cx, int kid, cudaStream_t s);
int record_launch_error(const char *what);
int set_error(int code, const std::string &msg);

// Dynamic shared memory of a line-solver launch.
template <class Prob>
inline size_t line_smem(const LinePlan &lp)
{
    return (size_t)line_words<Prob>() * lp.TL * lp.LS * sizeof(typename Prob::Real) + (size_t)lp.n * sizeof(int);
}

// The plan of a line problem: make_line_plan's partitions, and for the
// unpaired, non-cyclic strided problems (the y sweeps and the modal solves) a
// line stride LS chosen for the build and the emission, where one warp
// touches TL lines x 32/TL rows: LS = banks/TL (mod banks), banks = 32
// four-byte words (FP32 rows) or 16 eight-byte words per half-warp (FP64
// rows), puts those accesses on distinct banks.  The solve (one line per
// warp) only uses the odd partition stride PS.  Measured at 256^3: the y
// sweeps 2-5% and the modal solves 3-4% faster in both forms.  The unpaired
// cyclic (FP32 z) sweeps keep the odd LS: the longer stride takes three of
// their blocks past the 196 KB shared-memory configuration into the 228 KB
// one, whose 28 KB of L1 (against 60 KB) cost their stencil loads 11-43%.
// The paired builds step rows by 2, where no LS avoids 2-way conflicts; they
// keep the odd LS too.
template <class Prob>
inline LinePlan plan_for(int n, bool cyclic, int tl, int pmax)
{
    LinePlan lp = make_line_plan(n, cyclic, tl, pmax);
    if (!Prob::CONTIG && !PairRows<Prob>::on && !cyclic && tl > 1) {
        const int banks = sizeof(typename Prob::Real) == 4 ? 32 : 16;
        const int want = tl < banks ? banks / tl : 1;
        const int ls = lp.P * lp.PS;
        lp.LS = ls + ((want - ls) % banks + banks) % banks;
    }
    return lp;
}

// The shared memory (KiB) a line family lets its blocks take per SM: all of
// it (228 KiB) by default, less for the one-block-per-SM form of long lines
// (LongLines), whose stencil builds need the L1 that the rest leaves.
template <class P, class = void>
struct SmemKiB { static constexpr int v = 228; };
template <class P>
struct SmemKiB<P, std::void_t<decltype(P::SMEM_KIB)>> { static constexpr int v = P::SMEM_KIB; };

// Lines per block: the requested count, halved until MINB blocks fit in the
// family's share of the SM's shared memory (1 KB reserved per block);
// extra: static shared memory the kernel adds per block.
template <class Prob>
inline int fit_tl(int n, bool cyclic, int want, int pmax, size_t extra = 0)
{
    const size_t budget = (size_t)SmemKiB<Prob>::v * 1024 / Prob::MINB - 1024 - extra;
    int tl = want;
    while (tl > 1 && line_smem<Prob>(plan_for<Prob>(n, cyclic, tl, pmax)) > budget) tl /= 2;
    return tl;
}

// Opt a kernel in to smem bytes of dynamic shared memory on the current
// device.  The attribute belongs to the function on each device, so the
// largest size set so far is kept per device (cache: one entry per ordinal).
inline void smem_opt_in(const void *fn, size_t smem, size_t *cache)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (smem > cache[dev]) {
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cache[dev] = smem;
    }
}

template <class Prob>
inline void launch_lines(const Prob &p, const LinePlan &lp, dim3 grid, cudaStream_t s, int kid, const Shapes &cx)
{
    const size_t smem = line_smem<Prob>(lp);
    static size_t configured[64] = {};
    smem_opt_in((const void *)line_solve_kernel<Prob>, smem, configured);
    probe_begin(cx, kid, s);
    line_solve_kernel<Prob><<<grid, Prob::NT, smem, s>>>(p, lp);
    probe_end(cx, kid, s);
    record_launch_error(kernel_name(kid));
}

// The SM's unified L1/shared-memory configurations: the shared-memory share
// (KiB) the driver picks for a given demand per SM; the L1 keeps the rest of
// the 256 KiB.
inline int smem_config_kib(size_t per_sm_bytes)
{
    static const int cfg[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
    for (int c : cfg)
        if ((size_t)c * 1024 >= per_sm_bytes) return c;
    return 228;
}

// A line family in one block per SM: the same warps per SM (NT x MINB threads
// in one block, so the same registers per thread) with its lines per block
// fitted to 132 KiB of shared memory, which leaves the SM 124 KiB of L1.  The
// z-sweep builds read every input through L1 about three times (their x and z
// neighbours come from other threads' cells): measured on B200, forcing their
// 256^3 blocks into the 228 KiB configuration (28 KiB of L1) made them 1.8x
// slower, and 512-row lines put them there by themselves (two blocks of 8
// lines x 512 rows need 213 KiB).
template <class P>
struct LongLines : P {
    static constexpr int NT = P::NT * P::MINB;
    static constexpr int MINB = 1;
    static constexpr int SMEM_KIB = 132;
};

// A strided line sweep (z or y lines: TL consecutive i per block, gy block
// rows).  With allow_long, the one-block-per-SM form runs instead where the
// usual form would leave less than 60 KiB of L1 or would have to halve its
// lines per block.  make(tl) builds the problem for tl lines per block.
template <class P, class Make>
inline void launch_strided(const Shapes &cx, int n, bool cyclic, int nlines, int gy, Make make, cudaStream_t s, int kid,
                           bool allow_long)
{
    const LinePlan a = plan_for<P>(n, cyclic, fit_tl<P>(n, cyclic, cx.tl_strided, cx.lanes), cx.lanes);
    if (allow_long) {
        using L = LongLines<P>;
        const LinePlan b = plan_for<L>(n, cyclic, fit_tl<L>(n, cyclic, cx.tl_strided, cx.lanes), cx.lanes);
        const size_t per_sm = (size_t)P::MINB * (line_smem<P>(a) + 1024);
        const int l1_kib = 256 - smem_config_kib(per_sm);
        if (b.TL > a.TL || l1_kib < 60) {
            launch_lines(L{make(b.TL)}, b, dim3((nlines + b.TL - 1) / b.TL, gy), s, kid, cx);
            return;
        }
    }
    launch_lines(make(a.TL), a, dim3((nlines + a.TL - 1) / a.TL, gy), s, kid, cx);
}

// An FP32 line problem whose rows are eliminated in FP64 (Shapes::mixed_rows):
// the problem's own build in the field type, its coefficients widened to FP64
// in shared memory, the partitioned solve in FP64 without the refinement pass
// (Refine<double> is off), and the solution rounded once to the field type when
// the problem emits it.  Launch shape of the FP64 family of the same axis
// (AX: 0 the z sweeps, 1 the x sweeps), or for the z sweeps with Z3 three
// blocks per SM and the shared-memory elimination (their FP32 builds need
// fewer registers than FP64 ones: measured at 256^3 9% faster than the FP64
// shape, at 512^3 3% slower).
template <class P, int AX, int Z3 = 0>
struct FP64Rows : P {
    using Real = double;
    static constexpr int MINB = AX ? LineOcc<double>::x : (Z3 ? 3 : LineOcc<double>::z);
    static constexpr int MREG = AX ? LineOcc<double>::reg_x : (Z3 ? 0 : LineOcc<double>::reg_z);
    static constexpr int NT = AX ? LineOcc<double>::nt_x : LineOcc<double>::nt_z;
    __device__ Coef<double, P::NRHS> build(int l, int r, const typename P::State &st) const
    {
        const auto c = P::build(l, r, st);
        Coef<double, P::NRHS> d;
        d.a = c.a; d.b = c.b; d.c = c.c;
#pragma unroll
        for (int q = 0; q < P::NRHS; q++) d.d[q] = c.d[q];
        return d;
    }
    __device__ void emit(int l, int r, const double *x, const typename P::State &st) const
    {
        typename P::Real xr[P::NRHS];
#pragma unroll
        for (int q = 0; q < P::NRHS; q++) xr[q] = (typename P::Real)x[q];
        P::emit(l, r, xr, st);
    }
};

// Lines per block of the one-line-per-thread solver (thomas_line_kernel).
constexpr int THOMAS_TL = 128;

// Doubles of c', d' scratch the one-line-per-thread solver needs for nlines
// lines of n rows in gy block rows with nrhs right-hand sides.
inline size_t thomas_words(int n, int nlines, int gy, int nrhs)
{
    return (size_t)(1 + nrhs) * n * ((size_t)(nlines + THOMAS_TL - 1) / THOMAS_TL) * THOMAS_TL * gy;
}

template <class P, class Make>
inline void launch_thomas(const Shapes &cx, int n, int nlines, int gy, Make make, cudaStream_t s, int kid)
{
    probe_begin(cx, kid, s);
    thomas_line_kernel<P><<<dim3((nlines + THOMAS_TL - 1) / THOMAS_TL, gy), THOMAS_TL, 0, s>>>(make(THOMAS_TL), n, cx.thomas_scr);
    probe_end(cx, kid, s);
    record_launch_error(kernel_name(kid));
}

// A z sweep (cyclic strided lines, nlines x gy of n rows): in the FP32-mixed
// form with mixed_rows 4 (8: three blocks per SM) its FP32-built rows are
// eliminated in FP64.
template <class P, class Make>
inline void launch_z(const Shapes &cx, int n, int nlines, int gy, Make make, cudaStream_t s, int kid)
{
    if constexpr (std::is_same<typename P::Real, float>::value) {
        if (cx.mixed_rows >= 8) {
            using Q = FP64Rows<P, 0, 1>;
            launch_strided<Q>(cx, n, true, nlines, gy, [&](int tl) { return Q{make(tl)}; }, s, kid, cx.long_lines >= 2);
            return;
        }
        if (cx.mixed_rows >= 4) {
            using Q = FP64Rows<P, 0>;
            launch_strided<Q>(cx, n, true, nlines, gy, [&](int tl) { return Q{make(tl)}; }, s, kid, cx.long_lines >= 2);
            return;
        }
    }
    launch_strided<P>(cx, n, true, nlines, gy, make, s, kid, cx.long_lines >= 2);
}

// A y sweep (non-cyclic strided lines, nlines x gy of n rows): the
// one-line-per-thread solver when the knob asks for it (y_solver 2 or 4,
// scratch allocated), else the partitioned line solver, in the
// one-block-per-SM form where long_lines asks for it for the y sweeps.
template <class P, class Make>
inline void launch_y(const Shapes &cx, int n, int nlines, int gy, Make make, cudaStream_t s, int kid)
{
    if (cx.y_solver >= 2 && cx.thomas_scr) {
        launch_thomas<P>(cx, n, nlines, gy, make, s, kid);
        return;
    }
    launch_strided<P>(cx, n, false, nlines, gy, make, s, kid, cx.long_lines >= 4);
}

// ---------------------------------------------------------------------------
// Ensemble launches: one line stage of many cases as line_solve_multi
// launches of up to MultiParams::K cases each.  An ensemble builds each
// step's launches twice in the same order: in planning mode every launch
// reserves its item counter in the arena, then (after one upload of the
// arena) in launch mode each launch takes its counter's device address.
// The launches of one stage run concurrently on the aux streams (forked from
// and joined back to the stage's stream).
// ---------------------------------------------------------------------------
struct MultiArena {
    std::vector<unsigned char> host;
    unsigned char *dev = nullptr;
    size_t cursor = 0;
    bool planning = true;
    std::vector<cudaStream_t> aux;       // streams for a stage's second and later launches
    std::vector<cudaEvent_t> join;       // one per aux stream
    cudaEvent_t fork = nullptr;
    int *counter()
    {
        const size_t off = (cursor + 15) & ~(size_t)15;
        cursor = off + 16;
        if (planning) {
            host.resize(cursor, 0);
            return nullptr;
        }
        return (int *)(dev + off);
    }
};

// One case's share of a multi-case line stage: the line length, cyclicity,
// requested lines per block, and the block grid (lines / TL rounded up, gy).
struct StageShape {
    int n;
    bool cyclic;
    int want, lines, gy;
};

template <class Prob>
inline void launch_lines_multi(MultiParams<Prob> &mp, int ncase, cudaStream_t s, const char *what)
{
    size_t smem = 0;
    for (int c = 0; c < ncase; c++) smem = std::max(smem, line_smem<Prob>(mp.lp[c]));
    static size_t conf[64] = {};
    smem_opt_in((const void *)line_solve_multi<Prob>, smem, conf);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, line_solve_multi<Prob>, Prob::NT, smem);
    const int grid = (int)std::min<long long>(mp.nitems, (long long)std::max(occ, 1) * sms);
    line_solve_multi<Prob><<<grid, Prob::NT, smem, s>>>(mp);
    record_launch_error(what);
}

// A line stage for a group of same-precision cases: per case the same plan
// and block grid as its one-case launch; the cases with the longest blocks
// first (so the blocks that pull the last items finish close together),
// MultiParams::K cases per launch.
template <class P, class R, class Shape, class Make>
inline void multi_stage(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s, const char *what, Shape shape,
                        Make make)
{
    struct Entry { P prob; LinePlan lp; int gx, gy; long long cost; };
    std::vector<Entry> es;
    for (const Ctx<R> *xp : cs) {
        const Ctx<R> &x = *xp;
        const StageShape sh = shape(x);
        const LinePlan lp = plan_for<P>(sh.n, sh.cyclic, fit_tl<P>(sh.n, sh.cyclic, sh.want, x.lanes, 64), x.lanes);
        es.push_back({make(x, lp.TL), lp, (sh.lines + lp.TL - 1) / lp.TL, sh.gy, (long long)sh.n * lp.TL});
    }
    std::stable_sort(es.begin(), es.end(), [](const Entry &a, const Entry &b) { return a.cost > b.cost; });
    constexpr int K = MultiParams<P>::K;
    const int nl = (int)((es.size() + K - 1) / K);
    const bool fan = !A.planning && nl > 1 && (int)A.aux.size() >= nl - 1;
    if (fan) cudaEventRecord(A.fork, s);
    for (int l = 0; l < nl; l++) {
        const size_t c0 = (size_t)l * K;
        const int nc = (int)std::min<size_t>(K, es.size() - c0);
        int *ctr = A.counter();
        if (A.planning) continue;
        MultiParams<P> mp;
        mp.start[0] = 0;
        for (int c = 0; c < nc; c++) {
            const Entry &e = es[c0 + c];
            mp.p[c] = e.prob;
            mp.lp[c] = e.lp;
            mp.gx[c] = e.gx;
            mp.start[c + 1] = mp.start[c] + e.gx * e.gy;
        }
        mp.nitems = mp.start[nc];
        mp.ctr = ctr;
        cudaStream_t ls = s;
        if (fan && l > 0) {
            ls = A.aux[l - 1];
            cudaStreamWaitEvent(ls, A.fork, 0);
        }
        launch_lines_multi(mp, nc, ls, what);
        if (fan && l > 0) {
            cudaEventRecord(A.join[l - 1], ls);
            cudaStreamWaitEvent(s, A.join[l - 1], 0);
        }
    }
}

// Whether a case runs its x sweeps in the wide shape (the rule of launch_x).
template <template <class, int, int> class X, class R>
inline bool x_is_wide(const Ctx<R> &cx)
{
    if constexpr (LineOcc<R>::f32) return fit_tl<X<R, 0, 0>>(cx.g.N1, true, cx.tl_contig, cx.lanes) < 4;
    return false;
}

// A multi-case x sweep: the cases split by shape, one launch per shape.
template <template <class, int, int> class X, class R, class Lines>
inline void multi_x(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s, const char *what, Lines lines)
{
    std::vector<Ctx<R> *> narrow, wide;
    for (Ctx<R> *c : cs) (x_is_wide<X>(*c) ? wide : narrow).push_back(c);
    auto shape = [&](const Ctx<R> &x) { return StageShape{x.g.N1, true, x.tl_contig, lines(x), x.g.N3}; };
    multi_stage<X<R, 0, 1>>(narrow, A, s, what, shape, [](const Ctx<R> &x, int tl) { return X<R, 0, 1>{x.g, x.f, tl}; });
    if constexpr (LineOcc<R>::f32)
        multi_stage<X<R, 1, 1>>(wide, A, s, what, shape, [](const Ctx<R> &x, int tl) { return X<R, 1, 1>{x.g, x.f, tl}; });
}

// An x sweep: lines along i, one block row per (j-range, k).  FP32 runs the
// 128-thread shape when at least 4 lines fit a block, else the wide shape;
// with mixed_rows >= 2 the FP32-built rows are eliminated in FP64 instead.
template <template <class, int, int> class X, class R>
inline void launch_x(const Ctx<R> &cx, int nlines, cudaStream_t s, int kid)
{
    const GridT<R> &g = cx.g;
    if constexpr (LineOcc<R>::f32) {
        if (cx.mixed_rows >= 2) {   // FP32-built rows eliminated in FP64
            using P = FP64Rows<X<R, 0, 0>, 1>;
            const LinePlan p = make_line_plan(g.N1, true, fit_tl<P>(g.N1, true, cx.tl_contig, cx.lanes), cx.lanes);
            launch_lines(P{X<R, 0, 0>{g, cx.f, p.TL}}, p, dim3((nlines + p.TL - 1) / p.TL, g.N3), s, kid, cx);
            return;
        }
    }
    const int tl = fit_tl<X<R, 0, 0>>(g.N1, true, cx.tl_contig, cx.lanes);
    if constexpr (LineOcc<R>::f32) {
        if (tl < 4) {
            const LinePlan p = make_line_plan(g.N1, true, fit_tl<X<R, 1, 0>>(g.N1, true, cx.tl_contig, cx.lanes), cx.lanes);
            launch_lines(X<R, 1, 0>{g, cx.f, p.TL}, p, dim3((nlines + p.TL - 1) / p.TL, g.N3), s, kid, cx);
            return;
        }
    }
    const LinePlan p = make_line_plan(g.N1, true, tl, cx.lanes);
    launch_lines(X<R, 0, 0>{g, cx.f, p.TL}, p, dim3((nlines + p.TL - 1) / p.TL, g.N3), s, kid, cx);
}

// Stage launchers (one per reference routine or fused group), instantiated
// for R = double and R = float.
template <class R> void launch_thermal(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_momentum_coeffi(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_solve_du(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_solve_dv(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_solve_dw(const Ctx<R> &cx, cudaStream_t s);
bool dwz_staging_possible(const Ctx<double> &cx);   // the TMA-staged dw_z can run this case
template <class R> void launch_blockld_v(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_blockld_u(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_pseudo_update(const Ctx<R> &cx, cudaStream_t s);   // standalone (Un = U + dU, ...)
template <class R> void launch_pseudo_prhs_fftx(const Ctx<R> &cx, cudaStream_t s, bool with_pseudo);
template <class R> void launch_poisson_rest(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_modal(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_poisson_fwd(const Ctx<R> &cx, cudaStream_t s);   // z FFTs (forward)
template <class R> void launch_poisson_back(const Ctx<R> &cx, cudaStream_t s);  // mean, z and x inverse FFTs, dP walls
template <class R> void launch_projection(const Ctx<R> &cx, cudaStream_t s);
template <class R> void launch_post(const Ctx<R> &cx, cudaStream_t s, int record_hist);
template <class R> void launch_ghost(const Ctx<R> &cx, R *a, cudaStream_t s);
// the line stages of a step for a group of same-precision cases, one launch per stage
template <class R> void launch_thermal_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s);
template <class R> void launch_momentum_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s);
template <class R> void launch_modal_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s);
template <class R> void launch_convert(const R *src, double *dst, long long n, cudaStream_t s);   // field -> FP64 staging
template <class R> void launch_convert_in(const double *src, R *dst, long long n, cudaStream_t s); // FP64 staging -> field
void launch_join(const float *hi, const float *lo, double *dst, long long n, cudaStream_t s);       // FP32 pair -> FP64 staging
template <class R> void launch_pack(const Ctx<R> &cx, const R *src, const R *lo, double *dst, int k0, int nk, cudaStream_t s);
template <class R> void launch_unpack(const Ctx<R> &cx, const double *src, R *dst, R *dst2, R *lo, int k0, int nk, cudaStream_t s);
template <class R> void launch_plane(const Ctx<R> &cx, const R *src, const R *lo, double *dst, int axis, int index, cudaStream_t s);
void launch_split(const double *src, float *hi, float *lo, long long n, cudaStream_t s);          // FP64 staging -> FP32 pair

} // namespace tcs
