// tcs_device.cuh -- device-side building blocks shared by every kernel of the
// PaScaL_TCS time step on one B200 (sm_100a).
//
// Layout: every 3-D field is one padded array (0:N1+1, 0:N2+1, 0:N3+1) with i
// fastest, exactly the reference's Fortran arrays (0:n1sub, 0:n2sub, 0:n3sub)
// on one rank, so host<->device copies are plain memcpys.
//
// Two numerical forms share the code through the field type R:
//   R = double  FP64 plain, the reference's arithmetic;
//   R = float   FP32-mixed: fields stored in FP32, stencils, ADI sweeps and
//               FFTs in FP32 with one FP64-residual refinement pass per
//               tridiagonal system; modal pressure solves, the divergence of
//               the pressure right-hand side, the projection and all
//               reductions in FP64 arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace tcs {

// ---------------------------------------------------------------------------
// Metric tables of one direction (length n+2, index 0..n+1), as computed by
// mpi_subdomain_mesh (module_mpi_subdomain.f90:153-299), plus reciprocals.
// ---------------------------------------------------------------------------
template <class R>
struct MetricT {
    const R *dx, *dmx;       // dx_sub, dmx_sub
    const R *rdx, *rdmx;     // 1/dx, 1/dmx (0 where dx or dmx is 0)
};

// Physical constants of module_global (module_global.f90:107-141) and the
// property polynomial coefficients (water/glycerol/constant).  Every member
// is of type R, so the host converts the FP64 set member by member.
template <class R>
struct PhysT {
    R Cmu, Cmt, Ct, Cmp, DeltaT, a12pera11;
    R a10, a11, a12, a13, a14, a15;
    R b10, b11, b12, b13, b14, b15;
    R c10, c11, c12, c13, c14, c15;
    R d10, d11, d12, d13, d14, d15;
    R KPP0, Rho0, Cp0, Mu0;
    R Tup, Tbt, Uup, Ubt, Vup, Vbt, Wup, Wbt;
    R MaxCFL, dtMax;
    R L1, L2, L3;
    R cK;                       // c10 / KPP0
    R cRC;                      // Rho0 * Cp0 / (a10 * b10)
    R k2, k3, k4, k5;           // 2 c12, 3 c13, 4 c14, 5 c15 (dKPP in Horner form)
    R n0, n1, n2, n3, n4, n5;   // d(invRhoCp)/dT numerator collected in powers of DeltaT*T
};
using Phys = PhysT<double>;

template <class R>
inline PhysT<R> phys_cast(const Phys &p)
{
    static_assert(sizeof(Phys) % sizeof(double) == 0, "Phys holds doubles only");
    PhysT<R> q;
    const double *src = reinterpret_cast<const double *>(&p);
    R *dst = reinterpret_cast<R *>(&q);
    for (size_t i = 0; i < sizeof(Phys) / sizeof(double); i++) dst[i] = (R)src[i];
    return q;
}

// Device scalar block (one per case, FP64 in both forms).  dt is read by
// every kernel so the step needs no host synchronisation and can be replayed
// as a CUDA graph.
enum : int {
    S_DT = 0, S_TIME, S_CFL, S_MAXDIV, S_NUBOT, S_NUTOP, S_KE, S_BLOWUP, S_AVER,
    S_STEP, S_FIXED_DT, S_NSCAL
};
// Device doubles past the public scalars: S_OOB, in a build with
// -DTCS_BOUNDS_CHECK, the number of out-of-range indices the kernels met
// (each one recorded here and its access redirected to a valid cell instead of
// made; the stand-in for a memory checker; 0 in the normal build); S_TIMEOUT,
// the number of bounded waits on asynchronous copies that ran out (a kernel
// that records one also sets S_BLOWUP, so the step stops and reports).
enum : int { S_OOB = S_NSCAL, S_TIMEOUT, S_NALLOC };

#if defined(TCS_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
#define TCS_OOB(scal, bad, fix)                          \
    do {                                                 \
        if (bad) { atomicAdd((scal) + S_OOB, 1.0); fix; } \
    } while (0)
#else
#define TCS_OOB(scal, bad, fix) do { } while (0)
#endif

template <class R>
struct GridT {
    int N1, N2, N3;             // interior cells
    int P1, P2;                 // padded strides: P1 = N1+2, P2 = N2+2
    long long NP;               // padded element count
    MetricT<R> m1, m2, m3;      // metrics in the field type
    MetricT<double> d1, d2, d3; // FP64 metrics (the FP64 parts of the mixed form)
    PhysT<R> ph;                // constants in the field type
    Phys phd;                   // FP64 constants
    double *scal;               // device scalars (S_*)
    int kdeg2;                  // KPP has no terms above t^2 (c13 = c14 = c15 = 0: water, glycerol, constant)
};
using Grid = GridT<double>;

// complex type of a precision
template <class R> struct CplxOf;
template <> struct CplxOf<double> { using T = double2; };
template <> struct CplxOf<float> { using T = float2; };
template <class R> using cplx_t = typename CplxOf<R>::T;

template <class R>
__host__ __device__ __forceinline__ cplx_t<R> mkc(R x, R y)
{
    cplx_t<R> c;
    c.x = x; c.y = y;
    return c;
}

// Division by a loop-invariant divisor d (1 <= d < 2^31) of x < 2^31 by a
// multiply-high and a shift: m = ceil(2^(32+s) / d) - 2^32 with 2^s >= d
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994).
struct FastDiv {
    unsigned d, m, s;
    __device__ __forceinline__ unsigned div(unsigned x) const
    {
        return (unsigned)(((unsigned long long)__umulhi(x, m) + x) >> s);
    }
};
inline FastDiv make_fastdiv(unsigned d)
{
    FastDiv f;
    f.d = d; f.s = 0;
    while ((1ull << f.s) < d) f.s++;
    f.m = (unsigned)((((1ull << (32 + f.s)) + d - 1) / d) - (1ull << 32));
    return f;
}

template <class R>
__host__ __device__ __forceinline__ long long ix(const GridT<R> &g, int i, int j, int k)
{
    TCS_OOB(g.scal, (unsigned)i > (unsigned)(g.N1 + 1) || (unsigned)j > (unsigned)(g.N2 + 1) || (unsigned)k > (unsigned)(g.N3 + 1),
            (i = 1, j = 1, k = 1));
    return (long long)i + (long long)g.P1 * ((long long)j + (long long)g.P2 * (long long)k);
}

// 2-D (j,k) tables: Mu and invRho are constant along i (module_solve_momentum.f90:156-171
// assigns whole rows Mu(:,j,k) inside the i loop, leaving f(T(n1sub,j,k))).
template <class R>
__host__ __device__ __forceinline__ int ix2(const GridT<R> &g, int j, int k)
{
    TCS_OOB(g.scal, (unsigned)j > (unsigned)(g.N2 + 1) || (unsigned)k > (unsigned)(g.N3 + 1), (j = 1, k = 1));
    return j + g.P2 * k;
}

// Read-only loads through the non-coherent cache.
template <class V>
__device__ __forceinline__ V ld(const V *p) { return __ldg(p); }

// Store one interior value and its periodic images: the on-device form of
// mpi_subdomain_ghostcell_update (module_mpi_subdomain.f90:758-791) on one
// rank -- x faces, then z faces including the x-ghost columns.
template <class R, class V>
__device__ __forceinline__ void store_periodic(const GridT<R> &g, V *a, int i, int j, int k, V v)
{
    a[ix(g, i, j, k)] = v;
    const int ig = (i == 1) ? g.N1 + 1 : ((i == g.N1) ? 0 : -1);
    const int kg = (k == 1) ? g.N3 + 1 : ((k == g.N3) ? 0 : -1);
    if (ig >= 0) a[ix(g, ig, j, k)] = v;
    if (kg >= 0) {
        a[ix(g, i, j, kg)] = v;
        if (ig >= 0) a[ix(g, ig, j, kg)] = v;
    }
}

// ---------------------------------------------------------------------------
// Temperature-dependent properties: mpi_thermal_coeffi
// (module_solve_thermal.f90:129-154), evaluated at the point where the
// stencil needs them instead of being stored.
// ---------------------------------------------------------------------------
// Horner forms of KPP = c10 (1 + c11 t + ... + c15 t^5) / KPP0 and its
// derivative.  With d2 (c13 = c14 = c15 = 0) the zero leading terms are
// skipped; in Horner form they only add exact zeros, so the values are the same.
template <class R>
__device__ __forceinline__ void kpp_eval(const PhysT<R> &p, bool d2, R T, R &kpp, R &dkpp)
{
    const R t = p.DeltaT * T;
    if (d2) {
        kpp = p.cK * (R(1) + t * (p.c11 + t * p.c12));
        dkpp = p.cK * (p.c11 + t * p.k2);
    } else {
        kpp = p.cK * (R(1) + t * (p.c11 + t * (p.c12 + t * (p.c13 + t * (p.c14 + t * p.c15)))));
        dkpp = p.cK * (p.c11 + t * (p.k2 + t * (p.k3 + t * (p.k4 + t * p.k5))));
    }
}

template <class R>
__device__ __forceinline__ R kpp_only(const PhysT<R> &p, bool d2, R T)
{
    const R t = p.DeltaT * T;
    if (d2) return p.cK * (R(1) + t * (p.c11 + t * p.c12));
    return p.cK * (R(1) + t * (p.c11 + t * (p.c12 + t * (p.c13 + t * (p.c14 + t * p.c15)))));
}

// invRhoCp = Rho0 Cp0 / (a10 (1 + A)) / (b10 (1 + B)) and its T-derivative
// share one reciprocal of q1 q2 = (1 + A)(1 + B): every property set of
// module_global.f90 has a14 = a15 = b14 = b15 = 0, so 1 + A is the q1 of
// module_solve_thermal.f90:149.  The derivative's numerator (:144-148) is
// collected into a polynomial in t = DeltaT*T with coefficients n0..n5.
template <class R>
__device__ __forceinline__ R qrcp(R b);
template <>
__device__ __forceinline__ double qrcp<double>(double b);

template <class R>
__device__ __forceinline__ void rhocp_eval(const PhysT<R> &p, R T, R &irc, R &dirc)
{
    const R t = p.DeltaT * T;
    const R q1 = R(1) + t * (p.a11 + t * (p.a12 + t * p.a13));
    const R q2 = R(1) + t * (p.b11 + t * (p.b12 + t * p.b13));
    const R rq = qrcp(q1 * q2);
    irc = p.cRC * rq;
    dirc = -(p.n0 + t * (p.n1 + t * (p.n2 + t * (p.n3 + t * (p.n4 + t * p.n5))))) * (rq * rq);
}

// ---------------------------------------------------------------------------
// Batched (cyclic) tridiagonal line solver.
//
// A thread block owns TL lines of n rows.  Coefficients are built straight
// into shared memory (normalised by the diagonal), then each warp solves one
// line with the PaScaL_TDMA scheme mapped onto lanes: lane p owns a
// contiguous partition of the line and runs the modified Thomas elimination
// of pascal_tdma.f90:503-541 on it, the 2P-row reduced system is folded to P
// rows and solved by parallel cyclic reduction across the lanes with warp
// shuffles, and every lane back-substitutes its partition
// (pascal_tdma.f90:567-576).  The result is written back in place and
// emitted by the caller in a coalesced order.
//
// With FP32 rows the block also keeps the rows as built; after the first
// solve it forms the residual d - (a x[r-1] + b x[r] + c x[r+1]) in FP64
// (the products of two floats are exact in FP64), solves once more for the
// correction with the same elimination and emits x + correction.
// ---------------------------------------------------------------------------
struct LinePlan {
    int n;       // rows per line
    int P;       // partitions (lanes) per line, <= 32; power of two when cyclic
    int m0, rem; // partition p has m0 + (p < rem) rows
    int PS;      // shared-memory stride between partitions (odd)
    int LS;      // shared-memory stride between lines (odd, or set per problem by plan_for)
    int TL;      // lines per block
    int cyclic;
};

template <class R, int NR>
struct Coef {
    R a, b, c, d[NR];
};

// Quotients of the line solver (correctly rounded in both forms: with the
// hardware's approximate FP32 reciprocal the y-sweep of solvedV kept 6e-6
// relative error after its refinement pass, against 5e-7 with this).
template <class R>
__device__ __forceinline__ R qdiv(R a, R b) { return a / b; }

// Reciprocals of the line solver.  FP64: the hardware's approximate
// reciprocal refined by two Newton-Raphson steps y <- y + y (1 - b y), the
// classical iteration (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990):
// each step squares the relative error, so the result is within about one ulp
// of the correctly rounded 1/b for every normal b (tcs_check_reciprocal
// measures it against the correctly rounded quotient).  It takes a handful of
// instructions where the correctly rounded quotient takes a few tens.  FP32:
// the approximate FP32 reciprocal refined by one Newton-Raphson step (the
// unrefined approximation cost the y sweep of solvedV accuracy, see qdiv).
template <class R>
__device__ __forceinline__ R qrcp(R b) { return R(1) / b; }
template <>
__device__ __forceinline__ float qrcp<float>(float b)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    return fmaf(y, fmaf(-b, y, 1.0f), y);
}
template <>
__device__ __forceinline__ double qrcp<double>(double b)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    return fma(y, e, y);
}

// The reciprocal a line family uses: qrcp where it measured faster (FR), the
// correctly rounded quotient elsewhere (the two agree to the last bit on every
// value tcs_check_reciprocal has tried; the choice moves register allocation
// and scheduling, so it is made per family by measurement).
template <bool FR, class R>
__device__ __forceinline__ R rcp_of(R b)
{
    if constexpr (FR) return qrcp(b);
    else return qdiv(R(1), b);
}
// What a lane keeps from the elimination of its partition so that another
// right-hand side can be solved with the same factors (the refinement pass).
template <class R>
struct LaneFactors {
    R A0, C0, Am, Cm, rr0, c0, den;
    R k1[5], k2[5];          // PCR multipliers per level (P <= 32: at most 5 levels)
};

// Solve one line held in shared memory (normalised rows: b == 1).
// A, C: coefficient rows; D: NR right-hand sides spaced by DS.  With REC the
// pivot reciprocals of rows 2.. are stored in F and the lane's remaining
// factors in *lf, for warp_resolve_line.
template <class R, int NR, bool REC = false, bool FR = false>
__device__ __forceinline__ void warp_solve_line(R *__restrict__ A, R *__restrict__ C, R *__restrict__ D, int DS,
                                                const LinePlan &lp, int lane,
                                                R *__restrict__ F = nullptr, LaneFactors<R> *lf = nullptr)
{
    const int P = lp.P;
    const bool act = lane < P;
    const int m = act ? lp.m0 + (lane < lp.rem ? 1 : 0) : 0;
    const int base = lane * lp.PS;
    R A0 = R(0), C0 = R(0), Am = R(0), Cm = R(0), D0[NR], Dm[NR];
    R rr0 = R(0), c0 = R(0);
#pragma unroll
    for (int q = 0; q < NR; q++) { D0[q] = R(0); Dm[q] = R(0); }

    if (act) {
        R *a = A + base, *c = C + base, *d = D + base;
        // forward elimination (rows 0 and 1 are already normalised)
        R am1 = a[1], cm1 = c[1], dm1[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) dm1[q] = d[q * DS + 1];
        for (int r = 2; r < m; r++) {
            const R ar = a[r];
            const R rr = rcp_of<FR>(R(1) - ar * cm1);
            if (REC) F[base + r] = rr;
#pragma unroll
            for (int q = 0; q < NR; q++) { dm1[q] = rr * (d[q * DS + r] - ar * dm1[q]); d[q * DS + r] = dm1[q]; }
            cm1 = rr * c[r]; c[r] = cm1;
            am1 = -rr * ar * am1; a[r] = am1;
        }
        Am = am1; Cm = cm1;
#pragma unroll
        for (int q = 0; q < NR; q++) Dm[q] = dm1[q];
        // backward elimination of the upper diagonal: rows m-3 .. 1
        if (m >= 3) {
            R ap1 = a[m - 2], cp1 = c[m - 2], dp1[NR];
#pragma unroll
            for (int q = 0; q < NR; q++) dp1[q] = d[q * DS + m - 2];
            for (int r = m - 3; r >= 1; r--) {
                const R cr = c[r];
#pragma unroll
                for (int q = 0; q < NR; q++) { dp1[q] = d[q * DS + r] - cr * dp1[q]; d[q * DS + r] = dp1[q]; }
                ap1 = a[r] - cr * ap1; a[r] = ap1;
                cp1 = -cr * cp1; c[r] = cp1;
            }
            // closure of row 0 with row 1 (pascal_tdma.f90:531-535)
            c0 = c[0];
            rr0 = rcp_of<FR>(R(1) - ap1 * c0);
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = rr0 * (d[q * DS] - c0 * dp1[q]);
            A0 = rr0 * a[0];
            C0 = -rr0 * c0 * cp1;
        } else {
            A0 = a[0]; C0 = c[0];
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = d[q * DS];
        }
    }
    const bool cyc = lp.cyclic != 0;
    if (!cyc) {
        if (lane == 0) A0 = R(0);
        if (lane == P - 1) Cm = R(0);
    }
    // Fold the 2P-row reduced system onto the first rows of every partition:
    //   alpha z_{p-1} + beta z_p + gamma z_{p+1} = delta,  z_p = x_first(p)
    const int prv = cyc ? ((lane - 1 + P) & (P - 1)) : (lane > 0 ? lane - 1 : 0);
    const R Amp = __shfl_sync(0xffffffffu, Am, prv);
    const R Cmp = __shfl_sync(0xffffffffu, Cm, prv);
    R al = -A0 * Amp;
    R be = R(1) - A0 * Cmp - C0 * Am;
    R ga = -C0 * Cm;
    R de[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const R Dmp = __shfl_sync(0xffffffffu, Dm[q], prv);
        de[q] = D0[q] - A0 * Dmp - C0 * Dm[q];
    }
    if (!act) { al = R(0); be = R(1); ga = R(0);
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = R(0); }
    // parallel cyclic reduction across the P lanes; every lane forms the
    // reciprocal of its own diagonal once per level and its neighbours read it
#pragma unroll
    for (int lev = 0; lev < 5; lev++) {
        const int s = 1 << lev;
        if (s >= P) break;
        int lo = lane - s, hi = lane + s;
        bool lo_ok = true, hi_ok = true;
        if (cyc) { lo = (lo + P) & (P - 1); hi = hi & (P - 1); }
        else { lo_ok = lo >= 0; hi_ok = hi < P; lo = lo_ok ? lo : lane; hi = hi_ok ? hi : lane; }
        const R rbe = rcp_of<FR>(be);
        R alm = __shfl_sync(0xffffffffu, al, lo), rbm = __shfl_sync(0xffffffffu, rbe, lo), gam = __shfl_sync(0xffffffffu, ga, lo);
        R alp = __shfl_sync(0xffffffffu, al, hi), rbp = __shfl_sync(0xffffffffu, rbe, hi), gap = __shfl_sync(0xffffffffu, ga, hi);
        R dem[NR], dep[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) { dem[q] = __shfl_sync(0xffffffffu, de[q], lo); dep[q] = __shfl_sync(0xffffffffu, de[q], hi); }
        if (!lo_ok) { alm = R(0); rbm = R(1); gam = R(0);
#pragma unroll
            for (int q = 0; q < NR; q++) dem[q] = R(0); }
        if (!hi_ok) { alp = R(0); rbp = R(1); gap = R(0);
#pragma unroll
            for (int q = 0; q < NR; q++) dep[q] = R(0); }
        const R k1 = al * rbm, k2 = ga * rbp;
        if (REC) { lf->k1[lev] = k1; lf->k2[lev] = k2; }
        const R nal = -k1 * alm, nga = -k2 * gap;
        const R nbe = be - k1 * gam - k2 * alp;
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = de[q] - k1 * dem[q] - k2 * dep[q];
        al = nal; be = nbe; ga = nga;
    }
    const R den = rcp_of<FR>(al + be + ga);
    if (REC) { lf->A0 = A0; lf->C0 = C0; lf->Am = Am; lf->Cm = Cm; lf->rr0 = rr0; lf->c0 = c0; lf->den = den; }
    R z[NR], xl[NR];
    const int nxt = cyc ? ((lane + 1) & (P - 1)) : (lane + 1 < 32 ? lane + 1 : lane);
#pragma unroll
    for (int q = 0; q < NR; q++) {
        z[q] = de[q] * den;
        const R zn = __shfl_sync(0xffffffffu, z[q], nxt);
        xl[q] = Dm[q] - Am * z[q] - Cm * zn;
    }
    if (act) {
        R *a = A + base, *c = C + base, *d = D + base;
#pragma unroll
        for (int q = 0; q < NR; q++) { d[q * DS] = z[q]; d[q * DS + m - 1] = xl[q]; }
        for (int r = 1; r < m - 1; r++) {
            const R ar = a[r], cr = c[r];
#pragma unroll
            for (int q = 0; q < NR; q++) d[q * DS + r] = d[q * DS + r] - ar * z[q] - cr * xl[q];
        }
    }
}

// The same elimination with the lane's partition held in registers (at most
// M rows; every loop is unrolled over M with the rows beyond m switched off),
// so no shared-memory access sits on the elimination chains.  The rows are
// read once and the solution (and, with REC, the eliminated rows and pivot
// reciprocals the refinement replays) written once.
template <class R, int NR, int M, bool REC = false, bool FR = false>
__device__ __forceinline__ void warp_solve_line_reg(R *__restrict__ A, R *__restrict__ C, R *__restrict__ D, int DS,
                                                    const LinePlan &lp, int lane,
                                                    R *__restrict__ F = nullptr, LaneFactors<R> *lf = nullptr)
{
    const int P = lp.P;
    const bool act = lane < P;
    const int m = act ? lp.m0 + (lane < lp.rem ? 1 : 0) : 0;
    const int base = lane * lp.PS;
    R a[M], c[M], d[NR][M];
#pragma unroll
    for (int r = 0; r < M; r++) {
        const bool on = r < m;
        a[r] = on ? A[base + r] : R(0);
        c[r] = on ? C[base + r] : R(0);
#pragma unroll
        for (int q = 0; q < NR; q++) d[q][r] = on ? D[q * DS + base + r] : R(0);
    }
    // forward elimination (rows 0 and 1 are already normalised)
#pragma unroll
    for (int r = 2; r < M; r++) {
        if (r < m) {
            const R ar = a[r];
            const R rr = rcp_of<FR>(R(1) - ar * c[r - 1]);
            if (REC) F[base + r] = rr;
#pragma unroll
            for (int q = 0; q < NR; q++) d[q][r] = rr * (d[q][r] - ar * d[q][r - 1]);
            c[r] = rr * c[r];
            a[r] = -rr * ar * a[r - 1];
        }
    }
    R Am = R(0), Cm = R(0), Dm[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) Dm[q] = R(0);
#pragma unroll
    for (int r = 1; r < M; r++)
        if (r == m - 1) {
            Am = a[r]; Cm = c[r];
#pragma unroll
            for (int q = 0; q < NR; q++) Dm[q] = d[q][r];
        }
    // backward elimination of the upper diagonal: rows m-3 .. 1
#pragma unroll
    for (int r = M - 3; r >= 1; r--) {
        if (r <= m - 3) {
            const R cr = c[r];
#pragma unroll
            for (int q = 0; q < NR; q++) d[q][r] = d[q][r] - cr * d[q][r + 1];
            a[r] = a[r] - cr * a[r + 1];
            c[r] = -cr * c[r + 1];
        }
    }
    R A0 = R(0), C0 = R(0), D0[NR], rr0 = R(0), c0 = R(0);
#pragma unroll
    for (int q = 0; q < NR; q++) D0[q] = R(0);
    if (act) {
        if (m >= 3) {
            // closure of row 0 with row 1 (pascal_tdma.f90:531-535)
            c0 = c[0];
            rr0 = rcp_of<FR>(R(1) - a[1] * c0);
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = rr0 * (d[q][0] - c0 * d[q][1]);
            A0 = rr0 * a[0];
            C0 = -rr0 * c0 * c[1];
        } else {
            A0 = a[0]; C0 = c[0];
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = d[q][0];
        }
    }
    const bool cyc = lp.cyclic != 0;
    if (!cyc) {
        if (lane == 0) A0 = R(0);
        if (lane == P - 1) Cm = R(0);
    }
    const int prv = cyc ? ((lane - 1 + P) & (P - 1)) : (lane > 0 ? lane - 1 : 0);
    const R Amp = __shfl_sync(0xffffffffu, Am, prv);
    const R Cmp = __shfl_sync(0xffffffffu, Cm, prv);
    R al = -A0 * Amp;
    R be = R(1) - A0 * Cmp - C0 * Am;
    R ga = -C0 * Cm;
    R de[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const R Dmp = __shfl_sync(0xffffffffu, Dm[q], prv);
        de[q] = D0[q] - A0 * Dmp - C0 * Dm[q];
    }
    if (!act) { al = R(0); be = R(1); ga = R(0);
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = R(0); }
#pragma unroll
    for (int lev = 0; lev < 5; lev++) {
        const int s = 1 << lev;
        if (s >= P) break;
        int lo = lane - s, hi = lane + s;
        bool lo_ok = true, hi_ok = true;
        if (cyc) { lo = (lo + P) & (P - 1); hi = hi & (P - 1); }
        else { lo_ok = lo >= 0; hi_ok = hi < P; lo = lo_ok ? lo : lane; hi = hi_ok ? hi : lane; }
        const R rbe = rcp_of<FR>(be);
        R alm = __shfl_sync(0xffffffffu, al, lo), rbm = __shfl_sync(0xffffffffu, rbe, lo), gam = __shfl_sync(0xffffffffu, ga, lo);
        R alp = __shfl_sync(0xffffffffu, al, hi), rbp = __shfl_sync(0xffffffffu, rbe, hi), gap = __shfl_sync(0xffffffffu, ga, hi);
        R dem[NR], dep[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) { dem[q] = __shfl_sync(0xffffffffu, de[q], lo); dep[q] = __shfl_sync(0xffffffffu, de[q], hi); }
        if (!lo_ok) { alm = R(0); rbm = R(1); gam = R(0);
#pragma unroll
            for (int q = 0; q < NR; q++) dem[q] = R(0); }
        if (!hi_ok) { alp = R(0); rbp = R(1); gap = R(0);
#pragma unroll
            for (int q = 0; q < NR; q++) dep[q] = R(0); }
        const R k1 = al * rbm, k2 = ga * rbp;
        if (REC) { lf->k1[lev] = k1; lf->k2[lev] = k2; }
        const R nal = -k1 * alm, nga = -k2 * gap;
        const R nbe = be - k1 * gam - k2 * alp;
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = de[q] - k1 * dem[q] - k2 * dep[q];
        al = nal; be = nbe; ga = nga;
    }
    const R den = rcp_of<FR>(al + be + ga);
    if (REC) { lf->A0 = A0; lf->C0 = C0; lf->Am = Am; lf->Cm = Cm; lf->rr0 = rr0; lf->c0 = c0; lf->den = den; }
    R z[NR], xl[NR];
    const int nxt = cyc ? ((lane + 1) & (P - 1)) : (lane + 1 < 32 ? lane + 1 : lane);
#pragma unroll
    for (int q = 0; q < NR; q++) {
        z[q] = de[q] * den;
        const R zn = __shfl_sync(0xffffffffu, z[q], nxt);
        xl[q] = Dm[q] - Am * z[q] - Cm * zn;
    }
#pragma unroll
    for (int r = 0; r < M; r++) {
        if (r < m) {
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const R x = (r == 0) ? z[q] : (r == m - 1 ? xl[q] : d[q][r] - a[r] * z[q] - c[r] * xl[q]);
                D[q * DS + base + r] = x;
            }
            if (REC) { A[base + r] = a[r]; C[base + r] = c[r]; }
        }
    }
}

// Solve a line with the register-resident elimination when the lane's
// partition fits MREG rows, else in shared memory.
template <class R, int NR, int MREG, bool REC = false, bool FR = false>
__device__ __forceinline__ void solve_line(R *A, R *C, R *D, int DS, const LinePlan &lp, int lane, R *F = nullptr,
                                           LaneFactors<R> *lf = nullptr)
{
    if (MREG > 0 && lp.m0 + (lp.rem ? 1 : 0) <= MREG)
        warp_solve_line_reg<R, NR, (MREG > 0 ? MREG : 1), REC, FR>(A, C, D, DS, lp, lane, F, lf);
    else
        warp_solve_line<R, NR, REC, FR>(A, C, D, DS, lp, lane, F, lf);
}

// Solve the same line for another right-hand side D (in place) with the
// factors of a recorded warp_solve_line: A, C hold its final eliminated rows,
// A0n, C0n the normalised rows before elimination, F the pivot reciprocals.
// The recurrences are the elimination's own, applied to D alone.
template <class R, int NR>
__device__ __forceinline__ void warp_resolve_line(const R *__restrict__ A, const R *__restrict__ C, R *__restrict__ D, int DS,
                                                  const R *__restrict__ A0n, const R *__restrict__ C0n,
                                                  const R *__restrict__ F, const LaneFactors<R> &lf, const LinePlan &lp, int lane)
{
    const int P = lp.P;
    const bool act = lane < P;
    const int m = act ? lp.m0 + (lane < lp.rem ? 1 : 0) : 0;
    const int base = lane * lp.PS;
    R D0[NR], Dm[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) { D0[q] = R(0); Dm[q] = R(0); }
    if (act) {
        R *d = D + base;
        const R *an = A0n + base, *cn = C0n + base, *f = F + base;
        R dm1[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) dm1[q] = d[q * DS + 1];
        for (int r = 2; r < m; r++) {
            const R rr = f[r], ar = an[r];
#pragma unroll
            for (int q = 0; q < NR; q++) { dm1[q] = rr * (d[q * DS + r] - ar * dm1[q]); d[q * DS + r] = dm1[q]; }
        }
#pragma unroll
        for (int q = 0; q < NR; q++) Dm[q] = dm1[q];
        if (m >= 3) {
            R dp1[NR];
#pragma unroll
            for (int q = 0; q < NR; q++) dp1[q] = d[q * DS + m - 2];
            for (int r = m - 3; r >= 1; r--) {
                const R cr = r >= 2 ? f[r] * cn[r] : cn[r];    // the forward pass's c of row r
#pragma unroll
                for (int q = 0; q < NR; q++) { dp1[q] = d[q * DS + r] - cr * dp1[q]; d[q * DS + r] = dp1[q]; }
            }
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = lf.rr0 * (d[q * DS] - lf.c0 * dp1[q]);
        } else {
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = d[q * DS];
        }
    }
    const bool cyc = lp.cyclic != 0;
    const int prv = cyc ? ((lane - 1 + P) & (P - 1)) : (lane > 0 ? lane - 1 : 0);
    R de[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const R Dmp = __shfl_sync(0xffffffffu, Dm[q], prv);
        de[q] = act ? D0[q] - lf.A0 * Dmp - lf.C0 * Dm[q] : R(0);
    }
#pragma unroll
    for (int lev = 0; lev < 5; lev++) {
        const int s = 1 << lev;
        if (s >= P) break;
        int lo = lane - s, hi = lane + s;
        bool lo_ok = true, hi_ok = true;
        if (cyc) { lo = (lo + P) & (P - 1); hi = hi & (P - 1); }
        else { lo_ok = lo >= 0; hi_ok = hi < P; lo = lo_ok ? lo : lane; hi = hi_ok ? hi : lane; }
#pragma unroll
        for (int q = 0; q < NR; q++) {
            R dem = __shfl_sync(0xffffffffu, de[q], lo), dep = __shfl_sync(0xffffffffu, de[q], hi);
            if (!lo_ok) dem = R(0);
            if (!hi_ok) dep = R(0);
            de[q] = de[q] - lf.k1[lev] * dem - lf.k2[lev] * dep;
        }
    }
    R z[NR], xl[NR];
    const int nxt = cyc ? ((lane + 1) & (P - 1)) : (lane + 1 < 32 ? lane + 1 : lane);
#pragma unroll
    for (int q = 0; q < NR; q++) {
        z[q] = de[q] * lf.den;
        const R zn = __shfl_sync(0xffffffffu, z[q], nxt);
        xl[q] = Dm[q] - lf.Am * z[q] - lf.Cm * zn;
    }
    if (act) {
        const R *a = A + base, *c = C + base;
        R *d = D + base;
#pragma unroll
        for (int q = 0; q < NR; q++) { d[q * DS] = z[q]; d[q * DS + m - 1] = xl[q]; }
        for (int r = 1; r < m - 1; r++) {
            const R ar = a[r], cr = c[r];
#pragma unroll
            for (int q = 0; q < NR; q++) d[q * DS + r] = d[q * DS + r] - ar * z[q] - cr * xl[q];
        }
    }
}

// The kernel.  Prob supplies:
//   using Real (row type: the field type, or double for FP64 solves of FP32 data);
//   static constexpr int NRHS, NT (threads per block), MINB (blocks per SM), MREG (rows per lane in
//   registers, 0: in shared memory);  static constexpr bool CONTIG (rows contiguous in memory);
//   struct State; __device__ State prepare()   -> per-block scalars (dt, stale values)
//   __device__ bool skip(), line_ok(int l)
//   __device__ Coef<Real, NRHS> build(int l, int r, const State &)
//   __device__ void emit(int l, int r, const Real *x, const State &)
// TL (lines per block) is a power of two; blockDim.x is Prob::NT (a multiple of 32).
template <class R>
struct Refine { static constexpr bool on = std::is_same<R, float>::value; };

// Blocks per SM a line-solver family is compiled for (each Prob's MINB; the
// register budget is 65536 / (NT MINB), and fit_tl sizes the lines per block
// to the matching shared-memory share).  Measured on B200 at 256^3: the FP64
// z-sweep stencils need 128 registers and spill below that; the FP64 x and y
// sweeps run fastest at 4 blocks (64 registers, no spills); the refined FP32
// rows need 28 B each, so the FP32 z and y sweeps and the modal solves run best
// at 3 blocks of 256 threads and the FP32 x sweeps at 6 blocks of 128.
template <class R>
struct LineOcc {
    static constexpr bool f32 = std::is_same<R, float>::value;
    static constexpr int z = f32 ? 3 : 2;
    static constexpr int x = f32 ? 6 : 4;
    static constexpr int y = f32 ? 3 : 4;
    static constexpr int modal = 3;
    // rows per lane solved in registers (0: in shared memory), per family:
    // wherever the registers allow it without spills (not the FP64 x/y sweeps
    // at 64 registers, nor the two-right-hand-side modal solves at 80)
    static constexpr int reg_z = 8;
    static constexpr int reg_x = f32 ? 8 : 0;
    static constexpr int reg_y = f32 ? 8 : 0;
    static constexpr int reg_modal = 0;
    // threads per block, per family (the FP32 x sweeps run best as 128-thread
    // blocks of 4 lines: the refined rows fill shared memory, and smaller
    // blocks wait less at their barriers)
    static constexpr int nt_z = 256, nt_x = f32 ? 128 : 256, nt_y = 256, nt_modal = 256;
    // the FP64 z sweeps build row-adjacent cells in pairs (PairRows)
    static constexpr bool pair_z = !f32;
    // the x sweeps' wide shape, for lines too long to fit 4 per 128-thread block
    static constexpr int xw = f32 ? 3 : 4, nt_xw = 256, reg_xw = reg_x;
};

// The block a line problem works on, read through vbx<ITEM>() / vby<ITEM>():
// blockIdx in a one-case launch (ITEM = 0), the work item's block in a
// multi-case launch (ITEM = 1, line_solve_multi).  The problem structs carry
// ITEM as a template parameter, so one-case launches keep reading blockIdx.
static __shared__ int2 s_vblk;
template <int ITEM> __device__ __forceinline__ int vbx() { return ITEM ? s_vblk.x : (int)blockIdx.x; }
template <int ITEM> __device__ __forceinline__ int vby() { return ITEM ? s_vblk.y : (int)blockIdx.y; }

// Shared-memory words (of the row type) per row: A, C, D[NR]; refined rows
// also keep the normalised rows as built (A0, C0, D0[NR]; D0 becomes the
// residual) and the pivot reciprocals F of the first solve.
template <class Prob>
__host__ __device__ constexpr int line_words()
{
    return Refine<typename Prob::Real>::on ? 5 + 2 * Prob::NRHS : 2 + Prob::NRHS;
}

// Problems whose line solves use qrcp (Prob::FAST_RCP).
template <class P, class = void>
struct FastRcp { static constexpr bool on = false; };
template <class P>
struct FastRcp<P, std::void_t<decltype(P::FAST_RCP)>> { static constexpr bool on = P::FAST_RCP; };

// Problems whose build takes row-adjacent cells in pairs (Prob::PAIR).
template <class P, class = void>
struct PairRows { static constexpr bool on = false; };
template <class P>
struct PairRows<P, std::void_t<decltype(P::PAIR)>> { static constexpr bool on = P::PAIR; };

// Unpaired strided builds that keep one line per thread and step its rows by
// NT / TL (Prob::LINE_PER_THREAD; default: FP32 rows).  Measured at 256^3: the
// FP32 sweeps and the modal solves faster (modal -3% in FP64, -10% in FP32;
// FP32 thermal_y -4%), the FP64 y sweeps and the FP32 dw_z slower (+4-8%, +3%).
template <class P, class = void>
struct LinePerThread { static constexpr bool on = std::is_same<typename P::Real, float>::value; };
template <class P>
struct LinePerThread<P, std::void_t<decltype(P::LINE_PER_THREAD)>> { static constexpr bool on = P::LINE_PER_THREAD; };

template <class Prob>
__device__ __forceinline__ void line_block(const Prob &prob, const LinePlan &lp)
{
    using R = typename Prob::Real;
    constexpr int NR = Prob::NRHS;
    constexpr bool REF = Refine<R>::on;
    extern __shared__ __align__(16) unsigned char smraw[];
    R *sm = reinterpret_cast<R *>(smraw);
    if (prob.skip()) return;
    const typename Prob::State st = prob.prepare();
    const int TL = lp.TL, n = lp.n, LS = lp.LS;
    const int lgTL = __ffs(TL) - 1;
    const int DS = TL * LS;
    R *sA = sm, *sC = sA + DS, *sD = sC + DS;
    R *sA0 = sD + NR * DS, *sF = sA0 + DS, *sC0 = sF + DS, *sD0 = sC0 + DS;   // refined rows only
    int *spos = reinterpret_cast<int *>(sm + (size_t)line_words<Prob>() * DS);
    // row -> shared-memory position: partition p holds rows start_p .. start_p + m_p - 1
    if (threadIdx.x < lp.P) {
        const int p = threadIdx.x, m = lp.m0 + (p < lp.rem ? 1 : 0);
        const int start = p * lp.m0 + (p < lp.rem ? p : lp.rem);
        for (int q = 0; q < m; q++) spos[start + q] = p * lp.PS + q;
    }
    __syncthreads();
    auto put = [&](int l, int r) {
        TCS_OOB(prob.g.scal, (unsigned)l >= (unsigned)TL || (unsigned)r >= (unsigned)n, return);
        const int pos = l * LS + spos[r];
        Coef<R, NR> cf;
        if (prob.line_ok(l)) {
            cf = prob.build(l, r, st);
        } else {
            cf.a = R(0); cf.b = R(1); cf.c = R(0);
#pragma unroll
            for (int q = 0; q < NR; q++) cf.d[q] = R(0);
        }
        const R rb = rcp_of<FastRcp<Prob>::on>(cf.b);
        const R an = cf.a * rb, cn = cf.c * rb;
        sA[pos] = an; sC[pos] = cn;
#pragma unroll
        for (int q = 0; q < NR; q++) sD[q * DS + pos] = cf.d[q] * rb;
        if (REF) {
            sA0[pos] = an; sC0[pos] = cn;
#pragma unroll
            for (int q = 0; q < NR; q++) sD0[q * DS + pos] = sD[q * DS + pos];
        }
    };
    if (Prob::CONTIG) {
        // lines in pairs: the loads their stencils share are issued once (1-2% on the x sweeps)
        int l = 0;
        for (; l + 1 < TL; l += 2)
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                put(l, r);
                put(l + 1, r);
            }
        for (; l < TL; l++)
            for (int r = threadIdx.x; r < n; r += blockDim.x) put(l, r);
    } else {
        if constexpr (PairRows<Prob>::on) {
            // two row-adjacent cells per thread: their loads are in flight together and
            // the loads their stencils share are issued once (measured on the FP64 z
            // sweeps: dw_z -8%, thermal_z -3%; slower on the y sweeps and in FP32).
            // Pair t = threadIdx.x + m NT of the block's TL x nh pairs is (line t mod TL,
            // pair t / TL); NT is a multiple of TL, so a thread keeps one line and steps
            // its pairs by NT / TL: the same cells in the same order, with less index
            // arithmetic per cell (dw_z -2%, dv_z -1%).
            const int nh = (n + 1) >> 1, l = threadIdx.x & (TL - 1), hstep = Prob::NT >> lgTL;
            for (int h = threadIdx.x >> lgTL; h < nh; h += hstep) {
                const int r = h << 1;
                if (r + 1 < n) {   // both cells in one block, so their loads can be merged and interleaved
                    put(l, r);
                    put(l, r + 1);
                } else {
                    put(l, r);
                }
            }
        } else if constexpr (LinePerThread<Prob>::on) {
            // the same cells and order as below, one line per thread
            const int l = threadIdx.x & (TL - 1), rstep = Prob::NT >> lgTL;
#pragma unroll 2
            for (int r = threadIdx.x >> lgTL; r < n; r += rstep) put(l, r);
        } else {
            // two cells per pass: their loads are in flight together (measured 3-7% on the FP64 z and y sweeps)
#pragma unroll 2
            for (int t = threadIdx.x; t < TL * n; t += blockDim.x) put(t & (TL - 1), t >> lgTL);
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int l = warp; l < TL; l += nw) {
        if (!REF) {
            solve_line<R, NR, Prob::MREG, false, FastRcp<Prob>::on>(sA + l * LS, sC + l * LS, sD + l * LS, DS, lp, lane);
            continue;
        }
        // FP32 rows: solve recording the factors, form the residual of the
        // solution against the rows as built in FP64 (it replaces D0), and
        // solve for the correction with the recorded factors.
        LaneFactors<R> lf;
        solve_line<R, NR, Prob::MREG, true, FastRcp<Prob>::on>(sA + l * LS, sC + l * LS, sD + l * LS, DS, lp, lane, sF + l * LS, &lf);
        __syncwarp();
        for (int r = lane; r < n; r += 32) {
            const int pos = l * LS + spos[r];
            const int rm = r > 0 ? r - 1 : (lp.cyclic ? n - 1 : -1);
            const int rp = r < n - 1 ? r + 1 : (lp.cyclic ? 0 : -1);
            const int pm = l * LS + spos[rm >= 0 ? rm : r], pp = l * LS + spos[rp >= 0 ? rp : r];
            const double a = (double)sA0[pos], c = (double)sC0[pos];
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const double xm = rm >= 0 ? (double)sD[q * DS + pm] : 0.0;
                const double xp = rp >= 0 ? (double)sD[q * DS + pp] : 0.0;
                const double res = (double)sD0[q * DS + pos] - (a * xm + (double)sD[q * DS + pos] + c * xp);
                sD0[q * DS + pos] = (R)res;
            }
        }
        __syncwarp();
        warp_resolve_line<R, NR>(sA + l * LS, sC + l * LS, sD0 + l * LS, DS, sA0 + l * LS, sC0 + l * LS,
                                 sF + l * LS, lf, lp, lane);
    }
    __syncthreads();
    auto out = [&](int l, int r) {
        if (!prob.line_ok(l)) return;
        TCS_OOB(prob.g.scal, (unsigned)l >= (unsigned)TL || (unsigned)r >= (unsigned)n, return);
        const int pos = l * LS + spos[r];
        R x[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) x[q] = REF ? sD[q * DS + pos] + sD0[q * DS + pos] : sD[q * DS + pos];
        prob.emit(l, r, x, st);
    };
    if (Prob::CONTIG) {
        for (int l = 0; l < TL; l++)
            for (int r = threadIdx.x; r < n; r += blockDim.x) out(l, r);
    } else if constexpr (PairRows<Prob>::on || LinePerThread<Prob>::on) {
        // one line per thread, as in the build
        const int l = threadIdx.x & (TL - 1);
        for (int r = threadIdx.x >> lgTL; r < n; r += Prob::NT >> lgTL) out(l, r);
    } else {
        for (int t = threadIdx.x; t < TL * n; t += blockDim.x) out(t & (TL - 1), t >> lgTL);
    }
}

template <class Prob>
__global__ void __launch_bounds__(Prob::NT, Prob::MINB) line_solve_kernel(Prob prob, LinePlan lp)
{
    line_block(prob, lp);
}

// Blocks per SM the one-line-per-thread kernel is compiled for
// (Prob::THOMAS_MINB; default 8, i.e. 64 registers).  Measured on B200 at
// 512^3: the y sweeps 4-18% faster at 64 registers than uncapped (80-96), and
// slower at 48 (spills).
template <class P, class = void>
struct ThomasMinB { static constexpr int v = 8; };
template <class P>
struct ThomasMinB<P, std::void_t<decltype(P::THOMAS_MINB)>> { static constexpr int v = P::THOMAS_MINB; };

// One line per thread: the plain Thomas elimination of a non-cyclic line in
// FP64 (the sequential elimination of tdma_single and tdma_many,
// PaScaL_TDMA/src/tdmas.f90:27-50 and 113-146), for the strided y lines and
// the modal solves.  A block of THOMAS_TL threads takes THOMAS_TL consecutive
// lines (the problem's TL is THOMAS_TL), thread l line l.  The forward sweep
// builds each row with the problem's own build, keeps c' and d' of the current
// row in registers and stores them for the back substitution in
// scr[row][line] (consecutive threads, consecutive words: every store and load
// of a warp is coalesced); the back substitution emits the rows from the last
// to the first.  No shared memory and no barrier: the build's loads of the
// next rows overlap the elimination of the current one.  scr holds
// (1 + NRHS) x n x (all lines of the grid) doubles.  Rows built in FP32 (the
// FP32-mixed form) are eliminated in FP64 and the solution rounded once when
// it is emitted, which stands in for the FP32 elimination and its FP64-residual
// refinement pass.
template <class Prob>
__global__ void __launch_bounds__(128, ThomasMinB<Prob>::v) thomas_line_kernel(Prob prob, int n, double *__restrict__ scr)
{
    using R = typename Prob::Real;
    constexpr int NR = Prob::NRHS;
    if (prob.skip()) return;
    const int l = threadIdx.x;
    if (!prob.line_ok(l)) return;
    const typename Prob::State st = prob.prepare();
    const long long nl = (long long)gridDim.x * gridDim.y * blockDim.x;
    const long long me = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + l;
    double *const sc = scr + me, *const sd = scr + nl * n + me;
    double cp = 0.0, dp[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) dp[q] = 0.0;
#pragma unroll 2
    for (int r = 0; r < n; r++) {
        const Coef<R, NR> cf = prob.build(l, r, st);
        const double a = r ? (double)cf.a : 0.0;
        const double m = rcp_of<FastRcp<Prob>::on>((double)cf.b - a * cp);
        cp = (double)cf.c * m;
#pragma unroll
        for (int q = 0; q < NR; q++) dp[q] = ((double)cf.d[q] - a * dp[q]) * m;
        if (r < n - 1) {
            sc[(long long)r * nl] = cp;
#pragma unroll
            for (int q = 0; q < NR; q++) sd[((long long)r * NR + q) * nl] = dp[q];
        }
    }
    double x[NR];
    R xr[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) { x[q] = dp[q]; xr[q] = R(x[q]); }
    prob.emit(l, n - 1, xr, st);
    for (int r = n - 2; r >= 0; r--) {
        const double c = sc[(long long)r * nl];
#pragma unroll
        for (int q = 0; q < NR; q++) { x[q] = sd[((long long)r * NR + q) * nl] - c * x[q]; xr[q] = R(x[q]); }
        prob.emit(l, r, xr, st);
    }
}

// The parameters of a multi-case line launch: the problems and plans of up to
// K cases, held in the kernel-parameter space (32 KB) so that, as in
// line_solve_kernel, the kernel reads their members as constant operands (a
// copy in global or shared memory costs registers and spills in the FP64
// sweeps).  Case c owns the work items start[c] .. start[c+1]-1, block
// (bx, by) being item start[c] + by * gx[c] + bx.
template <class Prob>
struct MultiParams {
    static constexpr int K = (int)((32000 - 64) / (sizeof(Prob) + sizeof(LinePlan) + 2 * sizeof(int)));
    static_assert(K >= 1, "a problem struct must fit the kernel-parameter space");
    Prob p[K];
    LinePlan lp[K];
    int start[K + 1];
    int gx[K];
    int nitems;
    int *ctr;   // [0] next item, [1] blocks done
};

// Many cases in one launch: a persistent grid whose blocks pull work items
// (case, bx, by) from a counter and run the same block body as
// line_solve_kernel on them.  Each block claims its next item while it works
// on the current one, so the counter's round trip stays off the critical
// path.  The last block to finish sets the counter back to 0, so the next
// launch (or graph replay) starts again from item 0.
template <class Prob>
__global__ void __launch_bounds__(Prob::NT, Prob::MINB) line_solve_multi(const __grid_constant__ MultiParams<Prob> mp)
{
    __shared__ int s_case;
    int nxt = 0;   // thread 0: the item claimed next
    if (threadIdx.x == 0) nxt = atomicAdd(mp.ctr, 1);
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = nxt;
            int c = -1;
            if (it < mp.nitems) {
                c = 0;
                while (it >= mp.start[c + 1]) c++;
                const int r = it - mp.start[c], by = r / mp.gx[c];
                s_vblk = make_int2(r - by * mp.gx[c], by);
                nxt = atomicAdd(mp.ctr, 1);
            }
            s_case = c;
        }
        __syncthreads();
        const int c = s_case;
        if (c < 0) break;
        const LinePlan lp = mp.lp[c];   // a local copy keeps the solver's row arrays in registers
        line_block(mp.p[c], lp);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(mp.ctr + 1, 1) == (int)gridDim.x - 1) {
            atomicExch(mp.ctr, 0);
            atomicExch(mp.ctr + 1, 0);
        }
    }
}

} // namespace tcs
