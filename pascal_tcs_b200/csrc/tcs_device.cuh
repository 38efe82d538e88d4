// tcs_device.cuh -- device-side building blocks shared by every kernel of the
// PaScaL_TCS time step on one B200 (sm_100a).
//
// Layout: every 3-D field is one padded array (0:N1+1, 0:N2+1, 0:N3+1) with i
// fastest, exactly the reference's Fortran arrays (0:n1sub, 0:n2sub, 0:n3sub)
// on one rank, so host<->device copies are plain memcpys.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tcs {

// ---------------------------------------------------------------------------
// Metric tables of one direction (length n+2, index 0..n+1), as computed by
// mpi_subdomain_mesh (module_mpi_subdomain.f90:153-299), plus reciprocals.
// ---------------------------------------------------------------------------
struct Metric {
    const double *dx, *dmx;       // dx_sub, dmx_sub
    const double *rdx, *rdmx;     // 1/dx, 1/dmx (0 where dx or dmx is 0)
};

// Physical constants of module_global (module_global.f90:107-141) and the
// property polynomial coefficients (water/glycerol/constant).
struct Phys {
    double Cmu, Cmt, Ct, Cmp, DeltaT, a12pera11;
    double a10, a11, a12, a13, a14, a15;
    double b10, b11, b12, b13, b14, b15;
    double c10, c11, c12, c13, c14, c15;
    double d10, d11, d12, d13, d14, d15;
    double KPP0, Rho0, Cp0, Mu0;
    double Tup, Tbt, Uup, Ubt, Vup, Vbt, Wup, Wbt;
    double MaxCFL, dtMax;
    double L1, L2, L3;
    double cK;       // c10 / KPP0
    double cRC;      // Rho0 * Cp0 / (a10 * b10)
    double k2, k3, k4, k5;               // 2 c12, 3 c13, 4 c14, 5 c15 (dKPP in Horner form)
    double n0, n1, n2, n3, n4, n5;       // d(invRhoCp)/dT numerator collected in powers of DeltaT*T
};

// Device scalar block (one per case).  dt is read by every kernel so the
// step needs no host synchronisation and can be replayed as a CUDA graph.
enum : int {
    S_DT = 0, S_TIME, S_CFL, S_MAXDIV, S_NUBOT, S_NUTOP, S_KE, S_BLOWUP, S_AVER,
    S_STEP, S_FIXED_DT, S_NSCAL
};

struct Grid {
    int N1, N2, N3;          // interior cells
    int P1, P2;              // padded strides: P1 = N1+2, P2 = N2+2
    long long NP;            // padded element count
    Metric m1, m2, m3;
    Phys ph;
    double *scal;            // device scalars (S_*)
};

__host__ __device__ __forceinline__ long long ix(const Grid &g, int i, int j, int k)
{
    return (long long)i + (long long)g.P1 * ((long long)j + (long long)g.P2 * (long long)k);
}

// 2-D (j,k) tables: Mu and invRho are constant along i (module_solve_momentum.f90:156-171
// assigns whole rows Mu(:,j,k) inside the i loop, leaving f(T(n1sub,j,k))).
__host__ __device__ __forceinline__ int ix2(const Grid &g, int j, int k) { return j + g.P2 * k; }

// Read-only loads through the non-coherent cache.
__device__ __forceinline__ double ld(const double *p) { return __ldg(p); }

// Store one interior value and its periodic images: the on-device form of
// mpi_subdomain_ghostcell_update (module_mpi_subdomain.f90:758-791) on one
// rank -- x faces, then z faces including the x-ghost columns.
__device__ __forceinline__ void store_periodic(const Grid &g, double *a, int i, int j, int k, double v)
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

// Periodic index maps for reads of values that the reference takes from a
// freshly ghost-updated array.
__device__ __forceinline__ int wrap1(const Grid &g, int i) { return i < 1 ? i + g.N1 : (i > g.N1 ? i - g.N1 : i); }
__device__ __forceinline__ int wrap3(const Grid &g, int k) { return k < 1 ? k + g.N3 : (k > g.N3 ? k - g.N3 : k); }

// ---------------------------------------------------------------------------
// Temperature-dependent properties: mpi_thermal_coeffi
// (module_solve_thermal.f90:129-154), evaluated at the point where the
// stencil needs them instead of being stored.
// ---------------------------------------------------------------------------
// Horner forms of KPP = c10 (1 + c11 t + ... + c15 t^5) / KPP0 and its derivative.
__device__ __forceinline__ void kpp_eval(const Phys &p, double T, double &kpp, double &dkpp)
{
    const double t = p.DeltaT * T;
    kpp = p.cK * (1.0 + t * (p.c11 + t * (p.c12 + t * (p.c13 + t * (p.c14 + t * p.c15)))));
    dkpp = p.cK * (p.c11 + t * (p.k2 + t * (p.k3 + t * (p.k4 + t * p.k5))));
}

__device__ __forceinline__ double kpp_only(const Phys &p, double T)
{
    const double t = p.DeltaT * T;
    return p.cK * (1.0 + t * (p.c11 + t * (p.c12 + t * (p.c13 + t * (p.c14 + t * p.c15)))));
}

// invRhoCp = Rho0 Cp0 / (a10 (1 + A)) / (b10 (1 + B)) and its T-derivative
// share one reciprocal of q1 q2 = (1 + A)(1 + B): every property set of
// module_global.f90 has a14 = a15 = b14 = b15 = 0, so 1 + A is the q1 of
// module_solve_thermal.f90:149.  The derivative's numerator (:144-148) is
// collected into a polynomial in t = DeltaT*T with coefficients n0..n5.
__device__ __forceinline__ void rhocp_eval(const Phys &p, double T, double &irc, double &dirc)
{
    const double t = p.DeltaT * T;
    const double q1 = 1.0 + t * (p.a11 + t * (p.a12 + t * p.a13));
    const double q2 = 1.0 + t * (p.b11 + t * (p.b12 + t * p.b13));
    const double rq = 1.0 / (q1 * q2);
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
// ---------------------------------------------------------------------------
struct LinePlan {
    int n;       // rows per line
    int P;       // partitions (lanes) per line, <= 32; power of two when cyclic
    int m0, rem; // partition p has m0 + (p < rem) rows
    int PS;      // shared-memory stride between partitions (odd)
    int LS;      // shared-memory stride between lines (odd)
    int TL;      // lines per block
    int cyclic;
};

__host__ __device__ __forceinline__ int lp_pos(const LinePlan &lp, int r)
{
    const int big = lp.rem * (lp.m0 + 1);
    int p, q;
    if (r < big) { p = r / (lp.m0 + 1); q = r - p * (lp.m0 + 1); }
    else { const int rr = r - big; p = lp.rem + rr / lp.m0; q = rr - (p - lp.rem) * lp.m0; }
    return p * lp.PS + q;
}

template <int NR>
struct Coef {
    double a, b, c, d[NR];
};

// Solve one line held in shared memory (normalised rows: b == 1).
// A, C: coefficient rows; D: NR right-hand sides spaced by DS.
template <int NR>
__device__ __forceinline__ void warp_solve_line(double *A, double *C, double *D, int DS, const LinePlan &lp, int lane)
{
    const int P = lp.P;
    const bool act = lane < P;
    const int m = act ? lp.m0 + (lane < lp.rem ? 1 : 0) : 0;
    const int base = lane * lp.PS;
    double A0 = 0.0, C0 = 0.0, Am = 0.0, Cm = 0.0, D0[NR], Dm[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) { D0[q] = 0.0; Dm[q] = 0.0; }

    if (act) {
        double *a = A + base, *c = C + base, *d = D + base;
        // forward elimination (rows 0 and 1 are already normalised)
        double am1 = a[1], cm1 = c[1], dm1[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) dm1[q] = d[q * DS + 1];
        for (int r = 2; r < m; r++) {
            const double ar = a[r];
            const double rr = 1.0 / (1.0 - ar * cm1);
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
            double ap1 = a[m - 2], cp1 = c[m - 2], dp1[NR];
#pragma unroll
            for (int q = 0; q < NR; q++) dp1[q] = d[q * DS + m - 2];
            for (int r = m - 3; r >= 1; r--) {
                const double cr = c[r];
#pragma unroll
                for (int q = 0; q < NR; q++) { dp1[q] = d[q * DS + r] - cr * dp1[q]; d[q * DS + r] = dp1[q]; }
                ap1 = a[r] - cr * ap1; a[r] = ap1;
                cp1 = -cr * cp1; c[r] = cp1;
            }
            // closure of row 0 with row 1 (pascal_tdma.f90:531-535)
            const double c0 = c[0];
            const double rr = 1.0 / (1.0 - ap1 * c0);
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = rr * (d[q * DS] - c0 * dp1[q]);
            A0 = rr * a[0];
            C0 = -rr * c0 * cp1;
        } else {
            A0 = a[0]; C0 = c[0];
#pragma unroll
            for (int q = 0; q < NR; q++) D0[q] = d[q * DS];
        }
    }
    const bool cyc = lp.cyclic != 0;
    if (!cyc) {
        if (lane == 0) A0 = 0.0;
        if (lane == P - 1) Cm = 0.0;
    }
    // Fold the 2P-row reduced system onto the first rows of every partition:
    //   alpha z_{p-1} + beta z_p + gamma z_{p+1} = delta,  z_p = x_first(p)
    const int prv = cyc ? ((lane - 1 + P) & (P - 1)) : (lane > 0 ? lane - 1 : 0);
    const double Amp = __shfl_sync(0xffffffffu, Am, prv);
    const double Cmp = __shfl_sync(0xffffffffu, Cm, prv);
    double al = -A0 * Amp;
    double be = 1.0 - A0 * Cmp - C0 * Am;
    double ga = -C0 * Cm;
    double de[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const double Dmp = __shfl_sync(0xffffffffu, Dm[q], prv);
        de[q] = D0[q] - A0 * Dmp - C0 * Dm[q];
    }
    if (!act) { al = 0.0; be = 1.0; ga = 0.0;
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = 0.0; }
    // parallel cyclic reduction across the P lanes
    for (int s = 1; s < P; s <<= 1) {
        int lo = lane - s, hi = lane + s;
        bool lo_ok = true, hi_ok = true;
        if (cyc) { lo = (lo + P) & (P - 1); hi = hi & (P - 1); }
        else { lo_ok = lo >= 0; hi_ok = hi < P; lo = lo_ok ? lo : lane; hi = hi_ok ? hi : lane; }
        double alm = __shfl_sync(0xffffffffu, al, lo), bem = __shfl_sync(0xffffffffu, be, lo), gam = __shfl_sync(0xffffffffu, ga, lo);
        double alp = __shfl_sync(0xffffffffu, al, hi), bep = __shfl_sync(0xffffffffu, be, hi), gap = __shfl_sync(0xffffffffu, ga, hi);
        double dem[NR], dep[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) { dem[q] = __shfl_sync(0xffffffffu, de[q], lo); dep[q] = __shfl_sync(0xffffffffu, de[q], hi); }
        if (!lo_ok) { alm = 0.0; bem = 1.0; gam = 0.0;
#pragma unroll
            for (int q = 0; q < NR; q++) dem[q] = 0.0; }
        if (!hi_ok) { alp = 0.0; bep = 1.0; gap = 0.0;
#pragma unroll
            for (int q = 0; q < NR; q++) dep[q] = 0.0; }
        const double k1 = al / bem, k2 = ga / bep;
        const double nal = -k1 * alm, nga = -k2 * gap;
        const double nbe = be - k1 * gam - k2 * alp;
#pragma unroll
        for (int q = 0; q < NR; q++) de[q] = de[q] - k1 * dem[q] - k2 * dep[q];
        al = nal; be = nbe; ga = nga;
    }
    const double den = 1.0 / (al + be + ga);
    double z[NR], xl[NR];
    const int nxt = cyc ? ((lane + 1) & (P - 1)) : (lane + 1 < 32 ? lane + 1 : lane);
#pragma unroll
    for (int q = 0; q < NR; q++) {
        z[q] = de[q] * den;
        const double zn = __shfl_sync(0xffffffffu, z[q], nxt);
        xl[q] = Dm[q] - Am * z[q] - Cm * zn;
    }
    if (act) {
        double *a = A + base, *c = C + base, *d = D + base;
#pragma unroll
        for (int q = 0; q < NR; q++) { d[q * DS] = z[q]; d[q * DS + m - 1] = xl[q]; }
        for (int r = 1; r < m - 1; r++) {
            const double ar = a[r], cr = c[r];
#pragma unroll
            for (int q = 0; q < NR; q++) d[q * DS + r] = d[q * DS + r] - ar * z[q] - cr * xl[q];
        }
    }
}

// The kernel.  Prob supplies:
//   static constexpr int NRHS;  static constexpr bool CONTIG (rows contiguous in memory);
//   struct State; __device__ State prepare()   -> per-block scalars (dt, stale values)
//   __device__ bool skip(), line_ok(int l)
//   __device__ Coef<NRHS> build(int l, int r, const State &)
//   __device__ void emit(int l, int r, const double *x, const State &)
// TL (lines per block) is a power of two; blockDim.x is 256.
template <class Prob>
__global__ void __launch_bounds__(256, 2) line_solve_kernel(Prob prob, LinePlan lp)
{
    constexpr int NR = Prob::NRHS;
    extern __shared__ double sm[];
    if (prob.skip()) return;
    const typename Prob::State st = prob.prepare();
    const int TL = lp.TL, n = lp.n, LS = lp.LS;
    const int lgTL = __ffs(TL) - 1;
    double *sA = sm, *sC = sA + TL * LS, *sD = sC + TL * LS;
    int *spos = (int *)(sD + NR * TL * LS);
    const int DS = TL * LS;
    // row -> shared-memory position: partition p holds rows start_p .. start_p + m_p - 1
    if (threadIdx.x < lp.P) {
        const int p = threadIdx.x, m = lp.m0 + (p < lp.rem ? 1 : 0);
        const int start = p * lp.m0 + (p < lp.rem ? p : lp.rem);
        for (int q = 0; q < m; q++) spos[start + q] = p * lp.PS + q;
    }
    __syncthreads();
    if (Prob::CONTIG) {
        for (int l = 0; l < TL; l++) {
            const bool ok = prob.line_ok(l);
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const int pos = l * LS + spos[r];
                if (ok) {
                    const Coef<NR> cf = prob.build(l, r, st);
                    const double rb = 1.0 / cf.b;
                    sA[pos] = cf.a * rb; sC[pos] = cf.c * rb;
#pragma unroll
                    for (int q = 0; q < NR; q++) sD[q * DS + pos] = cf.d[q] * rb;
                } else {
                    sA[pos] = 0.0; sC[pos] = 0.0;
#pragma unroll
                    for (int q = 0; q < NR; q++) sD[q * DS + pos] = 0.0;
                }
            }
        }
    } else {
        const int nitems = TL * n;
        for (int t = threadIdx.x; t < nitems; t += blockDim.x) {
            const int r = t >> lgTL, l = t & (TL - 1);
            const int pos = l * LS + spos[r];
            if (prob.line_ok(l)) {
                const Coef<NR> cf = prob.build(l, r, st);
                const double rb = 1.0 / cf.b;
                sA[pos] = cf.a * rb; sC[pos] = cf.c * rb;
#pragma unroll
                for (int q = 0; q < NR; q++) sD[q * DS + pos] = cf.d[q] * rb;
            } else {
                sA[pos] = 0.0; sC[pos] = 0.0;
#pragma unroll
                for (int q = 0; q < NR; q++) sD[q * DS + pos] = 0.0;
            }
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int l = warp; l < TL; l += nw)
        warp_solve_line<NR>(sA + l * LS, sC + l * LS, sD + l * LS, DS, lp, lane);
    __syncthreads();
    if (Prob::CONTIG) {
        for (int l = 0; l < TL; l++) {
            if (!prob.line_ok(l)) continue;
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const int pos = l * LS + spos[r];
                double x[NR];
#pragma unroll
                for (int q = 0; q < NR; q++) x[q] = sD[q * DS + pos];
                prob.emit(l, r, x, st);
            }
        }
    } else {
        const int nitems = TL * n;
        for (int t = threadIdx.x; t < nitems; t += blockDim.x) {
            const int r = t >> lgTL, l = t & (TL - 1);
            if (!prob.line_ok(l)) continue;
            const int pos = l * LS + spos[r];
            double x[NR];
#pragma unroll
            for (int q = 0; q < NR; q++) x[q] = sD[q * DS + pos];
            prob.emit(l, r, x, st);
        }
    }
}

} // namespace tcs
