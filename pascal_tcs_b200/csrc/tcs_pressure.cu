// tcs_pressure.cu -- pressure correction: mpi_pressure_RHS,
// mpi_pressure_Poisson_FFT2 and mpi_pressure_Projection
// (module_solve_pressure.f90:140-231, 489-744, 756-874) on one HBM-resident
// subdomain.  The FFTW calls of the reference (:565-567, 586-588, 660-662,
// 681-683) are replaced by hand-written shared-memory Stockham FFTs with
// radices 2, 3, 4, 5 and 8; the MPI transposes disappear because every pass
// reads the spectral array S(kx, j, kz) (kx fastest) with coalesced tiles.
//
//   prhs_fftx   pseudo-update (+ghosts) -> PRHS -> r2c along x   -> S
//   fftz<-1>    c2c along z (FFTW_FORWARD)                        S -> S
//   modal       y tridiagonal per (kx,kz), re and im together     S -> S
//   mean        unweighted mean of the solution (from the (0,0) mode)
//   fftz<+1>    c2c along z (FFTW_BACKWARD)                       S -> S
//   ifftx       c2r along x, /N1/N3, minus mean, periodic ghosts  S -> dP
//   dp_wall     wall extrapolation of dP (:719-736)
//   projection  U,V,W,P,dPhat,dP0 update (+ghosts, P walls)
//
// In the FP32-mixed form the spectrum S is stored in FP32 but every FFT pass
// computes in FP64 in shared memory, as do the right-hand side (divergence and
// the dPhat correction), the modal solves, the mean, the scaling, the wall
// extrapolations and the projection; each rounds once when it stores.  An
// FP32 FFT has an absolute error of a few ulp of the line's norm in every
// coefficient, and the Poisson solution is dominated by the lowest modes
// (divided by the smallest eigenvalues) while its right-hand side is dominated
// by grid-scale content: measured on the 64^3 case, an FP32 FFT left the
// pressure correction dP with 2e-2 relative error per step.  Rounding each
// FP64-computed coefficient to FP32 keeps every mode, small ones included,
// at FP32 relative accuracy.
#include "tcs_kernels.h"

namespace tcs {

#define IR(jj, kk) ld(f.iR2d + ix2(g, (jj), (kk)))   // FP64 invRho in both forms

template <class C> struct CReal;
template <> struct CReal<double2> { using T = double; };
template <> struct CReal<float2> { using T = float; };

template <class C> __device__ __forceinline__ C cmk(typename CReal<C>::T x, typename CReal<C>::T y) { C c; c.x = x; c.y = y; return c; }
template <class C> __device__ __forceinline__ C cmul(C a, C b) { return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <class C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <class C> __device__ __forceinline__ C cscale(C a, typename CReal<C>::T s) { return cmk<C>(a.x * s, a.y * s); }
// multiply by sign * i
template <int SIGN, class C>
__device__ __forceinline__ C cmuli(C a) { return SIGN > 0 ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x); }

// RX-point DFTs y_q = sum_r v_r exp(SIGN 2 pi i r q / RX), from the definition.
template <int RX, int SIGN, class C> struct Bfly;
template <int SIGN, class C> struct Bfly<2, SIGN, C> {
    __device__ static void run(C *v) { const C a = v[0], b = v[1]; v[0] = cadd(a, b); v[1] = csub(a, b); }
};
template <int SIGN, class C> struct Bfly<4, SIGN, C> {
    __device__ static void run(C *v)
    {
        const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]), c = cadd(v[1], v[3]);
        const C d = cmuli<SIGN>(csub(v[1], v[3]));
        v[0] = cadd(a, c); v[2] = csub(a, c); v[1] = cadd(b, d); v[3] = csub(b, d);
    }
};
template <int SIGN, class C> struct Bfly<3, SIGN, C> {
    __device__ static void run(C *v)
    {
        using T = typename CReal<C>::T;
        const T S3 = T(0.86602540378443864676);   // sin(2 pi / 3)
        const C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        const C m = csub(v[0], cscale(t1, T(0.5)));
        const C r = cmuli<SIGN>(cscale(t2, S3));
        v[0] = cadd(v[0], t1); v[1] = cadd(m, r); v[2] = csub(m, r);
    }
};
template <int SIGN, class C> struct Bfly<5, SIGN, C> {
    __device__ static void run(C *v)
    {
        using T = typename CReal<C>::T;
        const T C1 = T(0.30901699437494742410), C2 = T(-0.80901699437494742410);   // cos(2pi/5), cos(4pi/5)
        const T S1 = T(0.95105651629515357212), S2 = T(0.58778525229247312917);    // sin(2pi/5), sin(4pi/5)
        const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const C a1 = cadd(v[0], cadd(cscale(t1, C1), cscale(t2, C2)));
        const C a2 = cadd(v[0], cadd(cscale(t1, C2), cscale(t2, C1)));
        const C b1 = cmuli<SIGN>(cadd(cscale(t3, S1), cscale(t4, S2)));
        const C b2 = cmuli<SIGN>(csub(cscale(t3, S2), cscale(t4, S1)));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1); v[4] = csub(a1, b1); v[2] = cadd(a2, b2); v[3] = csub(a2, b2);
    }
};

template <int SIGN, class C> struct Bfly<8, SIGN, C> {
    // even and odd halves by 4-point DFTs, joined with the eighth roots of unity
    // w^q = exp(SIGN 2 pi i q / 8): w = (1 + SIGN i) / sqrt 2, w^2 = SIGN i, w^3 = SIGN i w
    __device__ static C w1(C a)
    {
        using T = typename CReal<C>::T;
        const T H = T(0.70710678118654752440);   // 1 / sqrt(2)
        return SIGN > 0 ? cmk<C>((a.x - a.y) * H, (a.x + a.y) * H) : cmk<C>((a.x + a.y) * H, (a.y - a.x) * H);
    }
    __device__ static void run(C *v)
    {
        C e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        Bfly<4, SIGN, C>::run(e);
        Bfly<4, SIGN, C>::run(o);
        o[1] = w1(o[1]);
        o[2] = cmuli<SIGN>(o[2]);
        o[3] = cmuli<SIGN>(w1(o[3]));
#pragma unroll
        for (int q = 0; q < 4; q++) { v[q] = cadd(e[q], o[q]); v[q + 4] = csub(e[q], o[q]); }
    }
};

struct SmemLines {
    double2 *b;
    int NL;
    __device__ double2 ld(int l, int q) const { return b[frow(q) * NL + l]; }
    __device__ void st(int l, int q, double2 v) const { b[frow(q) * NL + l] = v; }
};

// Line accessors made of lambdas (global-memory ends of a block FFT).
template <class F> struct LdFn { F f; __device__ double2 ld(int l, int q) const { return f(l, q); } };
template <class F> struct StFn { F f; __device__ void st(int l, int q, double2 v) const { f(l, q, v); } };
template <class F> __device__ __forceinline__ LdFn<F> ld_fn(F f) { return LdFn<F>{f}; }
template <class F> __device__ __forceinline__ StFn<F> st_fn(F f) { return StFn<F>{f}; }

// The z transforms: one Stockham pass of radix RX over NL lines (NL a power of two): butterfly
// jb of line l reads rows jb + r n/RX through src and writes rows
// o + r Ns, o = (jb / Ns) Ns RX + jb mod Ns, through dst; thread t takes line
// t mod NL and butterfly t / NL.
template <int RX, int SIGN, class Src, class Dst>
__device__ __forceinline__ void fft_pass_lf(const Src &src, const Dst &dst, int NL, int lgNL, int n, int Ns,
                                         const double2 *tw, const FastDiv &dns)
{
    using C = double2;
    const int nb = n / RX, ts = n / (Ns * RX);
    for (int t = threadIdx.x; t < (nb << lgNL); t += blockDim.x) {
        const int l = t & (NL - 1), jb = t >> lgNL;
        const int jq = (int)dns.div(jb), kk = jb - jq * Ns;
        C v[RX];
#pragma unroll
        for (int r = 0; r < RX; r++) v[r] = src.ld(l, jb + r * nb);
        if (kk) {
#pragma unroll
            for (int r = 1; r < RX; r++) {
                C w = __ldg(tw + r * kk * ts);
                if (SIGN > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Bfly<RX, SIGN, C>::run(v);
        const int o = jq * Ns * RX + kk;
#pragma unroll
        for (int r = 0; r < RX; r++) dst.st(l, o + r * Ns, v[r]);
    }
}

// A pass of the plan's radix RX (at most MAXR: the kernels that keep their
// registers for other work compile without the radix-8 butterfly).
template <int SIGN, int MAXR, class Src, class Dst>
__device__ __forceinline__ void fft_pass_any(int RX, const Src &src, const Dst &dst, int NL, int lgNL, int n, int Ns,
                                             const double2 *tw, const FastDiv &dns)
{
    switch (RX) {
    case 8: if constexpr (MAXR >= 8) fft_pass_lf<8, SIGN>(src, dst, NL, lgNL, n, Ns, tw, dns); break;
    case 4: fft_pass_lf<4, SIGN>(src, dst, NL, lgNL, n, Ns, tw, dns); break;
    case 2: fft_pass_lf<2, SIGN>(src, dst, NL, lgNL, n, Ns, tw, dns); break;
    case 3: fft_pass_lf<3, SIGN>(src, dst, NL, lgNL, n, Ns, tw, dns); break;
    default: fft_pass_lf<5, SIGN>(src, dst, NL, lgNL, n, Ns, tw, dns); break;
    }
}

// Unnormalised FFT of NL lines: the first pass reads through src, the last
// writes through dst, and the passes between them go through the two
// shared-memory buffers b0 and b1 (the first pass writes b0, so src may be
// b1).  A barrier follows every pass but the last.
template <int SIGN, int MAXR, class Src, class Dst>
__device__ void block_fft_lf(const Src &src, const Dst &dst, double2 *b0, double2 *b1, int NL, const FFTPlan &fp,
                          const double2 *tw)
{
    const int lgNL = __ffs(NL) - 1, n = fp.n, last = fp.npass - 1;
    if (last == 0) {
        fft_pass_any<SIGN, MAXR>(fp.radix[0], src, dst, NL, lgNL, n, 1, tw, fp.dns[0]);
        return;
    }
    const SmemLines s0{b0, NL}, s1{b1, NL};
    fft_pass_any<SIGN, MAXR>(fp.radix[0], src, s0, NL, lgNL, n, 1, tw, fp.dns[0]);
    __syncthreads();
    int Ns = fp.radix[0];
    bool in0 = true;
    for (int ps = 1; ps < last; ps++) {
        fft_pass_any<SIGN, MAXR>(fp.radix[ps], in0 ? s0 : s1, in0 ? s1 : s0, NL, lgNL, n, Ns, tw, fp.dns[ps]);
        __syncthreads();
        Ns *= fp.radix[ps];
        in0 = !in0;
    }
    fft_pass_any<SIGN, MAXR>(fp.radix[last], in0 ? s0 : s1, dst, NL, lgNL, n, Ns, tw, fp.dns[last]);
}

// The x transforms: lines held line-major (line stride ldl) and staged by the
// kernel, one Stockham pass of radix RX over nl lines per call.
template <int RX, int SIGN, class C>
__device__ __forceinline__ void fft_pass_lm(const C *src, C *dst, int nl, int ldl, int n, int Ns, const C *tw,
                                         const FastDiv &dnb, const FastDiv &dns)
{
    const int nb = n / RX, ts = n / (Ns * RX);
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
        const int l = (int)dnb.div(t), jb = t - l * nb;
        const C *s = src + l * ldl;
        C *d = dst + l * ldl;
        const int jq = (int)dns.div(jb), kk = jb - jq * Ns;
        C v[RX];
#pragma unroll
        for (int r = 0; r < RX; r++) v[r] = s[jb + r * nb];
        if (kk) {
#pragma unroll
            for (int r = 1; r < RX; r++) {
                C w = __ldg(tw + r * kk * ts);
                if (SIGN > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Bfly<RX, SIGN, C>::run(v);
        const int o = jq * Ns * RX + kk;
#pragma unroll
        for (int r = 0; r < RX; r++) d[o + r * Ns] = v[r];
    }
}

// Unnormalised FFT of nl lines held in buf0; buf1 is scratch.  Returns the
// buffer that holds the natural-order result.
template <int SIGN, class C>
__device__ C *block_fft_lm(C *buf0, C *buf1, int nl, int ldl, const FFTPlan &fp, const C *tw)
{
    C *src = buf0, *dst = buf1;
    int Ns = 1;
    for (int ps = 0; ps < fp.npass; ps++) {
        const int RX = fp.radix[ps];
        switch (RX) {
        case 2: fft_pass_lm<2, SIGN>(src, dst, nl, ldl, fp.n, Ns, tw, fp.dnb[ps], fp.dns[ps]); break;
        case 3: fft_pass_lm<3, SIGN>(src, dst, nl, ldl, fp.n, Ns, tw, fp.dnb[ps], fp.dns[ps]); break;
        case 4: fft_pass_lm<4, SIGN>(src, dst, nl, ldl, fp.n, Ns, tw, fp.dnb[ps], fp.dns[ps]); break;
        default: fft_pass_lm<5, SIGN>(src, dst, nl, ldl, fp.n, Ns, tw, fp.dnb[ps], fp.dns[ps]); break;
        }
        __syncthreads();
        C *t = src; src = dst; dst = t;
        Ns *= RX;
    }
    return src;
}

template <class R>
__device__ __forceinline__ long long sidx(const GridT<R> &g, int h1p, int kx, int j, int kz)
{
    TCS_OOB(g.scal, (unsigned)kx >= (unsigned)h1p || (unsigned)(j - 1) >= (unsigned)g.N2 || (unsigned)kz >= (unsigned)g.N3,
            (kx = 0, j = 1, kz = 0));
    return (long long)kx + (long long)h1p * ((long long)(j - 1) + (long long)g.N2 * (long long)kz);
}

// ---------------------------------------------------------------------------
// pseudo-update (:178-208) + ghost(U,V,W) + mpi_pressure_RHS (:182-229) +
// forward r2c FFT along x.  Block: NL lines (j..j+NL-1, k).  The FP64 form
// stores the updated velocities and evaluates the right-hand side from them.
// The FP32 form forms them in FP64 from the velocity's high and low words,
// stores them as such a pair, and evaluates the right-hand side from the FP64
// values, so the divergence carries no storage rounding.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) prhs_fftx_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p, int with_pseudo)
{
    using C = double2;                                 // FFT arithmetic is FP64 in both forms
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int N1 = g.N1, j0 = 1 + blockIdx.x * NL, k = 1 + blockIdx.y;
    const int nfl = (NL + 1) >> 1;                     // packed complex FFT lines
    C *b0 = reinterpret_cast<C *>(smraw), *b1 = b0 + nfl * N1;
    double *su = reinterpret_cast<double *>(b1 + nfl * N1);  // NL x N1 new U along the line
    const double *dx1 = g.d1.dx, *dx2 = g.d2.dx, *dx3 = g.d3.dx;
    const double *rdx1 = g.d1.rdx, *rdx2 = g.d2.rdx, *rdx3 = g.d3.rdx;
    const double *rdmx1 = g.d1.rdmx, *rdmx2 = g.d2.rdmx, *rdmx3 = g.d3.rdmx;
    const int sj = g.P1, sk = g.P1 * g.P2;   // 32-bit offsets (the padded grid is below 2^31 cells): measured 2-3% faster here
    // U..dW are only read here and Un..Wnlo only written, so the reads take the
    // read-only path and the next cell's loads need not wait for these stores.
    for (int t = threadIdx.x; t < NL * N1; t += blockDim.x) {
        const int l = (int)fp.dn.div(t), i = t - l * N1 + 1, j = j0 + l;
        if (j > g.N2) continue;
        const int c = ix(g, i, j, k);
        double un;
        if constexpr (HasLo<R>::on) {
            un = join(ld(f.U + c), ld(f.Ulo + c));
            if (with_pseudo) {
                const double vmask = (j == 1) ? 0.0 : 1.0;
                un += (double)ld(f.dU + c);
                const double vn = join(ld(f.V + c), ld(f.Vlo + c)) + (double)ld(f.dV + c) * vmask;
                const double wn = join(ld(f.W + c), ld(f.Wlo + c)) + (double)ld(f.dW + c);
                float h, lo;
                split(un, h, lo); store_periodic(g, f.Un, i, j, k, h); store_periodic(g, f.Unlo, i, j, k, lo);
                split(vn, h, lo); store_periodic(g, f.Vn, i, j, k, h); store_periodic(g, f.Vnlo, i, j, k, lo);
                split(wn, h, lo); store_periodic(g, f.Wn, i, j, k, h); store_periodic(g, f.Wnlo, i, j, k, lo);
            }
        } else if (with_pseudo) {
            const R u = ld(f.U + c) + ld(f.dU + c);
            const R vmask = (j == 1) ? R(0) : R(1);
            store_periodic(g, f.Un, i, j, k, u);
            store_periodic(g, f.Vn, i, j, k, ld(f.V + c) + ld(f.dV + c) * vmask);
            store_periodic(g, f.Wn, i, j, k, ld(f.W + c) + ld(f.dW + c));
            un = u;
        } else {
            un = ld(f.U + c);
        }
        su[l * N1 + (i - 1)] = un;
    }
    __syncthreads();
    const double dt = g.scal[S_DT], rdt = 1.0 / dt;
    const Phys &p = g.phd;
    const double rdtc = rdt / p.Cmp;   // 1 / (dt Cmp), once per thread
    for (int t = threadIdx.x; t < NL * N1; t += blockDim.x) {
        const int l = (int)fp.dn.div(t), i = t - l * N1 + 1, j = j0 + l;
        // two real lines per complex FFT line: line l is the real (l even) or
        // imaginary (l odd) part of packed line l/2
        double *const slot = reinterpret_cast<double *>(b0) + 2 * ((l >> 1) * N1 + (i - 1)) + (l & 1);
        if (j > g.N2) { *slot = 0.0; continue; }
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const int c = ix(g, i, j, k);
        const double jvm = (j == 1) ? 0.0 : 1.0, jvp = (j == g.N2) ? 0.0 : 1.0;
        const double Uc = su[l * N1 + (i - 1)], Uxp = su[l * N1 + (i == N1 ? 0 : i)];
        double Vc, Vyp, Wc, Wzp;
        const int ckp = (k == g.N3) ? ix(g, i, j, 1) : c + sk;
        if constexpr (HasLo<R>::on) {
            Vc = join(ld(f.V + c), ld(f.Vlo + c)); Vyp = join(ld(f.V + (c + sj)), ld(f.Vlo + (c + sj)));
            Wc = join(ld(f.W + c), ld(f.Wlo + c)); Wzp = join(ld(f.W + ckp), ld(f.Wlo + ckp));
            if (with_pseudo) {
                Vc += (double)ld(f.dV + c) * jvm;
                if (j < g.N2) Vyp += (double)ld(f.dV + (c + sj));
                Wc += (double)ld(f.dW + c);
                Wzp += (double)ld(f.dW + ckp);
            }
        } else if (with_pseudo) {
            Vc = ld(f.V + c) + ld(f.dV + c) * R(jvm);
            Vyp = (j < g.N2) ? ld(f.V + (c + sj)) + ld(f.dV + (c + sj)) : ld(f.V + (c + sj));
            Wc = ld(f.W + c) + ld(f.dW + c);
            Wzp = ld(f.W + ckp) + ld(f.dW + ckp);
        } else {
            Vc = ld(f.V + c); Vyp = ld(f.V + (c + sj)); Wc = ld(f.W + c); Wzp = ld(f.W + ckp);
        }
        const double DivUm = (Uxp - Uc) * rdx1[i] + (jvp * Vyp - jvm * Vc) * rdx2[j] + (Wzp - Wc) * rdx3[k];
        const double cbc = (1.0 - jvm) * p.Vbt * rdx2[j] - (1.0 - jvp) * p.Vup * rdx2[j];
        const R *dPh = f.dPhat;
        const double Pc = ld(dPh + c);
        const double ddpdx1 = (Pc - (double)ld(dPh + (c - 1))) * rdmx1[i], ddpdx2 = ((double)ld(dPh + (c + 1)) - Pc) * rdmx1[ip];
        const double ddpdy3 = (Pc - (double)ld(dPh + (c - sj))) * rdmx2[j], ddpdy4 = ((double)ld(dPh + (c + sj)) - Pc) * rdmx2[jp];
        const double ddpdz5 = (Pc - (double)ld(dPh + (c - sk))) * rdmx3[k], ddpdz6 = ((double)ld(dPh + (c + sk)) - Pc) * rdmx3[kp];
        const double iRjk = IR(j, k);
        const double iR1 = 0.5 * rdmx1[i] * (dx1[im] * iRjk + dx1[i] * iRjk);
        const double iR2_ = 0.5 * rdmx1[ip] * (dx1[ip] * iRjk + dx1[i] * iRjk);
        const double iR3 = 0.5 * rdmx2[j] * (dx2[jm] * iRjk + dx2[j] * (double)IR(jm, k));
        const double iR4 = 0.5 * rdmx2[jp] * (dx2[jp] * iRjk + dx2[j] * (double)IR(jp, k));
        const double iR5 = 0.5 * rdmx3[k] * (dx3[km] * iRjk + dx3[k] * (double)IR(j, km));
        const double iR6 = 0.5 * rdmx3[kp] * (dx3[kp] * iRjk + dx3[k] * (double)IR(j, kp));
        const double Extra = ((1.0 - iR2_) * ddpdx2 - (1.0 - iR1) * ddpdx1) * rdx1[i]
                           + ((1.0 - iR4) * ddpdy4 - (1.0 - iR3) * ddpdy3) * rdx2[j]
                           + ((1.0 - iR6) * ddpdz6 - (1.0 - iR5) * ddpdz5) * rdx3[k];
        *slot = (DivUm - cbc) * rdtc + Extra;
    }
    if (NL & 1)         // an odd line count leaves the last packed line without an imaginary part
        for (int t = threadIdx.x; t < N1; t += blockDim.x) b0[(NL >> 1) * N1 + t].y = 0.0;
    __syncthreads();
    const C *res = block_fft_lm<-1>(b0, b1, nfl, N1, fp, f.tw1);
    // Z = FFT(a + i b) of real a, b: A(k) = (Z(k) + conj Z(N-k)) / 2, B(k) = (Z(k) - conj Z(N-k)) / 2i
    for (int t = threadIdx.x; t < NL * h1p; t += blockDim.x) {
        const int l = (int)fp.dh.div(t), kx = t - l * h1p, j = j0 + l;
        if (j > g.N2) continue;
        const C z = res[(l >> 1) * N1 + kx], zr = res[(l >> 1) * N1 + (kx == 0 ? 0 : N1 - kx)];
        const C v = (l & 1) ? make_double2(0.5 * (z.y + zr.y), 0.5 * (zr.x - z.x))
                            : make_double2(0.5 * (z.x + zr.x), 0.5 * (z.y - zr.y));
        f.S[sidx(g, h1p, kx, j, k - 1)] = mkc<R>(R(v.x), R(v.y));
    }
}

// The split form of the same stage, for a one-radix plan of N1 (512 = 8^3,
// 256 = 4^4): prhs_kernel forms the pseudo-update and the right-hand side one
// cell per thread and stores the right-hand side in FP64 (padded layout, in
// f.prhs); fftx_uniform_kernel transforms its x lines.  The fused kernel above
// keeps the right-hand side in shared memory, but its FFT's registers and
// barriers hold its loads back (measured at 512^3: 3.55 ms FP64, 4.82 ms
// FP32-mixed).  The new U at the x-upper neighbour (periodic) is formed again
// from its inputs with the same arithmetic, so both forms give the same bits.
template <class R>
__global__ void __launch_bounds__(256) prhs_kernel(GridT<R> g, FieldsT<R> f, int with_pseudo)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const double *dx1 = g.d1.dx, *dx2 = g.d2.dx, *dx3 = g.d3.dx;
    const double *rdx1 = g.d1.rdx, *rdx2 = g.d2.rdx, *rdx3 = g.d3.rdx;
    const double *rdmx1 = g.d1.rdmx, *rdmx2 = g.d2.rdmx, *rdmx3 = g.d3.rdmx;
    const int sj = g.P1, sk = g.P1 * g.P2;   // 32-bit offsets (the padded grid is below 2^31 cells)
    const int c = (int)ix(g, i, j, k), cxp = c + ((i == g.N1) ? 1 - g.N1 : 1);
    // the new U at a cell, as the pseudo-update forms it
    auto unew = [&](int cc) -> double {
        if constexpr (HasLo<R>::on) {
            const double u = join(ld(f.U + cc), ld(f.Ulo + cc));
            return with_pseudo ? u + (double)ld(f.dU + cc) : u;
        } else {
            return with_pseudo ? (double)(ld(f.U + cc) + ld(f.dU + cc)) : (double)ld(f.U + cc);
        }
    };
    const double Uc = unew(c), Uxp = unew(cxp);
    const double jvm = (j == 1) ? 0.0 : 1.0, jvp = (j == g.N2) ? 0.0 : 1.0;
    const int ckp = (k == g.N3) ? (int)ix(g, i, j, 1) : c + sk;
    double Vc, Vyp, Wc, Wzp;
    if constexpr (HasLo<R>::on) {
        Vc = join(ld(f.V + c), ld(f.Vlo + c)); Vyp = join(ld(f.V + (c + sj)), ld(f.Vlo + (c + sj)));
        Wc = join(ld(f.W + c), ld(f.Wlo + c)); Wzp = join(ld(f.W + ckp), ld(f.Wlo + ckp));
        if (with_pseudo) {
            Vc += (double)ld(f.dV + c) * jvm;
            if (j < g.N2) Vyp += (double)ld(f.dV + (c + sj));
            Wc += (double)ld(f.dW + c);
            Wzp += (double)ld(f.dW + ckp);
            float h, lo;
            split(Uc, h, lo); store_periodic(g, f.Un, i, j, k, h); store_periodic(g, f.Unlo, i, j, k, lo);
            split(Vc, h, lo); store_periodic(g, f.Vn, i, j, k, h); store_periodic(g, f.Vnlo, i, j, k, lo);
            split(Wc, h, lo); store_periodic(g, f.Wn, i, j, k, h); store_periodic(g, f.Wnlo, i, j, k, lo);
        }
    } else if (with_pseudo) {
        const R vn = ld(f.V + c) + ld(f.dV + c) * R(jvm), wn = ld(f.W + c) + ld(f.dW + c);
        Vc = vn;
        Vyp = (j < g.N2) ? ld(f.V + (c + sj)) + ld(f.dV + (c + sj)) : ld(f.V + (c + sj));
        Wc = wn;
        Wzp = ld(f.W + ckp) + ld(f.dW + ckp);
        store_periodic(g, f.Un, i, j, k, R(Uc));
        store_periodic(g, f.Vn, i, j, k, vn);
        store_periodic(g, f.Wn, i, j, k, wn);
    } else {
        Vc = ld(f.V + c); Vyp = ld(f.V + (c + sj)); Wc = ld(f.W + c); Wzp = ld(f.W + ckp);
    }
    const double dt = g.scal[S_DT], rdt = 1.0 / dt;
    const Phys &p = g.phd;
    const double rdtc = rdt / p.Cmp;
    const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
    const double DivUm = (Uxp - Uc) * rdx1[i] + (jvp * Vyp - jvm * Vc) * rdx2[j] + (Wzp - Wc) * rdx3[k];
    const double cbc = (1.0 - jvm) * p.Vbt * rdx2[j] - (1.0 - jvp) * p.Vup * rdx2[j];
    const R *dPh = f.dPhat;
    const double Pc = ld(dPh + c);
    const double ddpdx1 = (Pc - (double)ld(dPh + (c - 1))) * rdmx1[i], ddpdx2 = ((double)ld(dPh + (c + 1)) - Pc) * rdmx1[ip];
    const double ddpdy3 = (Pc - (double)ld(dPh + (c - sj))) * rdmx2[j], ddpdy4 = ((double)ld(dPh + (c + sj)) - Pc) * rdmx2[jp];
    const double ddpdz5 = (Pc - (double)ld(dPh + (c - sk))) * rdmx3[k], ddpdz6 = ((double)ld(dPh + (c + sk)) - Pc) * rdmx3[kp];
    const double iRjk = IR(j, k);
    const double iR1 = 0.5 * rdmx1[i] * (dx1[im] * iRjk + dx1[i] * iRjk);
    const double iR2_ = 0.5 * rdmx1[ip] * (dx1[ip] * iRjk + dx1[i] * iRjk);
    const double iR3 = 0.5 * rdmx2[j] * (dx2[jm] * iRjk + dx2[j] * (double)IR(jm, k));
    const double iR4 = 0.5 * rdmx2[jp] * (dx2[jp] * iRjk + dx2[j] * (double)IR(jp, k));
    const double iR5 = 0.5 * rdmx3[k] * (dx3[km] * iRjk + dx3[k] * (double)IR(j, km));
    const double iR6 = 0.5 * rdmx3[kp] * (dx3[kp] * iRjk + dx3[k] * (double)IR(j, kp));
    const double Extra = ((1.0 - iR2_) * ddpdx2 - (1.0 - iR1) * ddpdx1) * rdx1[i]
                       + ((1.0 - iR4) * ddpdy4 - (1.0 - iR3) * ddpdy3) * rdx2[j]
                       + ((1.0 - iR6) * ddpdz6 - (1.0 - iR5) * ddpdz5) * rdx3[k];
    f.prhs[c] = (DivUm - cbc) * rdtc + Extra;
}

// The forward r2c x transform of the split form: NL right-hand-side lines
// (j0..j0+NL-1, k) packed two per complex line (real and imaginary parts),
// one butterfly per thread per pass in one line-major buffer, then the
// Hermitian separation into S as in the fused kernel.
template <int RX, class R>
__global__ void __launch_bounds__(512) fftx_uniform_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p)
{
    using C = double2;
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int N1 = g.N1, j0 = 1 + blockIdx.x * NL, k = 1 + blockIdx.y;
    const int nfl = (NL + 1) >> 1, ldl = frow(N1), nb = N1 / RX, lgN1 = __ffs(N1) - 1, lgnb = __ffs(nb) - 1;
    C *const b = reinterpret_cast<C *>(smraw);
    const double *const prhs = f.prhs;
    for (int t = threadIdx.x; t < (nfl << lgN1); t += blockDim.x) {
        const int p = t >> lgN1, q = t & (N1 - 1), ja = j0 + 2 * p;
        const double re = (2 * p < NL && ja <= g.N2) ? ld(prhs + ix(g, q + 1, ja, k)) : 0.0;
        const double im = (2 * p + 1 < NL && ja + 1 <= g.N2) ? ld(prhs + ix(g, q + 1, ja + 1, k)) : 0.0;
        b[p * ldl + frow(q)] = make_double2(re, im);
    }
    __syncthreads();
    const int p = threadIdx.x >> lgnb, jb = threadIdx.x & (nb - 1);
    C *const bl = b + p * ldl;
    C v[RX];
#pragma unroll
    for (int r = 0; r < RX; r++) v[r] = bl[frow(jb + r * nb)];
    Bfly<RX, -1, C>::run(v);            // the first pass: span 1, no twiddles
    int Ns = 1, o = jb * RX;            // span and output base of the pass just computed
    for (int ps = 1; ps < fp.npass; ps++) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RX; r++) bl[frow(o + r * Ns)] = v[r];
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RX; r++) v[r] = bl[frow(jb + r * nb)];
        Ns *= RX;
        const int jq = (int)fp.dns[ps].div(jb), kk = jb - jq * Ns, ts = N1 / (Ns * RX);
        if (kk) {
#pragma unroll
            for (int r = 1; r < RX; r++) v[r] = cmul(v[r], __ldg(f.tw1 + r * kk * ts));
        }
        Bfly<RX, -1, C>::run(v);
        o = jq * Ns * RX + kk;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RX; r++) bl[frow(o + r * Ns)] = v[r];
    __syncthreads();
    // Z = FFT(a + i b) of real a, b: A(k) = (Z(k) + conj Z(N-k)) / 2, B(k) = (Z(k) - conj Z(N-k)) / 2i
    for (int t = threadIdx.x; t < NL * h1p; t += blockDim.x) {
        const int l = (int)fp.dh.div(t), kx = t - l * h1p, j = j0 + l;
        if (j > g.N2) continue;
        const C *const bp = b + (l >> 1) * ldl;
        const C z = bp[frow(kx)], zr = bp[frow(kx == 0 ? 0 : N1 - kx)];
        const C v2 = (l & 1) ? make_double2(0.5 * (z.y + zr.y), 0.5 * (zr.x - z.x))
                             : make_double2(0.5 * (z.x + zr.x), 0.5 * (z.y - zr.y));
        f.S[sidx(g, h1p, kx, j, k - 1)] = mkc<R>(R(v2.x), R(v2.y));
    }
}

// c2c along z for NL consecutive kx at fixed j (NL a power of two): the first
// pass reads S and the last writes it, NL consecutive kx of one kz row per
// group of NL threads.
template <int SIGN, class R>
__global__ void __launch_bounds__(256) fftz_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p)
{
    using C = double2;
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int kx0 = blockIdx.x * NL, j = 1 + blockIdx.y;
    const int nl = min(NL, h1p - kx0);
    C *b0 = reinterpret_cast<C *>(smraw), *b1 = b0 + fft_buf_elems(NL, g.N3);
    cplx_t<R> *const S = f.S;
    auto ld = [&](int l, int kz) -> C {
        if (l >= nl) return make_double2(0.0, 0.0);
        const cplx_t<R> v = S[sidx(g, h1p, kx0 + l, j, kz)];
        return make_double2(v.x, v.y);
    };
    auto st = [&](int l, int kz, C v) {
        if (l < nl) S[sidx(g, h1p, kx0 + l, j, kz)] = mkc<R>(R(v.x), R(v.y));
    };
    block_fft_lf<SIGN, 8>(ld_fn(ld), st_fn(st), b0, b1, NL, fp, f.tw3);
}

// The z transform of a plan whose passes all have radix RX (512 = 8^3,
// 256 = 4^4, 64 = 8^2): one butterfly per thread per pass (blockDim.x =
// NL n / RX), so one shared-memory buffer holds the lines -- a pass writes the
// previous pass's outputs, the block waits, reads its own inputs, waits again
// -- and up to 16 lines per block read and write 16 consecutive kx of a kz row
// (256 bytes in FP64) together.  The first pass reads S, the last writes it.
template <int SIGN, int RX, class R>
__global__ void __launch_bounds__(1024, 1) fftz_uniform_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p)
{
    using C = double2;
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int kx0 = blockIdx.x * NL, j = 1 + blockIdx.y, nl = min(NL, h1p - kx0);
    C *const b = reinterpret_cast<C *>(smraw);
    const int n = fp.n, nb = n / RX, lgNL = __ffs(NL) - 1;
    const int l = threadIdx.x & (NL - 1), jb = threadIdx.x >> lgNL;   // jb < nb
    const bool ok = l < nl;
    cplx_t<R> *const S = f.S;
    C v[RX];
#pragma unroll
    for (int r = 0; r < RX; r++) {
        v[r] = make_double2(0.0, 0.0);
        if (ok) {
            const cplx_t<R> w = S[sidx(g, h1p, kx0 + l, j, jb + r * nb)];
            v[r] = make_double2(w.x, w.y);
        }
    }
    Bfly<RX, SIGN, C>::run(v);          // the first pass: span 1, no twiddles
    int Ns = 1, o = jb * RX;            // span and output base of the pass just computed
    for (int ps = 1; ps < fp.npass; ps++) {
#pragma unroll
        for (int r = 0; r < RX; r++) b[frow(o + r * Ns) * NL + l] = v[r];
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RX; r++) v[r] = b[frow(jb + r * nb) * NL + l];
        __syncthreads();
        Ns *= RX;
        const int jq = (int)fp.dns[ps].div(jb), kk = jb - jq * Ns, ts = n / (Ns * RX);
        if (kk) {
#pragma unroll
            for (int r = 1; r < RX; r++) {
                C w = __ldg(f.tw3 + r * kk * ts);
                if (SIGN > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Bfly<RX, SIGN, C>::run(v);
        o = jq * Ns * RX + kk;
    }
    if (ok) {
#pragma unroll
        for (int r = 0; r < RX; r++) S[sidx(g, h1p, kx0 + l, j, o + r * Ns)] = mkc<R>(R(v[r].x), R(v[r].y));
    }
}

// Modal y solves (:597-652): one tridiagonal system per (kx, kz), real and
// imaginary parts share the matrix.  Mode (0,0) is pinned at j=1; the
// imaginary parts of (0,0) and (0,N3/2) are zeroed after the solve.  The
// rows are FP64 in both forms: the zero and lowest wavenumbers are nearly
// singular, and the FP32 form reads and writes its FP32 spectrum around them.
template <class R, int ITEM = 0>
struct Modal {
    using Real = double;
    static constexpr int NRHS = 2;
    static constexpr bool FAST_RCP = true;    // measured faster with qrcp
    static constexpr int MINB = LineOcc<R>::modal;
    static constexpr int MREG = LineOcc<Real>::reg_modal;
    static constexpr int NT = LineOcc<Real>::nt_modal;
    static constexpr bool CONTIG = false;
    static constexpr bool LINE_PER_THREAD = true;   // measured faster in both forms
    GridT<R> g; FieldsT<R> f; int TL; int h1p;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int lk(int l) const { return vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return lk(l) < h1p; }
    __device__ Coef<double, 2> build(int l, int r, const State &st) const
    {
        const int kx = lk(l), kz = vby<ITEM>(), j = r + 1;
        const double am = f.fam[j], ap = f.fap[j];
        Coef<double, 2> cf;
        const cplx_t<R> s = f.S[sidx(g, h1p, kx, j, kz)];
        if (kx == 0 && kz == 0 && j == 1) {
            cf.a = 0.0; cf.b = 1.0; cf.c = 0.0; cf.d[0] = 0.0; cf.d[1] = s.y;
        } else {
            cf.a = am; cf.c = ap;
            cf.b = (-am - ap) - f.dxk2[kx] - f.dzk[kz];
            cf.d[0] = s.x; cf.d[1] = s.y;
        }
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const
    {
        const int kx = lk(l), kz = vby<ITEM>(), j = r + 1;
        const bool zi = (kx == 0) && (kz == 0 || kz == g.N3 / 2);
        f.S[sidx(g, h1p, kx, j, kz)] = mkc<R>(R(x[0]), zi ? R(0) : R(x[1]));
    }
};

// Unweighted mean of the solution (:703-710): the (i,k) sum of the inverse
// transform of one j-plane is the real part of its (0,0) coefficient.
template <class R>
__global__ void mean_kernel(GridT<R> g, FieldsT<R> f, int h1p)
{
    __shared__ double red[256];
    if (blown(g)) return;
    double s = 0.0;
    for (int j = 1 + threadIdx.x; j <= g.N2; j += blockDim.x) s += (double)f.S[sidx(g, h1p, 0, j, 0)].x;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) g.scal[S_AVER] = red[0] / (double)g.N1 / (double)g.N2 / (double)g.N3;
}

// c2r along x (:681-683) with the scaling (:694-700), the mean removal
// (:712-714) and the periodic ghosts of ghost(dP) (main.f90:189).
template <class R>
__global__ void __launch_bounds__(256) ifftx_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p)
{
    using C = double2;
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int N1 = g.N1, j0 = 1 + blockIdx.x * NL, k = 1 + blockIdx.y;
    C *b0 = reinterpret_cast<C *>(smraw), *b1 = b0 + ((NL + 1) >> 1) * N1;
    // the Hermitian spectrum of line l at kx (zero for lines past the grid)
    auto herm = [&](int l, int kx) -> C {
        const int j = j0 + l;
        C v = make_double2(0.0, 0.0);
        if (l < NL && j <= g.N2) {
            if (kx < h1p) {
                const cplx_t<R> w = f.S[sidx(g, h1p, kx, j, k - 1)];
                v = make_double2(w.x, w.y);
                if (kx == 0 || 2 * kx == N1) v.y = 0.0;   // c2r ignores these imaginary parts
            } else {
                const cplx_t<R> w = f.S[sidx(g, h1p, N1 - kx, j, k - 1)];
                v = make_double2(w.x, -w.y);
            }
        }
        return v;
    };
    // two lines per complex inverse FFT: Z = A + i B gives a + i b with a, b real
    const int nfl = (NL + 1) >> 1;
    for (int t = threadIdx.x; t < nfl * N1; t += blockDim.x) {
        const int p = (int)fp.dn.div(t), kx = t - p * N1;
        const C a = herm(2 * p, kx), b = herm(2 * p + 1, kx);
        b0[t] = make_double2(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    const C *res = block_fft_lm<1>(b0, b1, nfl, N1, fp, f.tw1);
    const double aver = g.scal[S_AVER];
    const double scale = 1.0 / ((double)N1 * (double)g.N3);   // the unnormalised transforms' 1/(N1 N3), once per thread
    for (int t = threadIdx.x; t < NL * N1; t += blockDim.x) {
        const int l = (int)fp.dn.div(t), i = t - l * N1 + 1, j = j0 + l;
        if (j > g.N2) continue;
        const C z = res[(l >> 1) * N1 + (i - 1)];
        const double v = ((l & 1) ? z.y : z.x) * scale - aver;
        store_periodic(g, f.dP, i, j, k, R(v));
    }
}

// The same for a one-radix plan of N1 (radix RX in every pass: 512 = 8^3,
// 256 = 4^4): one butterfly per thread per pass (blockDim.x = packed lines x
// N1 / RX), the packed lines line-major in one shared-memory buffer (row q of
// packed line p at p frow(N1) + frow(q)), and the last pass's outputs, which
// are consecutive i across consecutive threads, scaled and stored to dP from
// registers.
template <int RX, class R>
__global__ void __launch_bounds__(512) ifftx_uniform_kernel(GridT<R> g, FieldsT<R> f, FFTPlan fp, int NL, int h1p)
{
    using C = double2;
    extern __shared__ __align__(16) unsigned char smraw[];
    if (blown(g)) return;
    const int N1 = g.N1, j0 = 1 + blockIdx.x * NL, k = 1 + blockIdx.y;
    const int nfl = (NL + 1) >> 1, ldl = frow(N1), nb = N1 / RX, lgN1 = __ffs(N1) - 1, lgnb = __ffs(nb) - 1;
    C *const b = reinterpret_cast<C *>(smraw);
    auto herm = [&](int l, int kx) -> C {
        const int j = j0 + l;
        C v = make_double2(0.0, 0.0);
        if (l < NL && j <= g.N2) {
            if (kx < h1p) {
                const cplx_t<R> w = f.S[sidx(g, h1p, kx, j, k - 1)];
                v = make_double2(w.x, w.y);
                if (kx == 0 || 2 * kx == N1) v.y = 0.0;   // c2r ignores these imaginary parts
            } else {
                const cplx_t<R> w = f.S[sidx(g, h1p, N1 - kx, j, k - 1)];
                v = make_double2(w.x, -w.y);
            }
        }
        return v;
    };
    // two lines per complex inverse FFT: Z = A + i B gives a + i b with a, b real
    for (int t = threadIdx.x; t < (nfl << lgN1); t += blockDim.x) {
        const int p = t >> lgN1, kx = t & (N1 - 1);
        const C a = herm(2 * p, kx), c = herm(2 * p + 1, kx);
        b[p * ldl + frow(kx)] = make_double2(a.x - c.y, a.y + c.x);
    }
    __syncthreads();
    const int p = threadIdx.x >> lgnb, jb = threadIdx.x & (nb - 1);
    C *const bl = b + p * ldl;
    C v[RX];
#pragma unroll
    for (int r = 0; r < RX; r++) v[r] = bl[frow(jb + r * nb)];
    Bfly<RX, 1, C>::run(v);             // the first pass: span 1, no twiddles
    int Ns = 1, o = jb * RX;            // span and output base of the pass just computed
    for (int ps = 1; ps < fp.npass; ps++) {
        __syncthreads();                // every thread has read the previous pass's inputs
#pragma unroll
        for (int r = 0; r < RX; r++) bl[frow(o + r * Ns)] = v[r];
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RX; r++) v[r] = bl[frow(jb + r * nb)];
        Ns *= RX;
        const int jq = (int)fp.dns[ps].div(jb), kk = jb - jq * Ns, ts = N1 / (Ns * RX);
        if (kk) {
#pragma unroll
            for (int r = 1; r < RX; r++) {
                C w = __ldg(f.tw1 + r * kk * ts);
                w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Bfly<RX, 1, C>::run(v);
        o = jq * Ns * RX + kk;
    }
    const double aver = g.scal[S_AVER];
    const double scale = 1.0 / ((double)N1 * (double)g.N3);   // the unnormalised transforms' 1/(N1 N3), once per thread
    const int ja = j0 + 2 * p, jbm = ja + 1;
    const bool oka = 2 * p < NL && ja <= g.N2, okb = 2 * p + 1 < NL && jbm <= g.N2;
#pragma unroll
    for (int r = 0; r < RX; r++) {
        const int i = o + r * Ns + 1;
        if (oka) store_periodic(g, f.dP, i, ja, k, R(v[r].x * scale - aver));
        if (okb) store_periodic(g, f.dP, i, jbm, k, R(v[r].y * scale - aver));
    }
}

// dP wall extrapolation (:719-736) on every (i,k) including ghost columns,
// which is what the extrapolation followed by ghost(dP) produces.
template <class R>
__global__ void dp_wall_kernel(GridT<R> g, FieldsT<R> f, double ab, double bb, double at, double bt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i > g.N1 + 1 || blown(g)) return;
    R *dP = f.dP;
    dP[ix(g, i, 0, k)] = R(ab * (double)dP[ix(g, i, 1, k)] - bb * (double)dP[ix(g, i, 2, k)]);
    dP[ix(g, i, g.N2 + 1, k)] = R(at * (double)dP[ix(g, i, g.N2, k)] - bt * (double)dP[ix(g, i, g.N2 - 1, k)]);
}

// ---------------------------------------------------------------------------
// mpi_pressure_Projection (:756-874) + ghost(U,V,W,P,dPhat), one thread per
// cell, in FP64 arithmetic in both forms.  The reference sweeps k, then
// j = 2..N2, then j = 1, with i innermost, updating dPhat in place, so the
// pressure-correction term of a cell reads the NEW dPhat of its x-lower
// neighbour (i >= 2), of its y-lower neighbour (j >= 3) and of its z-lower
// neighbour (k >= 2), and the old value otherwise.  New values are
// recomputed from the old ones with the same arithmetic
// (dP0n = (dPhat + dP0)/2, dPhatn = 2 dP - dP0n) and written to the second
// buffers.  The P wall rows (:853-869) follow in p_wall_kernel.
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ double new_phat(const FieldsT<R> &f, long long n)
{
    // the FP32 form rounds dP0n to the stored type first, as the neighbour itself does
    const R dp0n = R(((double)ld(f.dPhat + n) + (double)ld(f.dP0 + n)) / 2.0);
    return (double)R(2.0 * (double)ld(f.dP + n) - (double)dp0n);
}

template <class R>
__global__ void __launch_bounds__(256) projection_kernel(GridT<R> g, FieldsT<R> f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const int im = i - 1, jm = j - 1, km = k - 1;
    const double *dx1 = g.d1.dx, *dx2 = g.d2.dx, *dx3 = g.d3.dx;
    const double *rdmx1 = g.d1.rdmx, *rdmx2 = g.d2.rdmx, *rdmx3 = g.d3.rdmx;
    const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
    const double dtc = g.scal[S_DT] * g.phd.Cmp;
    const double dPc = ld(f.dP + c), ph = ld(f.dPhat + c), p0 = ld(f.dP0 + c);
    const R dp0n = R((ph + p0) / 2.0);
    const R phn = R(2.0 * dPc - (double)dp0n);
    const double iRjk = IR(j, k);
    const double Xim = (i >= 2) ? new_phat(f, c - 1) : (double)ld(f.dPhat + c - 1);
    double invRhoc = 0.5 * rdmx1[i] * (dx1[i] * iRjk + dx1[im] * iRjk);
    double u0, v0, w0;       // the velocity after the pseudo-update (FP64 from the pair in the FP32 form)
    if constexpr (HasLo<R>::on) {
        u0 = join(f.U[c], f.Ulo[c]); v0 = join(f.V[c], f.Vlo[c]); w0 = join(f.W[c], f.Wlo[c]);
    } else {
        u0 = f.U[c]; v0 = f.V[c]; w0 = f.W[c];
    }
    const double un = u0 - dtc * ((dPc - (double)ld(f.dP + c - 1)) * rdmx1[i] + (invRhoc - 1.0) * (ph - Xim) * rdmx1[i]);
    double vn = v0;
    if (j >= 2) {   // the lower wall plane keeps V: dble(2 - j_indexS) = 0
        const double Xjm = (j >= 3) ? new_phat(f, c - sj) : (double)ld(f.dPhat + c - sj);
        invRhoc = 0.5 * rdmx2[j] * (dx2[j] * (double)IR(jm, k) + dx2[jm] * iRjk);
        vn = vn - dtc * ((dPc - (double)ld(f.dP + c - sj)) * rdmx2[j] + (invRhoc - 1.0) * (ph - Xjm) * rdmx2[j]);
    }
    const double Xkm = (k >= 2) ? new_phat(f, c - sk) : (double)ld(f.dPhat + c - sk);
    invRhoc = 0.5 * rdmx3[k] * (dx3[k] * (double)IR(j, km) + dx3[km] * iRjk);
    const double wn = w0 - dtc * ((dPc - (double)ld(f.dP + c - sk)) * rdmx3[k] + (invRhoc - 1.0) * (ph - Xkm) * rdmx3[k]);
    if constexpr (HasLo<R>::on) {
        float h, lo;
        split(un, h, lo); store_periodic(g, f.U, i, j, k, h); store_periodic(g, f.Ulo, i, j, k, lo);
        split(vn, h, lo); store_periodic(g, f.V, i, j, k, h); store_periodic(g, f.Vlo, i, j, k, lo);
        split(wn, h, lo); store_periodic(g, f.W, i, j, k, h); store_periodic(g, f.Wlo, i, j, k, lo);
    } else {
        store_periodic(g, f.U, i, j, k, R(un));
        store_periodic(g, f.V, i, j, k, R(vn));
        store_periodic(g, f.W, i, j, k, R(wn));
    }
    store_periodic(g, f.P, i, j, k, R((double)f.P[c] + dPc));
    store_periodic(g, f.dPhatn, i, j, k, phn);
    f.dP0n[c] = dp0n;
}

// P(i,0,k) = Pbc_a P(i,1,k) - Pbc_b P(i,2,k) and the top-wall counterpart
// (:853-869), then ghost(P).
template <class R>
__global__ void p_wall_kernel(GridT<R> g, FieldsT<R> f, double ab, double bb, double at, double bt)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, k = 1 + blockIdx.y;
    if (i > g.N1 || blown(g)) return;
    const R *P = f.P;
    store_periodic(g, f.P, i, 0, k, R(ab * (double)P[ix(g, i, 1, k)] - bb * (double)P[ix(g, i, 2, k)]));
    store_periodic(g, f.P, i, g.N2 + 1, k, R(at * (double)P[ix(g, i, g.N2, k)] - bt * (double)P[ix(g, i, g.N2 - 1, k)]));
}

template <class R>
static size_t fftx_smem(const Ctx<R> &cx)
{
    // two packed FFT buffers of (lines + 1) / 2 complex lines, and the new U of every line
    return (size_t)((cx.fft_lines_x + 1) / 2) * cx.g.N1 * 2 * sizeof(double2) + (size_t)cx.fft_lines_x * cx.g.N1 * sizeof(double);
}

template <class R>
void launch_pseudo_prhs_fftx(const Ctx<R> &cx, cudaStream_t s, bool with_pseudo)
{
    const GridT<R> &g = cx.g;
    const int NL = cx.fft_lines_x;
    if (cx.f.prhs && ifftx_form(cx.fp1u, NL) == 1) {   // the split form
        const size_t sm = ifftx_smem(cx.fp1u, NL, 1);
        const int nt = ((NL + 1) / 2) * (g.N1 / cx.fp1u.radix[0]);
        const dim3 gx((g.N2 + NL - 1) / NL, g.N3);
        static size_t c8[64] = {}, c4[64] = {};
        probe_begin(cx, K_PRHS_FFTX, s);
        prhs_kernel<R><<<dim3((g.N1 + 255) / 256, g.N2, g.N3), 256, 0, s>>>(g, cx.f, with_pseudo ? 1 : 0);
        record_launch_error("prhs");
        if (cx.fp1u.radix[0] == 8) {
            smem_opt_in((const void *)fftx_uniform_kernel<8, R>, sm, c8);
            fftx_uniform_kernel<8, R><<<gx, nt, sm, s>>>(g, cx.f, cx.fp1u, NL, cx.h1p);
        } else {
            smem_opt_in((const void *)fftx_uniform_kernel<4, R>, sm, c4);
            fftx_uniform_kernel<4, R><<<gx, nt, sm, s>>>(g, cx.f, cx.fp1u, NL, cx.h1p);
        }
        probe_end(cx, K_PRHS_FFTX, s);
        record_launch_error("fftx");
        return;
    }
    const size_t sm = fftx_smem(cx);
    static size_t conf[64] = {};
    smem_opt_in((const void *)prhs_fftx_kernel<R>, sm, conf);
    probe_begin(cx, K_PRHS_FFTX, s);
    prhs_fftx_kernel<R><<<dim3((g.N2 + NL - 1) / NL, g.N3), 256, sm, s>>>(g, cx.f, cx.fp1, NL, cx.h1p, with_pseudo ? 1 : 0);
    probe_end(cx, K_PRHS_FFTX, s);
    record_launch_error("prhs_fftx");
}

// A z transform: the one-radix form where the plan and the lines per block
// allow it (fftz_form), the general form otherwise.
template <int SIGN, class R>
static void launch_fftz(const Ctx<R> &cx, cudaStream_t s, int kid, const char *what)
{
    const GridT<R> &g = cx.g;
    const int h1p = cx.h1p, NL = cx.fft_lines_z, form = fftz_form(cx.fp3, NL);
    const dim3 grid((h1p + NL - 1) / NL, g.N2);
    probe_begin(cx, kid, s);
    if (form == 1) {
        const int rx = cx.fp3.radix[0];
        const size_t sm = fftz_smem(cx.fp3, NL, 1);
        static size_t c8[64] = {}, c4[64] = {};
        if (rx == 8) {
            smem_opt_in((const void *)fftz_uniform_kernel<SIGN, 8, R>, sm, c8);
            fftz_uniform_kernel<SIGN, 8, R><<<grid, NL * g.N3 / 8, sm, s>>>(g, cx.f, cx.fp3, NL, h1p);
        } else {
            smem_opt_in((const void *)fftz_uniform_kernel<SIGN, 4, R>, sm, c4);
            fftz_uniform_kernel<SIGN, 4, R><<<grid, NL * g.N3 / 4, sm, s>>>(g, cx.f, cx.fp3, NL, h1p);
        }
    } else {
        const size_t sm = fftz_smem(cx.fp3, NL, 2);
        static size_t cz[64] = {};
        smem_opt_in((const void *)fftz_kernel<SIGN, R>, sm, cz);
        fftz_kernel<SIGN, R><<<grid, 256, sm, s>>>(g, cx.f, cx.fp3, NL, h1p);
    }
    probe_end(cx, kid, s);
    record_launch_error(what);
}

// The Poisson solve after the right-hand side, in three parts so that an
// ensemble can run the modal solves of all its cases in one launch.
template <class R>
void launch_poisson_fwd(const Ctx<R> &cx, cudaStream_t s)
{
    launch_fftz<-1>(cx, s, K_FFTZ_FWD, "fftz_fwd");
}

template <class R>
void launch_modal(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    if (cx.y_solver == 4 && cx.thomas_scr) {   // FP64 rows in both forms: the one-line-per-thread solver
        launch_thomas<Modal<R>>(cx, g.N2, cx.h1p, g.N3, [&](int tl) { return Modal<R>{g, cx.f, tl, cx.h1p}; }, s, K_MODAL);
        return;
    }
    LinePlan pm = plan_for<Modal<R>>(g.N2, false, fit_tl<Modal<R>>(g.N2, false, cx.tl_modal, cx.lanes), cx.lanes);
    launch_lines(Modal<R>{g, cx.f, pm.TL, cx.h1p}, pm, dim3((cx.h1p + pm.TL - 1) / pm.TL, g.N3), s, K_MODAL, cx);
}

template <class R>
void launch_poisson_back(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    const int h1p = cx.h1p, NLx = cx.ifft_lines_x, form = ifftx_form(cx.fp1u, NLx);
    probe_begin(cx, K_MEAN, s);
    mean_kernel<R><<<1, 256, 0, s>>>(g, cx.f, h1p);
    probe_end(cx, K_MEAN, s);
    record_launch_error("mean");
    launch_fftz<1>(cx, s, K_FFTZ_INV, "fftz_inv");
    probe_begin(cx, K_IFFTX, s);
    const dim3 gx((g.N2 + NLx - 1) / NLx, g.N3);
    const size_t smx = ifftx_smem(cx.fp1u, NLx, form);
    if (form == 1) {
        const int nt = ((NLx + 1) / 2) * (g.N1 / cx.fp1u.radix[0]);
        static size_t c8[64] = {}, c4[64] = {};
        if (cx.fp1u.radix[0] == 8) {
            smem_opt_in((const void *)ifftx_uniform_kernel<8, R>, smx, c8);
            ifftx_uniform_kernel<8, R><<<gx, nt, smx, s>>>(g, cx.f, cx.fp1u, NLx, h1p);
        } else {
            smem_opt_in((const void *)ifftx_uniform_kernel<4, R>, smx, c4);
            ifftx_uniform_kernel<4, R><<<gx, nt, smx, s>>>(g, cx.f, cx.fp1u, NLx, h1p);
        }
    } else {
        static size_t cx2[64] = {};
        smem_opt_in((const void *)ifftx_kernel<R>, smx, cx2);
        ifftx_kernel<R><<<gx, 256, smx, s>>>(g, cx.f, cx.fp1, NLx, h1p);
    }
    probe_end(cx, K_IFFTX, s);
    record_launch_error("ifftx");
    probe_begin(cx, K_DP_WALL, s);
    dp_wall_kernel<R><<<dim3((g.N1 + 2 + 127) / 128, g.N3 + 2), 128, 0, s>>>(g, cx.f, cx.wall_ab, cx.wall_bb, cx.wall_at, cx.wall_bt);
    probe_end(cx, K_DP_WALL, s);
    record_launch_error("dp_wall");
}

template <class R>
void launch_poisson_rest(const Ctx<R> &cx, cudaStream_t s)
{
    launch_poisson_fwd(cx, s);
    launch_modal(cx, s);
    launch_poisson_back(cx, s);
}

template <class R>
void launch_projection(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    probe_begin(cx, K_PROJECT, s);
    projection_kernel<R><<<dim3((g.N1 + 255) / 256, g.N2, g.N3), 256, 0, s>>>(g, cx.f);
    probe_end(cx, K_PROJECT, s);
    record_launch_error("projection");
    probe_begin(cx, K_P_WALL, s);
    p_wall_kernel<R><<<dim3((g.N1 + 127) / 128, g.N3), 128, 0, s>>>(g, cx.f, cx.wall_ab, cx.wall_bb, cx.wall_at, cx.wall_bt);
    probe_end(cx, K_P_WALL, s);
    record_launch_error("p_wall");
}

#undef IR

// the two forms
// The modal solves of many cases in one launch.
template <class R>
void launch_modal_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s)
{
    multi_stage<Modal<R, 1>>(cs, A, s, "modal",
        [](const Ctx<R> &x) { return StageShape{x.g.N2, false, x.tl_modal, x.h1p, x.g.N3}; },
        [](const Ctx<R> &x, int tl) { return Modal<R, 1>{x.g, x.f, tl, x.h1p}; });
}

template void launch_modal_multi<double>(const std::vector<Ctx<double> *> &, MultiArena &, cudaStream_t);
template void launch_modal_multi<float>(const std::vector<Ctx<float> *> &, MultiArena &, cudaStream_t);
template void launch_modal<double>(const Ctx<double> &, cudaStream_t);
template void launch_modal<float>(const Ctx<float> &, cudaStream_t);
template void launch_pseudo_prhs_fftx<double>(const Ctx<double> &, cudaStream_t, bool);
template void launch_pseudo_prhs_fftx<float>(const Ctx<float> &, cudaStream_t, bool);
template void launch_poisson_rest<double>(const Ctx<double> &, cudaStream_t);
template void launch_poisson_rest<float>(const Ctx<float> &, cudaStream_t);
template void launch_poisson_fwd<double>(const Ctx<double> &, cudaStream_t);
template void launch_poisson_fwd<float>(const Ctx<float> &, cudaStream_t);
template void launch_poisson_back<double>(const Ctx<double> &, cudaStream_t);
template void launch_poisson_back<float>(const Ctx<float> &, cudaStream_t);
template void launch_projection<double>(const Ctx<double> &, cudaStream_t);
template void launch_projection<float>(const Ctx<float> &, cudaStream_t);

} // namespace tcs
