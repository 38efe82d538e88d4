// tcs_thermal.cu -- energy equation: mpi_thermal_coeffi + mpi_thermal_solver
// (module_solve_thermal.f90:116-532) as three fused kernels, one per ADI
// sweep.  Each kernel evaluates the temperature-dependent properties at the
// stencil points it needs, builds the tridiagonal rows straight into shared
// memory and solves its lines there; only the sweep result goes to HBM.
//
//   z sweep  (:236-366) lines (i,j), rows k, cyclic   -> R
//   x sweep  (:388-434) lines (j,k), rows i, cyclic   R -> R
//   y sweep  (:456-524) lines (i,k), rows j           R -> Tn = T + R (+ ghosts)
//
// Divisions by metric quantities are multiplications by reciprocal tables.
#include "tcs_kernels.h"

namespace tcs {

template <class R, int ITEM = 0>
struct ThermalZ {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = true;    // measured faster with qrcp
    static constexpr int MINB = LineOcc<R>::z;
    static constexpr int MREG = LineOcc<Real>::reg_z;
    static constexpr int NT = LineOcc<Real>::nt_z;
    static constexpr bool CONTIG = false;
    static constexpr bool PAIR = LineOcc<Real>::pair_z;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt; };
    __device__ State prepare() const { return State{R(g.scal[S_DT])}; }
    __device__ int li(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    // The right-hand side of :236-361 is the explicit operator minus the three
    // implicit operators applied to T.  Expanded, per direction d with faces
    // -/+ (kPP the face conductivity, ded the face gradient, u the face
    // velocity), the dK/dT products (e dkPP ded) of the explicit operator and
    // of the implicit one cancel, and so do the two dh Tc dv terms, leaving
    //   2 h rdx_d (kPP+ ded+ - kPP- ded-) - (u- ded- + u+ ded+) / 2.
    // This build evaluates that reduced form (the same value in exact
    // arithmetic, about half the arithmetic), except for the y direction on the
    // two wall-adjacent planes (j = 1, N2), where the jC_BC masks and the wall
    // terms keep the reference's full expression.  The z rows (am, ac, ap) are
    // the reference's, dK/dT terms included.
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 1 + vby<ITEM>(), k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const PhysT<R> &p = g.ph;
        const bool d2 = g.kdeg2 != 0;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const R *T = f.T;
        const R Tc = ld(T + c), Txm = ld(T + c - 1), Txp = ld(T + c + 1);
        const R Tym = ld(T + c - sj), Typ = ld(T + c + sj), Tzm = ld(T + c - sk), Tzp = ld(T + c + sk);
        R Kc, dKc, Kzm, dKzm, Kzp, dKzp, irc, dirc;
        kpp_eval(p, d2, Tc, Kc, dKc); kpp_eval(p, d2, Tzm, Kzm, dKzm); kpp_eval(p, d2, Tzp, Kzp, dKzp);
        const R Kxm = kpp_only(p, d2, Txm), Kxp = kpp_only(p, d2, Txp);
        rhocp_eval(p, Tc, irc, dirc);
        const bool wall = j == 1 || j == g.N2;
        const R Uc = ld(f.U + c), Uxp = ld(f.U + c + 1), Vc = ld(f.V + c), Vyp = ld(f.V + c + sj);
        const R Wc = ld(f.W + c), Wzp = ld(f.W + c + sk);
        const R h = R(0.5) * p.Ct * irc, dh = R(0.5) * p.Ct * dirc;
        const R dedx1 = (Tc - Txm) * rdmx1[i], dedx2 = (Txp - Tc) * rdmx1[ip];
        const R dedy3 = (Tc - Tym) * rdmx2[j], dedy4 = (Typ - Tc) * rdmx2[jp];
        const R dedz5 = (Tc - Tzm) * rdmx3[k], dedz6 = (Tzp - Tc) * rdmx3[kp];
        const R kPP1 = R(0.5) * rdmx1[i] * (dx1[i] * Kxm + dx1[im] * Kc), kPP2 = R(0.5) * rdmx1[ip] * (dx1[ip] * Kc + dx1[i] * Kxp);
        const R kPP5 = R(0.5) * rdmx3[k] * (dx3[k] * Kzm + dx3[km] * Kc), kPP6 = R(0.5) * rdmx3[kp] * (dx3[kp] * Kc + dx3[k] * Kzp);
        const R dkPP5 = R(0.5) * rdmx3[k] * (dx3[k] * dKzm + dx3[km] * dKc), dkPP6 = R(0.5) * rdmx3[kp] * (dx3[kp] * dKc + dx3[k] * dKzp);
        const R fx = kPP2 * dedx2 - kPP1 * dedx1, fz = kPP6 * dedz6 - kPP5 * dedz5;
        R rhs = R(2) * h * (fx * rdx1[i] + fz * rdx3[k]) - R(0.5) * (Uc * dedx1 + Uxp * dedx2) - R(0.5) * (Wc * dedz5 + Wzp * dedz6);
        R fy;
        if (!wall) {
            const R Kym = kpp_only(p, d2, Tym), Kyp = kpp_only(p, d2, Typ);
            const R kPP3 = R(0.5) * rdmx2[j] * (dx2[j] * Kym + dx2[jm] * Kc), kPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * Kc + dx2[j] * Kyp);
            fy = kPP4 * dedy4 - kPP3 * dedy3;
            rhs = rhs + R(2) * h * fy * rdx2[j] - R(0.5) * (Vc * dedy3 + Vyp * dedy4);
        } else {
            // the reference's y terms: convection, h ve2, the wall terms, minus the implicit y operator on T
            R Kym, dKym, Kyp, dKyp;
            kpp_eval(p, d2, Tym, Kym, dKym); kpp_eval(p, d2, Typ, Kyp, dKyp);
            const R jem = (j == 1) ? R(0.0) : R(1.0), jep = (j == g.N2) ? R(0.0) : R(1.0);   // jC_BC(jm), jC_BC(jp)
            const R e3 = (dx2[j] * Tym + dx2[jm] * Tc) * (R(0.5) * rdmx2[j]);
            const R e4 = (dx2[jp] * Tc + dx2[j] * Typ) * (R(0.5) * rdmx2[jp]);
            const R kPP3 = R(0.5) * rdmx2[j] * (dx2[j] * Kym + dx2[jm] * Kc), kPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * Kc + dx2[j] * Kyp);
            const R dkPP3 = R(0.5) * rdmx2[j] * (dx2[j] * dKym + dx2[jm] * dKc), dkPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * dKc + dx2[j] * dKyp);
            fy = kPP4 * dedy4 - kPP3 * dedy3;
            const R ve2 = (kPP4 * dedy4 - kPP3 * dedy3 - e4 * dkPP4 * dedy4 + e3 * dkPP3 * dedy3) * rdx2[j];
            R ebc_up = -R(0.25) * Vyp * rdmx2[jp] * p.Tup;
            R ebc_dn = R(0.25) * Vc * rdmx2[j] * p.Tbt;
            ebc_up = ebc_up + h * rdx2[j] * kPP4 * rdmx2[jp] * p.Tup + h * rdx2[j] * dkPP4 * dedy4 * p.Tup;
            ebc_dn = ebc_dn + h * rdx2[j] * kPP3 * rdmx2[j] * p.Tbt - h * rdx2[j] * dkPP3 * dedy3 * p.Tbt;
            const R eACJ = h * rdx2[j] * (kPP4 * rdmx2[jp] + kPP3 * rdmx2[j] - dx2[jp] * (R(0.5) * rdmx2[jp]) * dkPP4 * dedy4 * jep + dx2[jm] * (R(0.5) * rdmx2[j]) * dkPP3 * dedy3 * jem)
                              + (R(0.25) * Vc * rdmx2[j] - R(0.25) * Vyp * rdmx2[jp]);
            const R eAPJ = (-h * rdx2[j] * (kPP4 * rdmx2[jp] + dx2[j] * (R(0.5) * rdmx2[jp]) * dkPP4 * dedy4) + R(0.25) * Vyp * rdmx2[jp]) * jep;
            const R eAMJ = (-h * rdx2[j] * (kPP3 * rdmx2[j] - dx2[j] * (R(0.5) * rdmx2[j]) * dkPP3 * dedy3) - R(0.25) * Vc * rdmx2[j]) * jem;
            rhs = rhs - R(0.25) * (Vc * dedy3 + Vyp * dedy4) + h * ve2 + (R(1.0) - jem) * ebc_dn + (R(1.0) - jep) * ebc_up
                  - (eAPJ * Typ + eACJ * Tc + eAMJ * Tym);
        }
        const R dv = fx * rdx1[i] + fy * rdx2[j] + fz * rdx3[k];
        const R eACK = h * rdx3[k] * (kPP6 * rdmx3[kp] + kPP5 * rdmx3[k] - dx3[kp] * (R(0.5) * rdmx3[kp]) * dkPP6 * dedz6 + dx3[km] * (R(0.5) * rdmx3[k]) * dkPP5 * dedz5)
                          + (-R(0.25) * Wzp * rdmx3[kp] + R(0.25) * Wc * rdmx3[k]);
        const R eAPK = -h * rdx3[k] * (kPP6 * rdmx3[kp] + dx3[k] * (R(0.5) * rdmx3[kp]) * dkPP6 * dedz6) + R(0.25) * Wzp * rdmx3[kp];
        const R eAMK = -h * rdx3[k] * (kPP5 * rdmx3[k] - dx3[k] * (R(0.5) * rdmx3[k]) * dkPP5 * dedz5) - R(0.25) * Wc * rdmx3[k];
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = eACK * dt - R(0.5) * dh * dv * dt + R(1.0);
        cf.c = eAPK * dt;
        cf.a = eAMK * dt;
        cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const
    {
        f.scr[ix(g, li(l), 1 + vby<ITEM>(), r + 1)] = x[0];
    }
};

// Stage 2 (:388-429): jm, jp, km, kp keep the values of the last stage-1
// iteration (N2-1, N2+1, N3-1, N3+1).
template <class R, int WIDE = 0, int ITEM = 0>
struct ThermalX {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = true;    // measured faster with qrcp
    static constexpr int MINB = WIDE ? LineOcc<R>::xw : LineOcc<R>::x;
    static constexpr int MREG = WIDE ? LineOcc<Real>::reg_xw : LineOcc<Real>::reg_x;
    static constexpr int NT = WIDE ? LineOcc<Real>::nt_xw : LineOcc<Real>::nt_x;
    static constexpr bool CONTIG = true;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt; };
    __device__ State prepare() const { return State{R(g.scal[S_DT])}; }
    __device__ int lj(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + vby<ITEM>();
        const int im = i - 1, ip = i + 1, jm = g.N2 - 1, jp = g.N2 + 1, km = g.N3 - 1, kp = g.N3 + 1;
        const PhysT<R> &p = g.ph;
        const bool d2 = g.kdeg2 != 0;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k);
        const R *T = f.T;
        const R Tc = ld(T + c), Txm = ld(T + c - 1), Txp = ld(T + c + 1);
        const R Tjm = ld(T + ix(g, i, jm, k)), Tjp = ld(T + ix(g, i, jp, k));
        const R Tkm = ld(T + ix(g, i, j, km)), Tkp = ld(T + ix(g, i, j, kp));
        R Kc, dKc, Kxm, dKxm, Kxp, dKxp, irc, dirc;
        kpp_eval(p, d2, Tc, Kc, dKc); kpp_eval(p, d2, Txm, Kxm, dKxm); kpp_eval(p, d2, Txp, Kxp, dKxp);
        const R Kjm = kpp_only(p, d2, Tjm), Kjp = kpp_only(p, d2, Tjp), Kkm = kpp_only(p, d2, Tkm), Kkp = kpp_only(p, d2, Tkp);
        rhocp_eval(p, Tc, irc, dirc);
        const R h = R(0.5) * p.Ct * irc;
        const R kPP1 = R(0.5) * rdmx1[i] * (dx1[i] * Kxm + dx1[im] * Kc), kPP2 = R(0.5) * rdmx1[ip] * (dx1[ip] * Kc + dx1[i] * Kxp);
        const R kPP3 = R(0.5) * rdmx2[j] * (dx2[j] * Kjm + dx2[jm] * Kc), kPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * Kc + dx2[j] * Kjp);
        const R kPP5 = R(0.5) * rdmx3[k] * (dx3[k] * Kkm + dx3[km] * Kc), kPP6 = R(0.5) * rdmx3[kp] * (dx3[kp] * Kc + dx3[k] * Kkp);
        const R dkPP1 = R(0.5) * rdmx1[i] * (dx1[i] * dKxm + dx1[im] * dKc), dkPP2 = R(0.5) * rdmx1[ip] * (dx1[ip] * dKc + dx1[i] * dKxp);
        const R dedx1 = (Tc - Txm) * rdmx1[i], dedx2 = (Txp - Tc) * rdmx1[ip];
        const R dedy3 = (Tc - Tjm) * rdmx2[j], dedy4 = (Tjp - Tc) * rdmx2[jp];
        const R dedz5 = (Tc - Tkm) * rdmx3[k], dedz6 = (Tkp - Tc) * rdmx3[kp];
        const R Uc = ld(f.U + c), Uxp = ld(f.U + c + 1);
        const R eACI = h * rdx1[i] * (kPP2 * rdmx1[ip] + kPP1 * rdmx1[i] - dx1[ip] * (R(0.5) * rdmx1[ip]) * dkPP2 * dedx2 + dx1[im] * (R(0.5) * rdmx1[i]) * dkPP1 * dedx1)
                          + (R(0.25) * Uc * rdmx1[i] - R(0.25) * Uxp * rdmx1[ip])
                          - R(0.5) * h * ((kPP2 * dedx2 - kPP1 * dedx1) * rdx1[i] + (kPP4 * dedy4 - kPP3 * dedy3) * rdx2[j] + (kPP6 * dedz6 - kPP5 * dedz5) * rdx3[k]);
        const R eAPI = -h * rdx1[i] * (kPP2 * rdmx1[ip] + dx1[i] * (R(0.5) * rdmx1[ip]) * dkPP2 * dedx2) + R(0.25) * Uxp * rdmx1[ip];
        const R eAMI = -h * rdx1[i] * (kPP1 * rdmx1[i] - dx1[i] * (R(0.5) * rdmx1[i]) * dkPP1 * dedx1) - R(0.25) * Uc * rdmx1[i];
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = eACI * dt + R(1.0);
        cf.c = eAPI * dt;
        cf.a = eAMI * dt;
        cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const
    {
        f.scr[ix(g, r + 1, lj(l), 1 + vby<ITEM>())] = x[0];
    }
};

// Stage 3 (:456-507): km, kp stale (N3-1, N3+1); T += solution (:518-524).
template <class R, int ITEM = 0>
struct ThermalY {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = std::is_same<R, float>::value;   // measured faster in FP32 only
    static constexpr int MINB = LineOcc<R>::y;
    static constexpr int MREG = LineOcc<Real>::reg_y;
    static constexpr int NT = LineOcc<Real>::nt_y;
    static constexpr bool CONTIG = false;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt; };
    __device__ State prepare() const { return State{R(g.scal[S_DT])}; }
    __device__ int li(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = r + 1, k = 1 + vby<ITEM>();
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = g.N3 - 1, kp = g.N3 + 1;
        const PhysT<R> &p = g.ph;
        const bool d2 = g.kdeg2 != 0;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const R *T = f.T;
        const R Tc = ld(T + c), Txm = ld(T + c - 1), Txp = ld(T + c + 1), Tym = ld(T + c - sj), Typ = ld(T + c + sj);
        const R Tkm = ld(T + ix(g, i, j, km)), Tkp = ld(T + ix(g, i, j, kp));
        R Kc, dKc, Kym, dKym, Kyp, dKyp, irc, dirc;
        kpp_eval(p, d2, Tc, Kc, dKc); kpp_eval(p, d2, Tym, Kym, dKym); kpp_eval(p, d2, Typ, Kyp, dKyp);
        const R Kxm = kpp_only(p, d2, Txm), Kxp = kpp_only(p, d2, Txp), Kkm = kpp_only(p, d2, Tkm), Kkp = kpp_only(p, d2, Tkp);
        rhocp_eval(p, Tc, irc, dirc);
        const R h = R(0.5) * p.Ct * irc;
        const R jem = (j == 1) ? R(0.0) : R(1.0), jep = (j == g.N2) ? R(0.0) : R(1.0);
        const R KPP1 = R(0.5) * rdmx1[i] * (dx1[i] * Kxm + dx1[im] * Kc), KPP2 = R(0.5) * rdmx1[ip] * (dx1[ip] * Kc + dx1[i] * Kxp);
        const R kPP3 = R(0.5) * rdmx2[j] * (dx2[j] * Kym + dx2[jm] * Kc), kPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * Kc + dx2[j] * Kyp);
        const R KPP5 = R(0.5) * rdmx3[k] * (dx3[k] * Kkm + dx3[km] * Kc), KPP6 = R(0.5) * rdmx3[kp] * (dx3[kp] * Kc + dx3[k] * Kkp);
        const R dkPP3 = R(0.5) * rdmx2[j] * (dx2[j] * dKym + dx2[jm] * dKc), dkPP4 = R(0.5) * rdmx2[jp] * (dx2[jp] * dKc + dx2[j] * dKyp);
        const R dedx1 = (Tc - Txm) * rdmx1[i], dedx2 = (Txp - Tc) * rdmx1[ip];
        const R dedy3 = (Tc - Tym) * rdmx2[j], dedy4 = (Typ - Tc) * rdmx2[jp];
        const R dedz5 = (Tc - Tkm) * rdmx3[k], dedz6 = (Tkp - Tc) * rdmx3[kp];
        const R Vc = ld(f.V + c), Vyp = ld(f.V + c + sj);
        const R eACJ = h * rdx2[j] * (kPP4 * rdmx2[jp] + kPP3 * rdmx2[j] - dx2[jp] * (R(0.5) * rdmx2[jp]) * dkPP4 * dedy4 * jep + dx2[jm] * (R(0.5) * rdmx2[j]) * dkPP3 * dedy3 * jem)
                          + (R(0.25) * Vc * rdmx2[j] - R(0.25) * Vyp * rdmx2[jp])
                          - R(0.5) * h * ((KPP2 * dedx2 - KPP1 * dedx1) * rdx1[i] + (kPP4 * dedy4 - kPP3 * dedy3) * rdx2[j] + (KPP6 * dedz6 - KPP5 * dedz5) * rdx3[k]);
        const R eAPJ = (-h * rdx2[j] * (kPP4 * rdmx2[jp] + dx2[j] * (R(0.5) * rdmx2[jp]) * dkPP4 * dedy4) + R(0.25) * Vyp * rdmx2[jp]) * jep;
        const R eAMJ = (-h * rdx2[j] * (kPP3 * rdmx2[j] - dx2[j] * (R(0.5) * rdmx2[j]) * dkPP3 * dedy3) - R(0.25) * Vc * rdmx2[j]) * jem;
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = eACJ * dt + R(1.0);
        cf.c = eAPJ * dt;
        cf.a = eAMJ * dt;
        cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const
    {
        const int i = li(l), j = r + 1, k = 1 + vby<ITEM>();
        store_periodic(g, f.Tn, i, j, k, ld(f.T + ix(g, i, j, k)) + x[0]);
    }
};

template <class R>
void launch_thermal(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    launch_z<ThermalZ<R>>(cx, g.N3, g.N1, g.N2, [&](int tl) { return ThermalZ<R>{g, cx.f, tl}; }, s, K_THERMAL_Z);
    launch_x<ThermalX>(cx, g.N2, s, K_THERMAL_X);
    launch_y<ThermalY<R>>(cx, g.N2, g.N1, g.N3, [&](int tl) { return ThermalY<R>{g, cx.f, tl}; }, s, K_THERMAL_Y);
}

// The same three sweeps for many cases, one launch per sweep.
template <class R>
void launch_thermal_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s)
{
    multi_stage<ThermalZ<R, 1>>(cs, A, s, "thermal_z",
        [](const Ctx<R> &x) { return StageShape{x.g.N3, true, x.tl_strided, x.g.N1, x.g.N2}; },
        [](const Ctx<R> &x, int tl) { return ThermalZ<R, 1>{x.g, x.f, tl}; });
    multi_x<ThermalX>(cs, A, s, "thermal_x", [](const Ctx<R> &x) { return x.g.N2; });
    multi_stage<ThermalY<R, 1>>(cs, A, s, "thermal_y",
        [](const Ctx<R> &x) { return StageShape{x.g.N2, false, x.tl_strided, x.g.N1, x.g.N3}; },
        [](const Ctx<R> &x, int tl) { return ThermalY<R, 1>{x.g, x.f, tl}; });
}

// the two forms
template void launch_thermal<double>(const Ctx<double> &, cudaStream_t);
template void launch_thermal<float>(const Ctx<float> &, cudaStream_t);
template void launch_thermal_multi<double>(const std::vector<Ctx<double> *> &, MultiArena &, cudaStream_t);
template void launch_thermal_multi<float>(const std::vector<Ctx<float> *> &, MultiArena &, cudaStream_t);

} // namespace tcs
