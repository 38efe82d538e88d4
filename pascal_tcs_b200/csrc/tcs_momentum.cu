// tcs_momentum.cu -- momentum increments: mpi_momentum_coeffi, solvedU/V/W,
// blockLdV/U and the standalone pseudo-update (module_solve_momentum.f90).
//
// Each solved* routine is three fused kernels (z, x, y sweeps) on the shared
// line solver; the y sweep writes the increment with its periodic ghosts, which
// is the ghost update the driver performs right after (main.f90:151-169).
//
// Mu and invRho are the 2-D (j,k) tables of mpi_momentum_coeffi: the
// reference assigns whole rows Mu(:,j,k) inside its i loop (:156-171), so every
// value along i equals the one computed from T(n1sub,j,k).
#include "tcs_kernels.h"
#include "tcs_tma.cuh"

namespace tcs {

#define MU(jj, kk) ld(f.Mu2 + ix2(g, (jj), (kk)))
#define IR(jj, kk) ld(f.iR2 + ix2(g, (jj), (kk)))

// ---------------------------------------------------------------------------
// mpi_momentum_coeffi (:145-173) -> (j,k) tables from T(n1sub, j, k).
// ---------------------------------------------------------------------------
// Evaluated in FP64 in both forms; the FP32 form also keeps invRho in FP64
// (FieldsT::iR2d) for the pressure right-hand side and the projection.
template <class R>
__global__ void momentum_coeffi_kernel(GridT<R> g, FieldsT<R> f)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j > g.N2 + 1 || blown(g)) return;
    const Phys &p = g.phd;
    const double t1 = p.DeltaT * (double)f.T[ix(g, g.N1 + 1, j, k)];
    const double t2 = t1 * t1, t3 = t2 * t1, t4 = t3 * t1, t5 = t4 * t1;
    const double ra = (p.a10 + p.a10 * (p.a11 * t1 + p.a12 * t2 + p.a13 * t3 + p.a14 * t4 + p.a15 * t5));
    const double ir = p.Rho0 / ra;
    f.Mu2[ix2(g, j, k)] = (R)(ra * (p.d10 + p.d10 * (p.d11 * t1 + p.d12 * t2 + p.d13 * t3 + p.d14 * t4 + p.d15 * t5)) / p.Mu0);
    f.iR2[ix2(g, j, k)] = (R)ir;
    if constexpr (HasLo<R>::on) f.iR2d[ix2(g, j, k)] = ir;
}

template <class R>
void launch_momentum_coeffi(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    probe_begin(cx, K_MOM_COEFFI, s);
    momentum_coeffi_kernel<<<dim3((g.N2 + 2 + 127) / 128, g.N3 + 2), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_MOM_COEFFI, s);
    record_launch_error("momentum_coeffi");
}

// ---------------------------------------------------------------------------
// solvedU (:225-563)
// ---------------------------------------------------------------------------
template <class R, int ITEM = 0>
struct DUZ {
    using Real = R;
    static constexpr int NRHS = 1;
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
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 1 + vby<ITEM>(), k = r + 1;
        const int im = i - 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const PhysT<R> &p = g.ph;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const R *U = f.U, *V = f.V, *W = f.W;
        const R jum = (j == 1) ? R(0.0) : R(1.0), jup = (j == g.N2) ? R(0.0) : R(1.0);
        const R Uc = ld(U + c), Uxm = ld(U + c - 1), Uxp = ld(U + c + 1), Uym = ld(U + c - sj), Uyp = ld(U + c + sj);
        const R Uzm = ld(U + c - sk), Uzp = ld(U + c + sk);
        const R Vc = ld(V + c), Vxm = ld(V + c - 1), Vyp = ld(V + c + sj), Vxmyp = ld(V + c - 1 + sj);
        const R Wc = ld(W + c), Wxm = ld(W + c - 1), Wzp = ld(W + c + sk), Wxmzp = ld(W + c - 1 + sk);
        const R Mjk = MU(j, k), Mjmk = MU(jm, k), Mjpk = MU(jp, k), Mjkm = MU(j, km), Mjkp = MU(j, kp);
        const R iRjk = IR(j, k);
        const R u1 = R(0.5) * (Uxm + Uc), u2 = R(0.5) * (Uxp + Uc);
        const R v3 = R(0.5) * (dx1[im] * Vc + dx1[i] * Vxm) * rdmx1[i];
        const R v4 = R(0.5) * (dx1[im] * Vyp + dx1[i] * Vxmyp) * rdmx1[i];
        const R w5 = R(0.5) * (dx1[im] * Wc + dx1[i] * Wxm) * rdmx1[i];
        const R w6 = R(0.5) * (dx1[im] * Wzp + dx1[i] * Wxmzp) * rdmx1[i];
        const R dudx1 = (Uc - Uxm) * rdx1[im], dudx2 = (Uxp - Uc) * rdx1[i];
        const R dudy3 = (Uc - Uym) * rdmx2[j], dudy4 = (Uyp - Uc) * rdmx2[jp];
        const R dudz5 = (Uc - Uzm) * rdmx3[k], dudz6 = (Uzp - Uc) * rdmx3[kp];
        const R dvdx3 = (Vc - Vxm) * rdmx1[i], dvdx4 = (Vyp - Vxmyp) * rdmx1[i];
        const R dwdx5 = (Wc - Wxm) * rdmx1[i], dwdx6 = (Wzp - Wxmzp) * rdmx1[i];
        R mua = R(0.5) * (dx1[im] * Mjmk + dx1[i] * Mjmk) * rdmx1[i];
        const R muc = R(0.5) * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
        R mub = R(0.5) * (dx1[im] * Mjpk + dx1[i] * Mjpk) * rdmx1[i];
        const R mu3 = R(0.5) * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
        const R mu4 = R(0.5) * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
        mua = R(0.5) * (dx1[im] * Mjkm + dx1[i] * Mjkm) * rdmx1[i];
        mub = R(0.5) * (dx1[im] * Mjkp + dx1[i] * Mjkp) * rdmx1[i];
        const R mu5 = R(0.5) * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
        const R mu6 = R(0.5) * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
        const R invRhoc = R(0.5) * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R vu1 = (Mjk * dudx2 - Mjk * dudx1) * rdmx1[i];
        const R vu2 = (mu4 * dudy4 - mu3 * dudy3) * rdx2[j];
        const R vu3 = (mu6 * dudz6 - mu5 * dudz5) * rdx3[k];
        const R vu12 = (mu4 * dvdx4 - mu3 * dvdx3) * rdx2[j];
        const R vu13 = (mu6 * dwdx6 - mu5 * dwdx5) * rdx3[k];
        // The reduced right-hand side (see the thermal z sweep): the explicit
        // operator minus the implicit ones applied to U, with the x and z parts
        // collapsed (their coefficient terms cancel in exact arithmetic) and the
        // y part in the reference's form on the wall-adjacent planes only.
        R rhs = R(4.0) * ih * vu1 + R(2.0) * ih * (vu3 + vu13) - R(0.5) * (u1 * dudx1 + u2 * dudx2) - R(0.5) * (w5 * dudz5 + w6 * dudz6);
        rhs = rhs - p.Cmp * invRhoc * (ld(f.P + c) - ld(f.P + c - 1)) * rdmx1[i];
        const R Tc = R(0.5) * (dx1[im] * ld(f.T + c) + dx1[i] * ld(f.T + c - 1)) * rdmx1[i];
        rhs = rhs + p.Cmt * (Tc + p.a12pera11 * (Tc * Tc) * p.DeltaT) * invRhoc;
        if (j != 1 && j != g.N2) {
            rhs = rhs + R(2.0) * ih * (vu2 + vu12) - R(0.5) * (v3 * dudy3 + v4 * dudy4);
        } else {
            R ubc_dn = R(0.25) * v3 * rdmx2[j] * p.Ubt - R(0.25) * dudy3 * (dx1[i] * p.Vbt + dx1[im] * p.Vbt) * rdmx1[i] * R(0.5);
            R ubc_up = -R(0.25) * v4 * rdmx2[jp] * p.Uup - R(0.25) * dudy4 * (dx1[i] * p.Vup + dx1[im] * p.Vup) * rdmx1[i] * R(0.5);
            ubc_dn = ubc_dn + ih * rdx2[j] * mu3 * rdmx2[j] * p.Ubt;
            ubc_dn = ubc_dn - ih * rdx2[j] * mu3 * rdmx1[i] * (p.Vbt - p.Vbt);
            ubc_up = ubc_up + ih * rdx2[j] * mu4 * rdmx2[jp] * p.Uup;
            ubc_up = ubc_up + ih * rdx2[j] * mu4 * rdmx1[i] * (p.Vup - p.Vup);
            const R mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + R(0.25) * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
            const R mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + R(0.25) * (v4 * rdmx2[jp])) * jup;
            const R mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + R(0.25) * (-v3 * rdmx2[j])) * jum;
            rhs = rhs + ih * (vu2 + vu12) + (R(1.0) - jum) * ubc_dn + (R(1.0) - jup) * ubc_up - (mAPJ * Uyp + mACJ * Uc + mAMJ * Uym)
                  - (R(0.25) * (v4 * jup * dudy4 + v3 * jum * dudy3) - ih * rdx2[j] * (mu4 * dvdx4 * jup - mu3 * dvdx3 * jum));
        }
        const R mACK = ih * rdx3[k] * (mu6 * rdmx3[kp] + mu5 * rdmx3[k]) + R(0.25) * (-w6 * rdmx3[kp] + w5 * rdmx3[k]);
        const R mAPK = -ih * rdx3[k] * mu6 * rdmx3[kp] + R(0.25) * (w6 * rdmx3[kp]);
        const R mAMK = -ih * rdx3[k] * mu5 * rdmx3[k] + R(0.25) * (-w5 * rdmx3[k]);
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACK * dt + R(1.0); cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, li(l), 1 + vby<ITEM>(), r + 1)] = x[0]; }
};

template <class R, int WIDE = 0, int ITEM = 0>
struct DUX {
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
        const int i = r + 1, j = lj(l), k = 1 + vby<ITEM>(), im = i - 1;
        const PhysT<R> &p = g.ph;
        const R *dx1 = g.m1.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx;
        const long long c = ix(g, i, j, k);
        const R Uc = ld(f.U + c), Uxm = ld(f.U + c - 1), Uxp = ld(f.U + c + 1);
        const R Mjk = MU(j, k), iRjk = IR(j, k);
        const R u1 = R(0.5) * (Uxm + Uc), u2 = R(0.5) * (Uxp + Uc);
        const R dudx1 = (Uc - Uxm) * rdx1[im], dudx2 = (Uxp - Uc) * rdx1[i];
        const R invRhoc = R(0.5) * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACI = ih * rdmx1[i] * (Mjk * rdx1[i] + Mjk * rdx1[im]) * R(2.0) + R(0.25) * (dudx2 * R(0.5) + dudx1 * R(0.5) - u2 * rdx1[i] + u1 * rdx1[im]);
        const R mAPI = -ih * rdmx1[i] * Mjk * rdx1[i] * R(2.0) + R(0.25) * (u2 * rdx1[i] + dudx2 * R(0.5));
        const R mAMI = -ih * rdmx1[i] * Mjk * rdx1[im] * R(2.0) + R(0.25) * (-u1 * rdx1[im] + dudx1 * R(0.5));
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACI * dt + R(1.0); cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, r + 1, lj(l), 1 + vby<ITEM>())] = x[0]; }
};

template <class R, int ITEM = 0>
struct DUY {
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
        const int i = li(l), j = r + 1, k = 1 + vby<ITEM>(), im = i - 1, jm = j - 1, jp = j + 1;
        const PhysT<R> &p = g.ph;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx;
        const R *rdx2 = g.m2.rdx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const R jum = (j == 1) ? R(0.0) : R(1.0), jup = (j == g.N2) ? R(0.0) : R(1.0);
        const R v3 = R(0.5) * (dx1[im] * ld(f.V + c) + dx1[i] * ld(f.V + c - 1)) * rdmx1[i];
        const R v4 = R(0.5) * (dx1[im] * ld(f.V + c + sj) + dx1[i] * ld(f.V + c - 1 + sj)) * rdmx1[i];
        const R Mjk = MU(j, k), Mjmk = MU(jm, k), Mjpk = MU(jp, k), iRjk = IR(j, k);
        const R mua = R(0.5) * (dx1[im] * Mjmk + dx1[i] * Mjmk) * rdmx1[i];
        const R muc = R(0.5) * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
        const R mub = R(0.5) * (dx1[im] * Mjpk + dx1[i] * Mjpk) * rdmx1[i];
        const R mu3 = R(0.5) * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
        const R mu4 = R(0.5) * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
        const R invRhoc = R(0.5) * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + R(0.25) * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const R mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + R(0.25) * (v4 * rdmx2[jp])) * jup;
        const R mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + R(0.25) * (-v3 * rdmx2[j])) * jum;
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACJ * dt + R(1.0); cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { store_periodic(g, f.dU, li(l), r + 1, 1 + vby<ITEM>(), x[0]); }
};

// ---------------------------------------------------------------------------
// solvedV (:569-924): rows j = j_indexS(=2)..N2.  Stage 2 uses mu1, mu2 left
// by the last stage-1 iteration (i=N1, j=N2, k=N3); the y stage scales the
// upper coefficient by jvp = jS_BC(j-1) and the lower one by jvm = jS_BC(j+1).
// ---------------------------------------------------------------------------
template <class R, int ITEM = 0>
struct DVZ {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = std::is_same<R, float>::value;   // measured faster in FP32 only
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
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 2 + vby<ITEM>(), k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const PhysT<R> &p = g.ph;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const R *U = f.U, *V = f.V, *W = f.W, *dU = f.dU;
        const R jvp = (jm >= 2) ? R(1.0) : R(0.0);               // jS_BC(jm)
        const R jvm = (jp <= g.N2) ? R(1.0) : R(0.0);            // jS_BC(jp)
        const R Vc = ld(V + c), Vym = ld(V + c - sj), Vyp = ld(V + c + sj), Vxm = ld(V + c - 1), Vxp = ld(V + c + 1);
        const R Vzm = ld(V + c - sk), Vzp = ld(V + c + sk);
        const R Uc = ld(U + c), Uym = ld(U + c - sj), Uxp = ld(U + c + 1), Uxpym = ld(U + c + 1 - sj);
        const R Wc = ld(W + c), Wym = ld(W + c - sj), Wzp = ld(W + c + sk), Wzpym = ld(W + c + sk - sj);
        const R dUc = ld(dU + c), dUym = ld(dU + c - sj), dUxp = ld(dU + c + 1), dUxpym = ld(dU + c + 1 - sj);
        const R Mjk = MU(j, k), Mjmk = MU(jm, k), Mjkm = MU(j, km), Mjmkm = MU(jm, km), Mjkp = MU(j, kp), Mjmkp = MU(jm, kp);
        const R iRjk = IR(j, k), iRjmk = IR(jm, k);
        const R v3 = R(0.5) * (Vym + Vc), v4 = R(0.5) * (Vc + Vyp);
        const R u1 = (dx2[jm] * Uc + dx2[j] * Uym) * rdmx2[j] * R(0.5);
        const R u2 = (dx2[jm] * Uxp + dx2[j] * Uxpym) * rdmx2[j] * R(0.5);
        const R w5 = (dx2[jm] * Wc + dx2[j] * Wym) * rdmx2[j] * R(0.5);
        const R w6 = (dx2[jm] * Wzp + dx2[j] * Wzpym) * rdmx2[j] * R(0.5);
        const R ddu1 = (dx2[jm] * dUc + dx2[j] * dUym) * rdmx2[j] * R(0.5);
        const R ddu2 = (dx2[jm] * dUxp + dx2[j] * dUxpym) * rdmx2[j] * R(0.5);
        const R dvdx1 = (Vc - Vxm) * rdmx1[i], dvdx2 = (Vxp - Vc) * rdmx1[ip];
        const R dvdy3 = (Vc - Vym) * rdx2[jm], dvdy4 = (Vyp - Vc) * rdx2[j];
        const R dvdz5 = (Vc - Vzm) * rdmx3[k], dvdz6 = (Vzp - Vc) * rdmx3[kp];
        const R dudy1 = (Uc - Uym) * rdmx2[j], dudy2 = (Uxp - Uxpym) * rdmx2[j];
        const R dwdy5 = (Wc - Wym) * rdmx2[j], dwdy6 = (Wzp - Wzpym) * rdmx2[j];
        const R ddudy1 = (dUc - dUym) * rdmx2[j], ddudy2 = (dUxp - dUxpym) * rdmx2[j];
        // Mu(im,..) = Mu(i,..) = Mu(ip,..): the three x-neighbour averages coincide
        const R mxy = R(0.5) * (dx2[jm] * Mjk + dx2[j] * Mjmk) * rdmx2[j];
        const R mu1 = R(0.5) * (dx1[im] * mxy + dx1[i] * mxy) * rdmx1[i];
        const R mu2 = R(0.5) * (dx1[ip] * mxy + dx1[i] * mxy) * rdmx1[ip];
        const R mua = R(0.5) * (dx2[jm] * Mjkm + dx2[j] * Mjmkm) * rdmx2[j];
        const R mub = R(0.5) * (dx2[jm] * Mjkp + dx2[j] * Mjmkp) * rdmx2[j];
        const R mu5 = R(0.5) * (dx3[km] * mxy + dx3[k] * mua) * rdmx3[k];
        const R mu6 = R(0.5) * (dx3[kp] * mxy + dx3[k] * mub) * rdmx3[kp];
        const R invRhoc = R(0.5) * (dx2[jm] * iRjk + dx2[j] * iRjmk) * rdmx2[j];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R vv1 = (mu2 * dvdx2 - mu1 * dvdx1) * rdx1[i];
        const R vv2 = (Mjk * dvdy4 - Mjmk * dvdy3) * rdmx2[j];
        const R vv3 = (mu6 * dvdz6 - mu5 * dvdz5) * rdx3[k];
        const R vv21 = (mu2 * dudy2 - mu1 * dudy1) * rdx1[i];
        const R vv23 = (mu6 * dwdy6 - mu5 * dwdy5) * rdx3[k];
        // The reduced right-hand side (see DUZ); the y part keeps the
        // reference's form on the planes next to the walls (j = 2, N2).
        R rhs = R(2.0) * ih * (vv1 + vv21 + vv3 + vv23) - R(0.5) * (u1 * dvdx1 + u2 * dvdx2) - R(0.5) * (w5 * dvdz5 + w6 * dvdz6)
                - R(0.25) * (ddu1 * dvdx1 + ddu2 * dvdx2) + ih * rdx1[i] * (mu2 * ddudy2 - mu1 * ddudy1);
        rhs = rhs - p.Cmp * invRhoc * (ld(f.P + c) - ld(f.P + c - sj)) * rdmx2[j];
        if (jvp != R(0.0) && jvm != R(0.0)) {
            rhs = rhs + R(4.0) * ih * vv2 - R(0.5) * (v3 * dvdy3 + v4 * dvdy4);
        } else {
            R vbc_dn = (R(0.25) * rdx2[jm] * v3 * p.Vbt - R(0.25) * R(0.5) * dvdy3 * p.Vbt);
            R vbc_up = (-R(0.25) * rdx2[j] * v4 * p.Vup - R(0.25) * R(0.5) * dvdy4 * p.Vup);
            vbc_dn = vbc_dn + ih * rdmx2[j] * Mjmk * rdx2[jm] * p.Vbt * R(2.0);
            vbc_up = vbc_up + ih * rdmx2[j] * Mjk * rdx2[j] * p.Vup * R(2.0);
            const R mACJ = ih * rdmx2[j] * (Mjk * rdx2[j] + Mjmk * rdx2[jm]) * R(2.0) + R(0.25) * (dvdy4 * R(0.5) + dvdy3 * R(0.5) - v4 * rdx2[j] + v3 * rdx2[jm]);
            const R mAPJ = (-ih * rdmx2[j] * Mjk * rdx2[j] * R(2.0) + R(0.25) * (v4 * rdx2[j] + dvdy4 * R(0.5))) * jvp;
            const R mAMJ = (-ih * rdmx2[j] * Mjmk * rdx2[jm] * R(2.0) + R(0.25) * (-v3 * rdx2[jm] + dvdy3 * R(0.5))) * jvm;
            rhs = rhs + R(2.0) * ih * vv2 + (R(1.0) - jvm) * vbc_dn + (R(1.0) - jvp) * vbc_up - (mAPJ * Vyp + mACJ * Vc + mAMJ * Vym);
        }
        const R mACK = ih * rdx3[k] * (mu6 * rdmx3[kp] + mu5 * rdmx3[k]) + R(0.25) * (-w6 * rdmx3[kp] + w5 * rdmx3[k]);
        const R mAPK = -ih * rdx3[k] * mu6 * rdmx3[kp] + R(0.25) * (w6 * rdmx3[kp]);
        const R mAMK = -ih * rdx3[k] * mu5 * rdmx3[k] + R(0.25) * (-w5 * rdmx3[k]);
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACK * dt + R(1.0); cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, li(l), 2 + vby<ITEM>(), r + 1)] = x[0]; }
};

// mu1, mu2 of solvedV's last stage-1 iteration (i = N1, j = N2, k = N3).
template <class R>
__device__ __forceinline__ void dv_stale_mu12(const GridT<R> &g, const FieldsT<R> &f, R &mu1, R &mu2)
{
    const int i = g.N1, j = g.N2, k = g.N3, im = i - 1, ip = i + 1, jm = j - 1;
    const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
    const R mxy = R(0.5) * (dx2[jm] * MU(j, k) + dx2[j] * MU(jm, k)) * rdmx2[j];
    mu1 = R(0.5) * (dx1[im] * mxy + dx1[i] * mxy) * rdmx1[i];
    mu2 = R(0.5) * (dx1[ip] * mxy + dx1[i] * mxy) * rdmx1[ip];
}

template <class R, int WIDE = 0, int ITEM = 0>
struct DVX {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = true;    // measured faster with qrcp
    static constexpr int MINB = WIDE ? LineOcc<R>::xw : LineOcc<R>::x;
    static constexpr int MREG = WIDE ? LineOcc<Real>::reg_xw : LineOcc<Real>::reg_x;
    static constexpr int NT = WIDE ? LineOcc<Real>::nt_xw : LineOcc<Real>::nt_x;
    static constexpr bool CONTIG = true;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt, mu1, mu2; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dv_stale_mu12(g, f, s.mu1, s.mu2);
        return s;
    }
    __device__ int lj(int l) const { return 2 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + vby<ITEM>(), ip = i + 1, jm = j - 1;
        const PhysT<R> &p = g.ph;
        const R *dx2 = g.m2.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const R mu1 = st.mu1, mu2 = st.mu2;
        const R u1 = (dx2[jm] * ld(f.U + c) + dx2[j] * ld(f.U + c - sj)) * rdmx2[j] * R(0.5);
        const R u2 = (dx2[jm] * ld(f.U + c + 1) + dx2[j] * ld(f.U + c + 1 - sj)) * rdmx2[j] * R(0.5);
        const R invRhoc = R(0.5) * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + R(0.25) * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const R mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + R(0.25) * (u2 * rdmx1[ip]);
        const R mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + R(0.25) * (-u1 * rdmx1[i]);
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACI * dt + R(1.0); cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, r + 1, lj(l), 1 + vby<ITEM>())] = x[0]; }
};

template <class R, int ITEM = 0>
struct DVY {
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
        const int i = li(l), j = r + 2, k = 1 + vby<ITEM>(), jm = j - 1, jp = j + 1;
        const PhysT<R> &p = g.ph;
        const R *dx2 = g.m2.dx, *rdx2 = g.m2.rdx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const R jvp = (jm >= 2) ? R(1.0) : R(0.0), jvm = (jp <= g.N2) ? R(1.0) : R(0.0);
        const R Vc = ld(f.V + c), Vym = ld(f.V + c - sj), Vyp = ld(f.V + c + sj);
        const R v3 = R(0.5) * (Vym + Vc), v4 = R(0.5) * (Vc + Vyp);
        const R dvdy3 = (Vc - Vym) * rdx2[jm], dvdy4 = (Vyp - Vc) * rdx2[j];
        const R Mjk = MU(j, k), Mjmk = MU(jm, k);
        const R invRhoc = R(0.5) * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACJ = ih * rdmx2[j] * (Mjk * rdx2[j] + Mjmk * rdx2[jm]) * R(2.0) + R(0.25) * (dvdy4 * R(0.5) + dvdy3 * R(0.5) - v4 * rdx2[j] + v3 * rdx2[jm]);
        const R mAPJ = (-ih * rdmx2[j] * Mjk * rdx2[j] * R(2.0) + R(0.25) * (v4 * rdx2[j] + dvdy4 * R(0.5))) * jvp;
        const R mAMJ = (-ih * rdmx2[j] * Mjmk * rdx2[jm] * R(2.0) + R(0.25) * (-v3 * rdx2[jm] + dvdy3 * R(0.5))) * jvm;
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACJ * dt + R(1.0); cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { store_periodic(g, f.dV, li(l), r + 2, 1 + vby<ITEM>(), x[0]); }
};

// ---------------------------------------------------------------------------
// solvedW (:930-1272).  Stage 2 uses stale mu1, mu2 and stage 3 stale mu3,
// mu4 (last stage-1 iteration) and a stale km = N3-1 (last stage-2 iteration).
// ---------------------------------------------------------------------------
template <class R, int ITEM = 0>
struct DWZ {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = std::is_same<R, float>::value;   // measured faster in FP32 only
    static constexpr int MINB = LineOcc<R>::z;
    static constexpr int MREG = LineOcc<Real>::reg_z;
    static constexpr int NT = LineOcc<Real>::nt_z;
    static constexpr bool CONTIG = false;
    static constexpr bool PAIR = LineOcc<Real>::pair_z;
    static constexpr bool LINE_PER_THREAD = false;   // the unpaired FP32 build: measured slower
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt; };
    __device__ State prepare() const { return State{R(g.scal[S_DT])}; }
    __device__ int li(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    // The stencil inputs of a cell, read through val(array, di, dj, dk): from
    // global memory (build) or from the staged tiles (dwz_staged_kernel), with
    // the same arithmetic after them.
    enum : int { A_W = 0, A_U, A_V, A_DU, A_DV, A_P };
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const long long c = ix(g, li(l), 1 + vby<ITEM>(), r + 1), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const R *const arr[6] = {f.W, f.U, f.V, f.dU, f.dV, f.P};
        return build_with([&](int a, int di, int dj, int dk) { return ld(arr[a] + (c + di + dj * sj + dk * sk)); }, l, r, st);
    }
    template <class Val>
    __device__ __forceinline__ Coef<R, 1> build_with(const Val &val, int l, int r, const State &st) const
    {
        const int i = li(l), j = 1 + vby<ITEM>(), k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1;
        const PhysT<R> &p = g.ph;
        const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const R *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const R jwm = (j == 1) ? R(0.0) : R(1.0), jwp = (j == g.N2) ? R(0.0) : R(1.0);
        const R Wc = val(A_W, 0, 0, 0), Wzm = val(A_W, 0, 0, -1), Wzp = val(A_W, 0, 0, 1), Wxm = val(A_W, -1, 0, 0), Wxp = val(A_W, 1, 0, 0);
        const R Wym = val(A_W, 0, -1, 0), Wyp = val(A_W, 0, 1, 0);
        const R Uc = val(A_U, 0, 0, 0), Uzm = val(A_U, 0, 0, -1), Uxp = val(A_U, 1, 0, 0), Uxpzm = val(A_U, 1, 0, -1);
        const R Vc = val(A_V, 0, 0, 0), Vzm = val(A_V, 0, 0, -1), Vyp = val(A_V, 0, 1, 0), Vypzm = val(A_V, 0, 1, -1);
        const R dUc = val(A_DU, 0, 0, 0), dUzm = val(A_DU, 0, 0, -1), dUxp = val(A_DU, 1, 0, 0), dUxpzm = val(A_DU, 1, 0, -1);
        const R dVc = val(A_DV, 0, 0, 0), dVzm = val(A_DV, 0, 0, -1), dVyp = val(A_DV, 0, 1, 0), dVypzm = val(A_DV, 0, 1, -1);
        const R Mjk = MU(j, k), Mjkm = MU(j, km), Mjmk = MU(jm, k), Mjmkm = MU(jm, km), Mjpk = MU(jp, k), Mjpkm = MU(jp, km);
        const R iRjk = IR(j, k), iRjkm = IR(j, km);
        const R w5 = R(0.5) * (Wc + Wzm), w6 = R(0.5) * (Wc + Wzp);
        const R u1 = (dx3[km] * Uc + dx3[k] * Uzm) * rdmx3[k] * R(0.5);
        const R u2 = (dx3[km] * Uxp + dx3[k] * Uxpzm) * rdmx3[k] * R(0.5);
        const R v3 = (dx3[km] * Vc + dx3[k] * Vzm) * rdmx3[k] * R(0.5);
        const R v4 = (dx3[km] * Vyp + dx3[k] * Vypzm) * rdmx3[k] * R(0.5);
        const R dwdx1 = (Wc - Wxm) * rdmx1[i], dwdx2 = (Wxp - Wc) * rdmx1[ip];
        const R dwdy3 = (Wc - Wym) * rdmx2[j], dwdy4 = (Wyp - Wc) * rdmx2[jp];
        const R dwdz5 = (Wc - Wzm) * rdx3[km], dwdz6 = (Wzp - Wc) * rdx3[k];
        const R dudz1 = (Uc - Uzm) * rdmx3[k], dudz2 = (Uxp - Uxpzm) * rdmx3[k];
        const R dvdz3 = (Vc - Vzm) * rdmx3[k], dvdz4 = (Vyp - Vypzm) * rdmx3[k];
        const R ddudz1 = (dUc - dUzm) * rdmx3[k], ddudz2 = (dUxp - dUxpzm) * rdmx3[k];
        const R ddvdz3 = (dVc - dVzm) * rdmx3[k], ddvdz4 = (dVyp - dVypzm) * rdmx3[k];
        const R ddu1 = (dx3[km] * dUc + dx3[k] * dUzm) * rdmx3[k] * R(0.5);
        const R ddu2 = (dx3[km] * dUxp + dx3[k] * dUxpzm) * rdmx3[k] * R(0.5);
        const R ddv3 = (dx3[km] * dVc + dx3[k] * dVzm) * rdmx3[k] * R(0.5) * jwm;
        const R ddv4 = (dx3[km] * dVyp + dx3[k] * dVypzm) * rdmx3[k] * R(0.5) * jwp;
        const R mxz = R(0.5) * (dx3[km] * Mjk + dx3[k] * Mjkm) * rdmx3[k];   // mua = muc = mub (x)
        const R mu1 = R(0.5) * (dx1[im] * mxz + dx1[i] * mxz) * rdmx1[i];
        const R mu2 = R(0.5) * (dx1[ip] * mxz + dx1[i] * mxz) * rdmx1[ip];
        const R mua = R(0.5) * (dx3[km] * Mjmk + dx3[k] * Mjmkm) * rdmx3[k];
        const R mub = R(0.5) * (dx3[km] * Mjpk + dx3[k] * Mjpkm) * rdmx3[k];
        const R mu3 = R(0.5) * (dx2[jm] * mxz + dx2[j] * mua) * rdmx2[j];
        const R mu4 = R(0.5) * (dx2[jp] * mxz + dx2[j] * mub) * rdmx2[jp];
        const R invRhoc = R(0.5) * (dx3[km] * iRjk + dx3[k] * iRjkm) * rdmx3[k];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R vw1 = (mu2 * dwdx2 - mu1 * dwdx1) * rdx1[i];
        const R vw2 = (mu4 * dwdy4 - mu3 * dwdy3) * rdx2[j];
        const R vw3 = (Mjk * dwdz6 - Mjkm * dwdz5) * rdmx3[k];
        const R vw31 = (mu2 * dudz2 - mu1 * dudz1) * rdx1[i];
        const R vw32 = (mu4 * dvdz4 - mu3 * dvdz3) * rdx2[j];
        // The reduced right-hand side (see DUZ); the y part keeps the
        // reference's form on the wall-adjacent planes (j = 1, N2).
        R rhs = R(2.0) * ih * (vw1 + vw31) + R(4.0) * ih * vw3 - R(0.5) * (u1 * dwdx1 + u2 * dwdx2) - R(0.5) * (w5 * dwdz5 + w6 * dwdz6)
                - R(0.25) * (ddu1 * dwdx1 + ddu2 * dwdx2) + ih * rdx1[i] * (mu2 * ddudz2 - mu1 * ddudz1);
        rhs = rhs - p.Cmp * invRhoc * (val(A_P, 0, 0, 0) - val(A_P, 0, 0, -1)) * rdmx3[k];
        if (j != 1 && j != g.N2) {
            rhs = rhs + R(2.0) * ih * (vw2 + vw32) - R(0.5) * (v3 * dwdy3 + v4 * dwdy4)
                  - R(0.25) * (ddv3 * dwdy3 + ddv4 * dwdy4) + ih * rdx2[j] * (mu4 * ddvdz4 - mu3 * ddvdz3);
        } else {
            R zbc_dn = R(0.25) * v3 * rdmx2[j] * p.Wbt - R(0.25) * dwdy3 * (dx3[km] * p.Vbt + dx3[k] * p.Vbt) * rdmx3[k] * R(0.5);
            R zbc_up = -R(0.25) * v4 * rdmx2[jp] * p.Wup - R(0.25) * dwdy4 * (dx3[km] * p.Vup + dx3[k] * p.Vup) * rdmx3[k] * R(0.5);
            zbc_dn = zbc_dn + ih * rdx2[j] * mu3 * rdmx2[jp] * p.Wbt;
            zbc_up = zbc_up + ih * rdx2[j] * mu4 * rdmx2[j] * p.Wup;
            zbc_dn = zbc_dn - ih * rdx2[j] * mu3 * rdmx3[k] * (p.Vbt - p.Vbt);
            zbc_up = zbc_up + ih * rdx2[j] * mu4 * rdmx3[k] * (p.Vup - p.Vup);
            const R mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + R(0.25) * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
            const R mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + R(0.25) * (v4 * rdmx2[jp])) * jwp;
            const R mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + R(0.25) * (-v3 * rdmx2[j])) * jwm;
            rhs = rhs + ih * (vw2 + vw32) + (R(1.0) - jwm) * zbc_dn + (R(1.0) - jwp) * zbc_up - (mAPJ * Wyp + mACJ * Wc + mAMJ * Wym)
                  - (R(0.25) * (v3 * jwm * dwdy3 + v4 * jwp * dwdy4) - ih * rdx2[j] * (mu4 * dvdz4 * jwp - mu3 * dvdz3 * jwm))
                  - (R(0.25) * (ddv3 * jwm * dwdy3 + ddv4 * jwp * dwdy4) - ih * rdx2[j] * (mu4 * ddvdz4 * jwp - mu3 * ddvdz3 * jwm));
        }
        const R mACK = ih * rdmx3[k] * (Mjk * rdx3[k] + Mjkm * rdx3[km]) * R(2.0) + R(0.25) * (-w6 * rdx3[k] + w5 * rdx3[km] + R(0.5) * dwdz6 + R(0.5) * dwdz5);
        const R mAPK = -ih * rdmx3[k] * Mjk * rdx3[k] * R(2.0) + R(0.25) * (w6 * rdx3[k] + R(0.5) * dwdz6);
        const R mAMK = -ih * rdmx3[k] * Mjkm * rdx3[km] * R(2.0) + R(0.25) * (-w5 * rdx3[km] + R(0.5) * dwdz5);
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACK * dt + R(1.0); cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, li(l), 1 + vby<ITEM>(), r + 1)] = x[0]; }
};

// mu1..mu4 of solvedW's last stage-1 iteration (i = N1, j = N2, k = N3).
template <class R>
__device__ __forceinline__ void dw_stale_mu(const GridT<R> &g, const FieldsT<R> &f, R &mu1, R &mu2, R &mu3, R &mu4)
{
    const int i = g.N1, j = g.N2, k = g.N3, im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1;
    const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
    const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const R mxz = R(0.5) * (dx3[km] * MU(j, k) + dx3[k] * MU(j, km)) * rdmx3[k];
    mu1 = R(0.5) * (dx1[im] * mxz + dx1[i] * mxz) * rdmx1[i];
    mu2 = R(0.5) * (dx1[ip] * mxz + dx1[i] * mxz) * rdmx1[ip];
    const R mua = R(0.5) * (dx3[km] * MU(jm, k) + dx3[k] * MU(jm, km)) * rdmx3[k];
    const R mub = R(0.5) * (dx3[km] * MU(jp, k) + dx3[k] * MU(jp, km)) * rdmx3[k];
    mu3 = R(0.5) * (dx2[jm] * mxz + dx2[j] * mua) * rdmx2[j];
    mu4 = R(0.5) * (dx2[jp] * mxz + dx2[j] * mub) * rdmx2[jp];
}

template <class R, int WIDE = 0, int ITEM = 0>
struct DWX {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = true;    // measured faster with qrcp
    static constexpr int MINB = WIDE ? LineOcc<R>::xw : LineOcc<R>::x;
    static constexpr int MREG = WIDE ? LineOcc<Real>::reg_xw : LineOcc<Real>::reg_x;
    static constexpr int NT = WIDE ? LineOcc<Real>::nt_xw : LineOcc<Real>::nt_x;
    static constexpr bool CONTIG = true;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt, mu1, mu2, mu3, mu4; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dw_stale_mu(g, f, s.mu1, s.mu2, s.mu3, s.mu4);
        return s;
    }
    __device__ int lj(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + vby<ITEM>(), ip = i + 1, km = k - 1;
        const PhysT<R> &p = g.ph;
        const R *dx3 = g.m3.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sk = (long long)g.P1 * g.P2;
        const R mu1 = st.mu1, mu2 = st.mu2, mu3 = st.mu3, mu4 = st.mu4;
        (void)mu1; (void)mu2; (void)mu3; (void)mu4;
        const R u1 = (dx3[km] * ld(f.U + c) + dx3[k] * ld(f.U + c - sk)) * rdmx3[k] * R(0.5);
        const R u2 = (dx3[km] * ld(f.U + c + 1) + dx3[k] * ld(f.U + c + 1 - sk)) * rdmx3[k] * R(0.5);
        const R invRhoc = R(0.5) * (dx3[km] * IR(j, k) + dx3[k] * IR(j, km)) * rdmx3[k];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + R(0.25) * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const R mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + R(0.25) * (u2 * rdmx1[ip]);
        const R mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + R(0.25) * (-u1 * rdmx1[i]);
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACI * dt + R(1.0); cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { f.scr[ix(g, r + 1, lj(l), 1 + vby<ITEM>())] = x[0]; }
};

template <class R, int ITEM = 0>
struct DWY {
    using Real = R;
    static constexpr int NRHS = 1;
    static constexpr bool FAST_RCP = std::is_same<R, float>::value;   // measured faster in FP32 only
    static constexpr int MINB = LineOcc<R>::y;
    static constexpr int MREG = LineOcc<Real>::reg_y;
    static constexpr int NT = LineOcc<Real>::nt_y;
    static constexpr bool CONTIG = false;
    GridT<R> g; FieldsT<R> f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { R dt, mu1, mu2, mu3, mu4; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dw_stale_mu(g, f, s.mu1, s.mu2, s.mu3, s.mu4);
        return s;
    }
    __device__ int li(int l) const { return 1 + vbx<ITEM>() * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<R, 1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = r + 1, k = 1 + vby<ITEM>(), jp = j + 1, km = g.N3 - 1;
        const PhysT<R> &p = g.ph;
        const R *dx3 = g.m3.dx, *rdx2 = g.m2.rdx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const R jwm = (j == 1) ? R(0.0) : R(1.0), jwp = (j == g.N2) ? R(0.0) : R(1.0);
        const R mu1 = st.mu1, mu2 = st.mu2, mu3 = st.mu3, mu4 = st.mu4;
        (void)mu1; (void)mu2; (void)mu3; (void)mu4;
        const long long ckm = ix(g, i, j, km);
        const R v3 = (dx3[km] * ld(f.V + c) + dx3[k] * ld(f.V + ckm)) * rdmx3[k] * R(0.5);
        const R v4 = (dx3[km] * ld(f.V + c + sj) + dx3[k] * ld(f.V + ckm + sj)) * rdmx3[k] * R(0.5);
        const R invRhoc = R(0.5) * (dx3[km] * IR(j, k) + dx3[k] * IR(j, km)) * rdmx3[k];
        const R ih = R(0.5) * p.Cmu * invRhoc;
        const R mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + R(0.25) * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const R mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + R(0.25) * (v4 * rdmx2[jp])) * jwp;
        const R mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + R(0.25) * (-v3 * rdmx2[j])) * jwm;
        const R dt = st.dt;
        Coef<R, 1> cf;
        cf.b = mACJ * dt + R(1.0); cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.scr + c);
        return cf;
    }
    __device__ void emit(int l, int r, const R *x, const State &st) const { store_periodic(g, f.dW, li(l), r + 1, 1 + vby<ITEM>(), x[0]); }
};

// ---------------------------------------------------------------------------
// solvedW's z sweep with its stencil inputs staged by TMA (FP64 form,
// TCS_TUNE_Z_STAGING 2).  The same lines, rows, arithmetic and solve as the
// DWZ line-solver launch (DWZ::build_with is shared, so the results are the
// same bits); only where the stencil inputs come from differs.  A block of
// 512 threads owns 8 lines (i0..i0+7) of one j; the rows are built in passes of
// ZS_CH = 64 k-planes, one cell per thread per pass, from shared-memory boxes
// of the six input arrays that the tensor memory accelerator copies one pass
// ahead (two buffers):
//   W       i0-1..i0+8 x j-1..j+1 x k-1..k+64      (x and y neighbours, k +-1)
//   U, dU   i0-1..i0+8 x j        x k-1..k+63
//   V, dV   i0-1..i0+8 x j..j+1   x k-1..k+63
//   P       i0-1..i0+8 x j        x k-1..k+63
// Every box starts at x = i0-1 = 8 bx, an even element, so its first byte is
// 16-byte aligned as TMA requires, and is 10 doubles (80 bytes) wide.  It
// requires N3 a multiple of ZS_CH and an even N1 (the row pitch a multiple of
// 16 bytes); launch_solve_dw checks both.
// ---------------------------------------------------------------------------
constexpr int ZS_CH = 64, ZS_TL = 8, ZS_NT = 512;
constexpr int ZS_WAIT = 1 << 22;   // polls of a bounded wait (each try_wait suspends briefly)
__host__ __device__ constexpr int zs_rows(int a) { return a == 0 ? 3 : ((a == 2 || a == 4) ? 2 : 1); }
__host__ __device__ constexpr int zs_planes(int a) { return a == 0 ? ZS_CH + 2 : ZS_CH + 1; }
__host__ __device__ constexpr int zs_bytes(int a) { return 10 * zs_rows(a) * zs_planes(a) * 8; }
__host__ __device__ constexpr int zs_off(int a) { return a == 0 ? 0 : zs_off(a - 1) + (zs_bytes(a - 1) + 127) / 128 * 128; }
constexpr int ZS_BUF = zs_off(6);
constexpr int ZS_TX = zs_bytes(0) + zs_bytes(1) + zs_bytes(2) + zs_bytes(3) + zs_bytes(4) + zs_bytes(5);

struct alignas(64) DWZMaps {
    CUtensorMap m[6];   // DWZ's A_W, A_U, A_V, A_DU, A_DV, A_P
};

// Dynamic shared memory: two box buffers, the rows (A, C, D), the row map, two mbarriers.
inline size_t zs_smem(const LinePlan &lp)
{
    const size_t rows = (size_t)3 * ZS_TL * lp.LS * sizeof(double) + (size_t)lp.n * sizeof(int);
    return 2 * (size_t)ZS_BUF + ((rows + 15) & ~(size_t)15) + 2 * sizeof(uint64_t);
}

__global__ void __launch_bounds__(ZS_NT, 1) dwz_staged_kernel(const __grid_constant__ DWZ<double> prob,
                                                              const __grid_constant__ DWZMaps maps, LinePlan lp)
{
    using P = DWZ<double>;
    extern __shared__ __align__(128) unsigned char smraw[];
    if (prob.skip()) return;
    const P::State st = prob.prepare();
    const int n = lp.n, LS = lp.LS, DS = ZS_TL * LS, nch = n / ZS_CH;
    double *const sA = reinterpret_cast<double *>(smraw + 2 * ZS_BUF), *const sC = sA + DS, *const sD = sC + DS;
    int *const spos = reinterpret_cast<int *>(sD + DS);
    const size_t rows = (size_t)3 * DS * sizeof(double) + (size_t)n * sizeof(int);
    uint64_t *const bar = reinterpret_cast<uint64_t *>(smraw + 2 * ZS_BUF + ((rows + 15) & ~(size_t)15));
    const int x0 = ZS_TL * blockIdx.x, j = 1 + blockIdx.y;
    if (smem_u32(smraw) & 127) {   // the boxes need 128-byte aligned destinations: record and stop, copy nothing
        if (threadIdx.x == 0) {
            atomicAdd(prob.g.scal + S_TIMEOUT, 1.0);
            prob.g.scal[S_BLOWUP] = 1.0;
        }
        return;
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    if (threadIdx.x < lp.P) {
        const int p = threadIdx.x, m = lp.m0 + (p < lp.rem ? 1 : 0), start = p * lp.m0 + (p < lp.rem ? p : lp.rem);
        for (int q = 0; q < m; q++) spos[start + q] = p * lp.PS + q;
    }
    __syncthreads();
    auto issue = [&](int c) {   // thread 0: the boxes of pass c into buffer c & 1
        uint64_t *b = &bar[c & 1];
        unsigned char *dst = smraw + (c & 1) * ZS_BUF;
        mbar_arrive_expect_tx(b, ZS_TX);
#pragma unroll
        for (int a = 0; a < 6; a++) tma_load_3d(dst + zs_off(a), &maps.m[a], b, x0, a == P::A_W ? j - 1 : j, c * ZS_CH);
    };
    if (threadIdx.x == 0) {
        issue(0);
        if (nch > 1) issue(1);
    }
    const int l = threadIdx.x & (ZS_TL - 1), rr = threadIdx.x >> 3;   // one cell per thread per pass
    int c = 0;
    bool ok = true;
    for (; c < nch; c++) {
        const bool got = mbar_wait(&bar[c & 1], (c >> 1) & 1, ZS_WAIT);
        if (__syncthreads_or(!got)) { ok = false; break; }
        const double *const t = reinterpret_cast<const double *>(smraw + (c & 1) * ZS_BUF);
        // row r = c ZS_CH + rr is plane k = r + 1, plane k + dk of a box at z = rr + 1 + dk
        auto val = [&](int a, int di, int dj, int dk) -> double {
            int z = rr + 1 + dk, y = (a == P::A_W) ? 1 + dj : dj, x = l + 1 + di;
            TCS_OOB(prob.g.scal, (unsigned)z >= (unsigned)zs_planes(a) || (unsigned)y >= (unsigned)zs_rows(a) || (unsigned)x >= 10u,
                    (z = 0, y = 0, x = 0));
            return t[zs_off(a) / 8 + (z * zs_rows(a) + y) * 10 + x];
        };
        const int r = c * ZS_CH + rr;
        Coef<double, 1> cf;
        if (prob.line_ok(l)) {
            cf = prob.build_with(val, l, r, st);
        } else {
            cf.a = 0.0; cf.b = 1.0; cf.c = 0.0; cf.d[0] = 0.0;
        }
        const double rb = rcp_of<FastRcp<P>::on>(cf.b);
        const int pos = l * LS + spos[r];
        sA[pos] = cf.a * rb; sC[pos] = cf.c * rb; sD[pos] = cf.d[0] * rb;
        __syncthreads();   // every thread is done with this buffer
        if (threadIdx.x == 0 && c + 2 < nch) {
            fence_proxy_async();
            issue(c + 2);
        }
    }
    if (!ok) {
        // a copy did not arrive in time: record it, stop the step, and wait
        // (bounded) for this block's copies still in flight before leaving
        if (threadIdx.x == 0) {
            atomicAdd(prob.g.scal + S_TIMEOUT, 1.0);
            prob.g.scal[S_BLOWUP] = 1.0;
            for (int d = c; d < c + 2 && d < nch; d++) mbar_wait(&bar[d & 1], (d >> 1) & 1, ZS_WAIT);
        }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int ll = warp; ll < ZS_TL; ll += ZS_NT / 32)
        solve_line<double, 1, P::MREG, false, FastRcp<P>::on>(sA + ll * LS, sC + ll * LS, sD + ll * LS, DS, lp, lane);
    __syncthreads();
    if (prob.line_ok(l))
        for (int r = rr; r < n; r += ZS_NT / ZS_TL) {
            const double x = sD[l * LS + spos[r]];
            prob.emit(l, r, &x, st);
        }
}

// The tensor maps of the staged z sweep: one 3-D map (x = i, y = j, z = k over
// the padded array) per input array with that array's box.
typedef CUresult (*PfnTensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                            CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static PfnTensorMapEncodeTiled tensor_map_encoder()
{
    static PfnTensorMapEncodeTiled fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return (PfnTensorMapEncodeTiled)f;
    }();
    return fn;
}

static bool dwz_maps(const Ctx<double> &cx, DWZMaps &mp)
{
    const GridT<double> &g = cx.g;
    PfnTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    const double *src[6] = {cx.f.W, cx.f.U, cx.f.V, cx.f.dU, cx.f.dV, cx.f.P};
    const cuuint64_t dims[3] = {(cuuint64_t)g.P1, (cuuint64_t)g.P2, (cuuint64_t)g.N3 + 2};
    const cuuint64_t strides[2] = {(cuuint64_t)g.P1 * 8, (cuuint64_t)g.P1 * g.P2 * 8};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int a = 0; a < 6; a++) {
        const cuuint32_t box[3] = {10, (cuuint32_t)zs_rows(a), (cuuint32_t)zs_planes(a)};
        if (enc(&mp.m[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)src[a], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

// Whether the staged form can run this case (shape, shared memory, tensor-map encoder).
bool dwz_staging_possible(const Ctx<double> &cx)
{
    const GridT<double> &g = cx.g;
    if (g.N3 % ZS_CH || (g.P1 * 8) % 16) return false;
    if (zs_smem(make_line_plan(g.N3, true, ZS_TL, cx.lanes)) > 227 * 1024) return false;
    DWZMaps mp;
    return dwz_maps(cx, mp);
}

// Launches the staged form if the knob asks for it and the shape allows it.
static bool launch_dwz_staged(const Ctx<double> &cx, cudaStream_t s)
{
    const GridT<double> &g = cx.g;
    if (cx.z_staging != 2 || g.N3 % ZS_CH || (g.P1 * 8) % 16) return false;
    const LinePlan lp = make_line_plan(g.N3, true, ZS_TL, cx.lanes);
    const size_t sm = zs_smem(lp);
    if (sm > 227 * 1024) return false;
    DWZMaps mp;
    if (!dwz_maps(cx, mp)) return false;
    static size_t conf[64] = {};
    smem_opt_in((const void *)dwz_staged_kernel, sm, conf);
    probe_begin(cx, K_DW_Z, s);
    dwz_staged_kernel<<<dim3((g.N1 + ZS_TL - 1) / ZS_TL, g.N2), ZS_NT, sm, s>>>(DWZ<double>{g, cx.f, ZS_TL}, mp, lp);
    probe_end(cx, K_DW_Z, s);
    record_launch_error(kernel_name(K_DW_Z));
    return true;
}

template <class R>
void launch_solve_du(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    launch_z<DUZ<R>>(cx, g.N3, g.N1, g.N2, [&](int tl) { return DUZ<R>{g, cx.f, tl}; }, s, K_DU_Z);
    launch_x<DUX>(cx, g.N2, s, K_DU_X);
    launch_y<DUY<R>>(cx, g.N2, g.N1, g.N3, [&](int tl) { return DUY<R>{g, cx.f, tl}; }, s, K_DU_Y);
}

template <class R>
void launch_solve_dv(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    launch_z<DVZ<R>>(cx, g.N3, g.N1, g.N2 - 1, [&](int tl) { return DVZ<R>{g, cx.f, tl}; }, s, K_DV_Z);
    launch_x<DVX>(cx, g.N2 - 1, s, K_DV_X);
    launch_y<DVY<R>>(cx, g.N2 - 1, g.N1, g.N3, [&](int tl) { return DVY<R>{g, cx.f, tl}; }, s, K_DV_Y);
}

template <class R>
void launch_solve_dw(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    bool staged = false;
    if constexpr (std::is_same<R, double>::value) staged = launch_dwz_staged(cx, s);
    if (!staged) launch_z<DWZ<R>>(cx, g.N3, g.N1, g.N2, [&](int tl) { return DWZ<R>{g, cx.f, tl}; }, s, K_DW_Z);
    launch_x<DWX>(cx, g.N2, s, K_DW_X);
    launch_y<DWY<R>>(cx, g.N2, g.N1, g.N3, [&](int tl) { return DWY<R>{g, cx.f, tl}; }, s, K_DW_Y);
}

// ---------------------------------------------------------------------------
// blockLdV (:1278-1356): dV -= dt*M23 dW, j = 2..N2, then ghost(dV).
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R blockld_v_value(const GridT<R> &g, const FieldsT<R> &f, int i, int j, int k)
{
    const int jm = j - 1, km = k - 1, kp = k + 1;
    const R *dx2 = g.m2.dx, *dx3 = g.m3.dx, *rdx3 = g.m3.rdx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
    const R dWc = ld(f.dW + c), dWym = ld(f.dW + c - sj), dWzp = ld(f.dW + c + sk), dWzpym = ld(f.dW + c + sk - sj);
    const R dwm5 = (dx2[jm] * dWc + dx2[j] * dWym) * rdmx2[j] * R(0.5);
    const R dwm6 = (dx2[jm] * dWzp + dx2[j] * dWzpym) * rdmx2[j] * R(0.5);
    const R ddwdy5 = (dWc - dWym) * rdmx2[j], ddwdy6 = (dWzp - dWzpym) * rdmx2[j];
    const R Vc = ld(f.V + c);
    const R dvdz5 = (Vc - ld(f.V + c - sk)) * rdmx3[k], dvdz6 = (ld(f.V + c + sk) - Vc) * rdmx3[kp];
    const R invRhoc = R(0.5) * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
    const R mua = R(0.5) * (dx2[jm] * MU(j, km) + dx2[j] * MU(jm, km)) * rdmx2[j];
    const R muc = R(0.5) * (dx2[jm] * MU(j, k) + dx2[j] * MU(jm, k)) * rdmx2[j];
    const R mub = R(0.5) * (dx2[jm] * MU(j, kp) + dx2[j] * MU(jm, kp)) * rdmx2[j];
    const R mu5 = R(0.5) * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
    const R mu6 = R(0.5) * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
    const R dt = g.scal[S_DT];
    return f.dV[c] - dt * (R(0.25) * (dwm5 * dvdz5 + dwm6 * dvdz6) - R(0.5) * g.ph.Cmu * invRhoc * rdx3[k] * (mu6 * ddwdy6 - mu5 * ddwdy5));
}

// KZ planes per thread: every input of the KZ cells is loaded before the first store
template <class R, int KZ>
__global__ void blockld_v_kernel(GridT<R> g, FieldsT<R> f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 2 + blockIdx.y, k0 = 1 + KZ * blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    R v[KZ];
#pragma unroll
    for (int q = 0; q < KZ; q++) v[q] = k0 + q <= g.N3 ? blockld_v_value(g, f, i, j, k0 + q) : R(0);
#pragma unroll
    for (int q = 0; q < KZ; q++)
        if (k0 + q <= g.N3) store_periodic(g, f.dV, i, j, k0 + q, v[q]);
}

template <class R>
void launch_blockld_v(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    probe_begin(cx, K_BLOCKLDV, s);
    blockld_v_kernel<R, 2><<<dim3((g.N1 + 127) / 128, g.N2 - 1, (g.N3 + 1) / 2), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_BLOCKLDV, s);
    record_launch_error("blockld_v");
}

// blockLdU (:1362-1460): dU -= dt*(M12 dV + M13 dW), j = 1..N2 (no ghost
// update follows in the driver; only interior dU is read afterwards).
template <class R>
__device__ __forceinline__ R blockld_u_value(const GridT<R> &g, const FieldsT<R> &f, int i, int j, int k)
{
    const int im = i - 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
    const R *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
    const R *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
    const R jum = (j == 1) ? R(0.0) : R(1.0), jup = (j == g.N2) ? R(0.0) : R(1.0);
    const R Mjk = MU(j, k), iRjk = IR(j, k);
    const R invRhoc = R(0.5) * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
    const R dVc = ld(f.dV + c), dVxm = ld(f.dV + c - 1), dVyp = ld(f.dV + c + sj), dVxmyp = ld(f.dV + c - 1 + sj);
    const R dvm3 = (dx1[i] * dVxm + dx1[im] * dVc) * rdmx1[i] * R(0.5) * jum;
    const R dvm4 = (dx1[i] * dVxmyp + dx1[im] * dVyp) * rdmx1[i] * R(0.5) * jup;
    const R Uc = ld(f.U + c);
    const R dudy3 = (Uc - ld(f.U + c - sj)) * rdmx2[j], dudy4 = (ld(f.U + c + sj) - Uc) * rdmx2[jp];
    const R dvmdx3 = (dVc - dVxm) * rdmx1[i] * jum, dvmdx4 = (dVyp - dVxmyp) * rdmx1[i] * jup;
    R mua = R(0.5) * (dx1[im] * MU(jm, k) + dx1[i] * MU(jm, k)) * rdmx1[i];
    const R muc = R(0.5) * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
    R mub = R(0.5) * (dx1[im] * MU(jp, k) + dx1[i] * MU(jp, k)) * rdmx1[i];
    const R mu3 = R(0.5) * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
    const R mu4 = R(0.5) * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
    const R dWc = ld(f.dW + c), dWxm = ld(f.dW + c - 1), dWzp = ld(f.dW + c + sk), dWxmzp = ld(f.dW + c - 1 + sk);
    const R dwm5 = (dx1[i] * dWxm + dx1[im] * dWc) * rdmx1[i] * R(0.5);
    const R dwm6 = (dx1[i] * dWxmzp + dx1[im] * dWzp) * rdmx1[i] * R(0.5);
    const R dudz5 = (Uc - ld(f.U + c - sk)) * rdmx3[k], dudz6 = (ld(f.U + c + sk) - Uc) * rdmx3[kp];
    const R dwmdx5 = (dWc - dWxm) * rdmx1[i], dwmdx6 = (dWzp - dWxmzp) * rdmx1[i];
    mua = R(0.5) * (dx1[im] * MU(j, km) + dx1[i] * MU(j, km)) * rdmx1[i];
    mub = R(0.5) * (dx1[im] * MU(j, kp) + dx1[i] * MU(j, kp)) * rdmx1[i];
    const R mu5 = R(0.5) * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
    const R mu6 = R(0.5) * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
    const R dt = g.scal[S_DT], Cmu = g.ph.Cmu;
    return f.dU[c]
        - dt * (R(0.25) * (dvm4 * dudy4 + dvm3 * dudy3) - R(0.5) * Cmu * invRhoc * rdx2[j] * (mu4 * dvmdx4 - mu3 * dvmdx3))
        - dt * (R(0.25) * (dwm6 * dudz6 + dwm5 * dudz5) - R(0.5) * Cmu * invRhoc * rdx3[k] * (mu6 * dwmdx6 - mu5 * dwmdx5));
}

// KZ planes per thread: every input of the KZ cells is loaded before the first store
template <class R, int KZ>
__global__ void blockld_u_kernel(GridT<R> g, FieldsT<R> f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k0 = 1 + KZ * blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    R v[KZ];
#pragma unroll
    for (int q = 0; q < KZ; q++) v[q] = k0 + q <= g.N3 ? blockld_u_value(g, f, i, j, k0 + q) : R(0);
    const long long sk = (long long)g.P1 * g.P2;
#pragma unroll
    for (int q = 0; q < KZ; q++)
        if (k0 + q <= g.N3) f.dU[ix(g, i, j, k0) + q * sk] = v[q];
}

template <class R>
void launch_blockld_u(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    probe_begin(cx, K_BLOCKLDU, s);
    blockld_u_kernel<R, 2><<<dim3((g.N1 + 127) / 128, g.N2, (g.N3 + 1) / 2), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_BLOCKLDU, s);
    record_launch_error("blockld_u");
}

// Standalone mpi_momentum_pseudoupdateUVW (:178-208) + ghost(U,V,W): writes the
// second buffers; the caller swaps them in.  The step normally fuses this into
// the pressure right-hand side (tcs_pressure.cu).
template <class R>
__global__ void pseudo_update_kernel(GridT<R> g, FieldsT<R> f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const long long c = ix(g, i, j, k);
    const R vmask = (j == 1) ? R(0.0) : R(1.0);     // dble(2 - j_indexS) on the lower plane
    if constexpr (HasLo<R>::on) {                    // FP32 form: FP64 sums of the high/low pairs
        float h, lo;
        split(join(f.U[c], f.Ulo[c]) + (double)f.dU[c], h, lo);
        store_periodic(g, f.Un, i, j, k, h); store_periodic(g, f.Unlo, i, j, k, lo);
        split(join(f.V[c], f.Vlo[c]) + (double)f.dV[c] * (double)vmask, h, lo);
        store_periodic(g, f.Vn, i, j, k, h); store_periodic(g, f.Vnlo, i, j, k, lo);
        split(join(f.W[c], f.Wlo[c]) + (double)f.dW[c], h, lo);
        store_periodic(g, f.Wn, i, j, k, h); store_periodic(g, f.Wnlo, i, j, k, lo);
    } else {
        store_periodic(g, f.Un, i, j, k, f.U[c] + f.dU[c]);
        store_periodic(g, f.Vn, i, j, k, f.V[c] + f.dV[c] * vmask);
        store_periodic(g, f.Wn, i, j, k, f.W[c] + f.dW[c]);
    }
}

template <class R>
void launch_pseudo_update(const Ctx<R> &cx, cudaStream_t s)
{
    const GridT<R> &g = cx.g;
    probe_begin(cx, K_PSEUDO, s);
    pseudo_update_kernel<<<dim3((g.N1 + 127) / 128, g.N2, g.N3), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_PSEUDO, s);
    record_launch_error("pseudo_update");
}

#undef MU
#undef IR

// the two forms
// The nine sweeps of solvedU, solvedV and solvedW for many cases, one launch per sweep.
template <class R>
void launch_momentum_multi(const std::vector<Ctx<R> *> &cs, MultiArena &A, cudaStream_t s)
{
    auto z = [](int ny) {
        return [ny](const Ctx<R> &x) { return StageShape{x.g.N3, true, x.tl_strided, x.g.N1, x.g.N2 - ny}; };
    };
    auto y = [](int ny) {
        return [ny](const Ctx<R> &x) { return StageShape{x.g.N2 - ny, false, x.tl_strided, x.g.N1, x.g.N3}; };
    };
    auto lines = [](int ny) { return [ny](const Ctx<R> &x) { return x.g.N2 - ny; }; };
    multi_stage<DUZ<R, 1>>(cs, A, s, "du_z", z(0), [](const Ctx<R> &x, int tl) { return DUZ<R, 1>{x.g, x.f, tl}; });
    multi_x<DUX>(cs, A, s, "du_x", lines(0));
    multi_stage<DUY<R, 1>>(cs, A, s, "du_y", y(0), [](const Ctx<R> &x, int tl) { return DUY<R, 1>{x.g, x.f, tl}; });
    multi_stage<DVZ<R, 1>>(cs, A, s, "dv_z", z(1), [](const Ctx<R> &x, int tl) { return DVZ<R, 1>{x.g, x.f, tl}; });
    multi_x<DVX>(cs, A, s, "dv_x", lines(1));
    multi_stage<DVY<R, 1>>(cs, A, s, "dv_y", y(1), [](const Ctx<R> &x, int tl) { return DVY<R, 1>{x.g, x.f, tl}; });
    multi_stage<DWZ<R, 1>>(cs, A, s, "dw_z", z(0), [](const Ctx<R> &x, int tl) { return DWZ<R, 1>{x.g, x.f, tl}; });
    multi_x<DWX>(cs, A, s, "dw_x", lines(0));
    multi_stage<DWY<R, 1>>(cs, A, s, "dw_y", y(0), [](const Ctx<R> &x, int tl) { return DWY<R, 1>{x.g, x.f, tl}; });
}

template void launch_momentum_multi<double>(const std::vector<Ctx<double> *> &, MultiArena &, cudaStream_t);
template void launch_momentum_multi<float>(const std::vector<Ctx<float> *> &, MultiArena &, cudaStream_t);
template void launch_momentum_coeffi<double>(const Ctx<double> &, cudaStream_t);
template void launch_momentum_coeffi<float>(const Ctx<float> &, cudaStream_t);
template void launch_solve_du<double>(const Ctx<double> &, cudaStream_t);
template void launch_solve_du<float>(const Ctx<float> &, cudaStream_t);
template void launch_solve_dv<double>(const Ctx<double> &, cudaStream_t);
template void launch_solve_dv<float>(const Ctx<float> &, cudaStream_t);
template void launch_solve_dw<double>(const Ctx<double> &, cudaStream_t);
template void launch_solve_dw<float>(const Ctx<float> &, cudaStream_t);
template void launch_blockld_v<double>(const Ctx<double> &, cudaStream_t);
template void launch_blockld_v<float>(const Ctx<float> &, cudaStream_t);
template void launch_blockld_u<double>(const Ctx<double> &, cudaStream_t);
template void launch_blockld_u<float>(const Ctx<float> &, cudaStream_t);
template void launch_pseudo_update<double>(const Ctx<double> &, cudaStream_t);
template void launch_pseudo_update<float>(const Ctx<float> &, cudaStream_t);

} // namespace tcs
