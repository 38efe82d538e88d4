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

namespace tcs {

#define MU(jj, kk) ld(f.Mu2 + ix2(g, (jj), (kk)))
#define IR(jj, kk) ld(f.iR2 + ix2(g, (jj), (kk)))

// ---------------------------------------------------------------------------
// mpi_momentum_coeffi (:145-173) -> (j,k) tables from T(n1sub, j, k).
// ---------------------------------------------------------------------------
__global__ void momentum_coeffi_kernel(Grid g, Fields f)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j > g.N2 + 1 || blown(g)) return;
    const Phys &p = g.ph;
    const double t1 = p.DeltaT * f.T[ix(g, g.N1 + 1, j, k)];
    const double t2 = t1 * t1, t3 = t2 * t1, t4 = t3 * t1, t5 = t4 * t1;
    const double ra = (p.a10 + p.a10 * (p.a11 * t1 + p.a12 * t2 + p.a13 * t3 + p.a14 * t4 + p.a15 * t5));
    f.Mu2[ix2(g, j, k)] = ra * (p.d10 + p.d10 * (p.d11 * t1 + p.d12 * t2 + p.d13 * t3 + p.d14 * t4 + p.d15 * t5)) / p.Mu0;
    f.iR2[ix2(g, j, k)] = p.Rho0 / ra;
}

void launch_momentum_coeffi(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    probe_begin(cx, K_MOM_COEFFI, s);
    momentum_coeffi_kernel<<<dim3((g.N2 + 2 + 127) / 128, g.N3 + 2), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_MOM_COEFFI, s);
    record_launch_error("momentum_coeffi");
}

// ---------------------------------------------------------------------------
// solvedU (:225-563)
// ---------------------------------------------------------------------------
struct DUZ {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 1 + blockIdx.y, k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const Phys &p = g.ph;
        const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const double *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const double *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const double *U = f.U, *V = f.V, *W = f.W;
        const double jum = (j == 1) ? 0.0 : 1.0, jup = (j == g.N2) ? 0.0 : 1.0;
        const double Uc = ld(U + c), Uxm = ld(U + c - 1), Uxp = ld(U + c + 1), Uym = ld(U + c - sj), Uyp = ld(U + c + sj);
        const double Uzm = ld(U + c - sk), Uzp = ld(U + c + sk);
        const double Vc = ld(V + c), Vxm = ld(V + c - 1), Vyp = ld(V + c + sj), Vxmyp = ld(V + c - 1 + sj);
        const double Wc = ld(W + c), Wxm = ld(W + c - 1), Wzp = ld(W + c + sk), Wxmzp = ld(W + c - 1 + sk);
        const double Mjk = MU(j, k), Mjmk = MU(jm, k), Mjpk = MU(jp, k), Mjkm = MU(j, km), Mjkp = MU(j, kp);
        const double iRjk = IR(j, k);
        const double u1 = 0.5 * (Uxm + Uc), u2 = 0.5 * (Uxp + Uc);
        const double v3 = 0.5 * (dx1[im] * Vc + dx1[i] * Vxm) * rdmx1[i];
        const double v4 = 0.5 * (dx1[im] * Vyp + dx1[i] * Vxmyp) * rdmx1[i];
        const double w5 = 0.5 * (dx1[im] * Wc + dx1[i] * Wxm) * rdmx1[i];
        const double w6 = 0.5 * (dx1[im] * Wzp + dx1[i] * Wxmzp) * rdmx1[i];
        const double dudx1 = (Uc - Uxm) * rdx1[im], dudx2 = (Uxp - Uc) * rdx1[i];
        const double dudy3 = (Uc - Uym) * rdmx2[j], dudy4 = (Uyp - Uc) * rdmx2[jp];
        const double dudz5 = (Uc - Uzm) * rdmx3[k], dudz6 = (Uzp - Uc) * rdmx3[kp];
        const double dvdx3 = (Vc - Vxm) * rdmx1[i], dvdx4 = (Vyp - Vxmyp) * rdmx1[i];
        const double dwdx5 = (Wc - Wxm) * rdmx1[i], dwdx6 = (Wzp - Wxmzp) * rdmx1[i];
        double mua = 0.5 * (dx1[im] * Mjmk + dx1[i] * Mjmk) * rdmx1[i];
        const double muc = 0.5 * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
        double mub = 0.5 * (dx1[im] * Mjpk + dx1[i] * Mjpk) * rdmx1[i];
        const double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
        const double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
        mua = 0.5 * (dx1[im] * Mjkm + dx1[i] * Mjkm) * rdmx1[i];
        mub = 0.5 * (dx1[im] * Mjkp + dx1[i] * Mjkp) * rdmx1[i];
        const double mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
        const double mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
        const double invRhoc = 0.5 * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double vu1 = (Mjk * dudx2 - Mjk * dudx1) * rdmx1[i];
        const double vu2 = (mu4 * dudy4 - mu3 * dudy3) * rdx2[j];
        const double vu3 = (mu6 * dudz6 - mu5 * dudz5) * rdx3[k];
        const double vu12 = (mu4 * dvdx4 - mu3 * dvdx3) * rdx2[j];
        const double vu13 = (mu6 * dwdx6 - mu5 * dwdx5) * rdx3[k];
        double rhs = ih * (2.0 * vu1 + vu2 + vu3 + vu12 + vu13);
        rhs = rhs - p.Cmp * invRhoc * (ld(f.P + c) - ld(f.P + c - 1)) * rdmx1[i];
        const double Tc = 0.5 * (dx1[im] * ld(f.T + c) + dx1[i] * ld(f.T + c - 1)) * rdmx1[i];
        rhs = rhs + p.Cmt * (Tc + p.a12pera11 * (Tc * Tc) * p.DeltaT) * invRhoc;
        double ubc_dn = 0.25 * v3 * rdmx2[j] * p.Ubt - 0.25 * dudy3 * (dx1[i] * p.Vbt + dx1[im] * p.Vbt) * rdmx1[i] * 0.5;
        double ubc_up = -0.25 * v4 * rdmx2[jp] * p.Uup - 0.25 * dudy4 * (dx1[i] * p.Vup + dx1[im] * p.Vup) * rdmx1[i] * 0.5;
        ubc_dn = ubc_dn + ih * rdx2[j] * mu3 * rdmx2[j] * p.Ubt;
        ubc_dn = ubc_dn - ih * rdx2[j] * mu3 * rdmx1[i] * (p.Vbt - p.Vbt);
        ubc_up = ubc_up + ih * rdx2[j] * mu4 * rdmx2[jp] * p.Uup;
        ubc_up = ubc_up + ih * rdx2[j] * mu4 * rdmx1[i] * (p.Vup - p.Vup);
        rhs = rhs + (1.0 - jum) * ubc_dn + (1.0 - jup) * ubc_up;
        const double mACI = ih * rdmx1[i] * (Mjk * rdx1[i] + Mjk * rdx1[im]) * 2.0 + 0.25 * (dudx2 * 0.5 + dudx1 * 0.5 - u2 * rdx1[i] + u1 * rdx1[im]);
        const double mAPI = -ih * rdmx1[i] * Mjk * rdx1[i] * 2.0 + 0.25 * (u2 * rdx1[i] + dudx2 * 0.5);
        const double mAMI = -ih * rdmx1[i] * Mjk * rdx1[im] * 2.0 + 0.25 * (-u1 * rdx1[im] + dudx1 * 0.5);
        const double mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + 0.25 * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const double mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + 0.25 * (v4 * rdmx2[jp])) * jup;
        const double mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + 0.25 * (-v3 * rdmx2[j])) * jum;
        const double mACK = ih * rdx3[k] * (mu6 * rdmx3[kp] + mu5 * rdmx3[k]) + 0.25 * (-w6 * rdmx3[kp] + w5 * rdmx3[k]);
        const double mAPK = -ih * rdx3[k] * mu6 * rdmx3[kp] + 0.25 * (w6 * rdmx3[kp]);
        const double mAMK = -ih * rdx3[k] * mu5 * rdmx3[k] + 0.25 * (-w5 * rdmx3[k]);
        rhs = rhs - (mAPI * Uxp + mACI * Uc + mAMI * Uxm + mAPJ * Uyp + mACJ * Uc + mAMJ * Uym + mAPK * Uzp + mACK * Uc + mAMK * Uzm);
        rhs = rhs - (0.25 * (v4 * jup * dudy4 + v3 * jum * dudy3) - ih * rdx2[j] * (mu4 * dvdx4 * jup - mu3 * dvdx3 * jum));
        rhs = rhs - (0.25 * (w6 * dudz6 + w5 * dudz5) - ih * rdx3[k] * (mu6 * dwdx6 - mu5 * dwdx5));
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACK * dt + 1.0; cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, li(l), 1 + blockIdx.y, r + 1)] = x[0]; }
};

struct DUX {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = true;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int lj(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + blockIdx.y, im = i - 1;
        const Phys &p = g.ph;
        const double *dx1 = g.m1.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx;
        const long long c = ix(g, i, j, k);
        const double Uc = ld(f.U + c), Uxm = ld(f.U + c - 1), Uxp = ld(f.U + c + 1);
        const double Mjk = MU(j, k), iRjk = IR(j, k);
        const double u1 = 0.5 * (Uxm + Uc), u2 = 0.5 * (Uxp + Uc);
        const double dudx1 = (Uc - Uxm) * rdx1[im], dudx2 = (Uxp - Uc) * rdx1[i];
        const double invRhoc = 0.5 * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACI = ih * rdmx1[i] * (Mjk * rdx1[i] + Mjk * rdx1[im]) * 2.0 + 0.25 * (dudx2 * 0.5 + dudx1 * 0.5 - u2 * rdx1[i] + u1 * rdx1[im]);
        const double mAPI = -ih * rdmx1[i] * Mjk * rdx1[i] * 2.0 + 0.25 * (u2 * rdx1[i] + dudx2 * 0.5);
        const double mAMI = -ih * rdmx1[i] * Mjk * rdx1[im] * 2.0 + 0.25 * (-u1 * rdx1[im] + dudx1 * 0.5);
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACI * dt + 1.0; cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, r + 1, lj(l), 1 + blockIdx.y)] = x[0]; }
};

struct DUY {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = r + 1, k = 1 + blockIdx.y, im = i - 1, jm = j - 1, jp = j + 1;
        const Phys &p = g.ph;
        const double *dx1 = g.m1.dx, *dx2 = g.m2.dx;
        const double *rdx2 = g.m2.rdx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const double jum = (j == 1) ? 0.0 : 1.0, jup = (j == g.N2) ? 0.0 : 1.0;
        const double v3 = 0.5 * (dx1[im] * ld(f.V + c) + dx1[i] * ld(f.V + c - 1)) * rdmx1[i];
        const double v4 = 0.5 * (dx1[im] * ld(f.V + c + sj) + dx1[i] * ld(f.V + c - 1 + sj)) * rdmx1[i];
        const double Mjk = MU(j, k), Mjmk = MU(jm, k), Mjpk = MU(jp, k), iRjk = IR(j, k);
        const double mua = 0.5 * (dx1[im] * Mjmk + dx1[i] * Mjmk) * rdmx1[i];
        const double muc = 0.5 * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
        const double mub = 0.5 * (dx1[im] * Mjpk + dx1[i] * Mjpk) * rdmx1[i];
        const double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
        const double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
        const double invRhoc = 0.5 * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + 0.25 * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const double mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + 0.25 * (v4 * rdmx2[jp])) * jup;
        const double mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + 0.25 * (-v3 * rdmx2[j])) * jum;
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACJ * dt + 1.0; cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { store_periodic(g, f.dU, li(l), r + 1, 1 + blockIdx.y, x[0]); }
};

// ---------------------------------------------------------------------------
// solvedV (:569-924): rows j = j_indexS(=2)..N2.  Stage 2 uses mu1, mu2 left
// by the last stage-1 iteration (i=N1, j=N2, k=N3); the y stage scales the
// upper coefficient by jvp = jS_BC(j-1) and the lower one by jvm = jS_BC(j+1).
// ---------------------------------------------------------------------------
struct DVZ {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 2 + blockIdx.y, k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const Phys &p = g.ph;
        const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const double *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const double *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const double *U = f.U, *V = f.V, *W = f.W, *dU = f.dU;
        const double jvp = (jm >= 2) ? 1.0 : 0.0;               // jS_BC(jm)
        const double jvm = (jp <= g.N2) ? 1.0 : 0.0;            // jS_BC(jp)
        const double Vc = ld(V + c), Vym = ld(V + c - sj), Vyp = ld(V + c + sj), Vxm = ld(V + c - 1), Vxp = ld(V + c + 1);
        const double Vzm = ld(V + c - sk), Vzp = ld(V + c + sk);
        const double Uc = ld(U + c), Uym = ld(U + c - sj), Uxp = ld(U + c + 1), Uxpym = ld(U + c + 1 - sj);
        const double Wc = ld(W + c), Wym = ld(W + c - sj), Wzp = ld(W + c + sk), Wzpym = ld(W + c + sk - sj);
        const double dUc = ld(dU + c), dUym = ld(dU + c - sj), dUxp = ld(dU + c + 1), dUxpym = ld(dU + c + 1 - sj);
        const double Mjk = MU(j, k), Mjmk = MU(jm, k), Mjkm = MU(j, km), Mjmkm = MU(jm, km), Mjkp = MU(j, kp), Mjmkp = MU(jm, kp);
        const double iRjk = IR(j, k), iRjmk = IR(jm, k);
        const double v3 = 0.5 * (Vym + Vc), v4 = 0.5 * (Vc + Vyp);
        const double u1 = (dx2[jm] * Uc + dx2[j] * Uym) * rdmx2[j] * 0.5;
        const double u2 = (dx2[jm] * Uxp + dx2[j] * Uxpym) * rdmx2[j] * 0.5;
        const double w5 = (dx2[jm] * Wc + dx2[j] * Wym) * rdmx2[j] * 0.5;
        const double w6 = (dx2[jm] * Wzp + dx2[j] * Wzpym) * rdmx2[j] * 0.5;
        const double ddu1 = (dx2[jm] * dUc + dx2[j] * dUym) * rdmx2[j] * 0.5;
        const double ddu2 = (dx2[jm] * dUxp + dx2[j] * dUxpym) * rdmx2[j] * 0.5;
        const double dvdx1 = (Vc - Vxm) * rdmx1[i], dvdx2 = (Vxp - Vc) * rdmx1[ip];
        const double dvdy3 = (Vc - Vym) * rdx2[jm], dvdy4 = (Vyp - Vc) * rdx2[j];
        const double dvdz5 = (Vc - Vzm) * rdmx3[k], dvdz6 = (Vzp - Vc) * rdmx3[kp];
        const double dudy1 = (Uc - Uym) * rdmx2[j], dudy2 = (Uxp - Uxpym) * rdmx2[j];
        const double dwdy5 = (Wc - Wym) * rdmx2[j], dwdy6 = (Wzp - Wzpym) * rdmx2[j];
        const double ddudy1 = (dUc - dUym) * rdmx2[j], ddudy2 = (dUxp - dUxpym) * rdmx2[j];
        // Mu(im,..) = Mu(i,..) = Mu(ip,..): the three x-neighbour averages coincide
        const double mxy = 0.5 * (dx2[jm] * Mjk + dx2[j] * Mjmk) * rdmx2[j];
        const double mu1 = 0.5 * (dx1[im] * mxy + dx1[i] * mxy) * rdmx1[i];
        const double mu2 = 0.5 * (dx1[ip] * mxy + dx1[i] * mxy) * rdmx1[ip];
        const double mua = 0.5 * (dx2[jm] * Mjkm + dx2[j] * Mjmkm) * rdmx2[j];
        const double mub = 0.5 * (dx2[jm] * Mjkp + dx2[j] * Mjmkp) * rdmx2[j];
        const double mu5 = 0.5 * (dx3[km] * mxy + dx3[k] * mua) * rdmx3[k];
        const double mu6 = 0.5 * (dx3[kp] * mxy + dx3[k] * mub) * rdmx3[kp];
        const double invRhoc = 0.5 * (dx2[jm] * iRjk + dx2[j] * iRjmk) * rdmx2[j];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double vv1 = (mu2 * dvdx2 - mu1 * dvdx1) * rdx1[i];
        const double vv2 = (Mjk * dvdy4 - Mjmk * dvdy3) * rdmx2[j];
        const double vv3 = (mu6 * dvdz6 - mu5 * dvdz5) * rdx3[k];
        const double vv21 = (mu2 * dudy2 - mu1 * dudy1) * rdx1[i];
        const double vv23 = (mu6 * dwdy6 - mu5 * dwdy5) * rdx3[k];
        double rhs = ih * (vv1 + 2.0 * vv2 + vv3 + vv21 + vv23);
        rhs = rhs - p.Cmp * invRhoc * (ld(f.P + c) - ld(f.P + c - sj)) * rdmx2[j];
        double vbc_dn = (0.25 * rdx2[jm] * v3 * p.Vbt - 0.25 * 0.5 * dvdy3 * p.Vbt);
        double vbc_up = (-0.25 * rdx2[j] * v4 * p.Vup - 0.25 * 0.5 * dvdy4 * p.Vup);
        vbc_dn = vbc_dn + ih * rdmx2[j] * Mjmk * rdx2[jm] * p.Vbt * 2.0;
        vbc_up = vbc_up + ih * rdmx2[j] * Mjk * rdx2[j] * p.Vup * 2.0;
        rhs = rhs + (1.0 - jvm) * vbc_dn + (1.0 - jvp) * vbc_up;
        const double mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + 0.25 * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const double mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + 0.25 * (u2 * rdmx1[ip]);
        const double mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + 0.25 * (-u1 * rdmx1[i]);
        const double mACJ = ih * rdmx2[j] * (Mjk * rdx2[j] + Mjmk * rdx2[jm]) * 2.0 + 0.25 * (dvdy4 * 0.5 + dvdy3 * 0.5 - v4 * rdx2[j] + v3 * rdx2[jm]);
        const double mAPJ = (-ih * rdmx2[j] * Mjk * rdx2[j] * 2.0 + 0.25 * (v4 * rdx2[j] + dvdy4 * 0.5)) * jvp;
        const double mAMJ = (-ih * rdmx2[j] * Mjmk * rdx2[jm] * 2.0 + 0.25 * (-v3 * rdx2[jm] + dvdy3 * 0.5)) * jvm;
        const double mACK = ih * rdx3[k] * (mu6 * rdmx3[kp] + mu5 * rdmx3[k]) + 0.25 * (-w6 * rdmx3[kp] + w5 * rdmx3[k]);
        const double mAPK = -ih * rdx3[k] * mu6 * rdmx3[kp] + 0.25 * (w6 * rdmx3[kp]);
        const double mAMK = -ih * rdx3[k] * mu5 * rdmx3[k] + 0.25 * (-w5 * rdmx3[k]);
        rhs = rhs - (mAPI * Vxp + mACI * Vc + mAMI * Vxm + mAPJ * Vyp + mACJ * Vc + mAMJ * Vym + mAPK * Vzp + mACK * Vc + mAMK * Vzm);
        rhs = rhs - (0.25 * (u2 * dvdx2 + u1 * dvdx1) - ih * rdx1[i] * (mu2 * dudy2 - mu1 * dudy1));
        rhs = rhs - (0.25 * (w6 * dvdz6 + w5 * dvdz5) - ih * rdx3[k] * (mu6 * dwdy6 - mu5 * dwdy5));
        rhs = rhs - (0.25 * (ddu2 * dvdx2 + ddu1 * dvdx1) - ih * rdx1[i] * (mu2 * ddudy2 - mu1 * ddudy1));
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACK * dt + 1.0; cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, li(l), 2 + blockIdx.y, r + 1)] = x[0]; }
};

// mu1, mu2 of solvedV's last stage-1 iteration (i = N1, j = N2, k = N3).
__device__ __forceinline__ void dv_stale_mu12(const Grid &g, const Fields &f, double &mu1, double &mu2)
{
    const int i = g.N1, j = g.N2, k = g.N3, im = i - 1, ip = i + 1, jm = j - 1;
    const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
    const double mxy = 0.5 * (dx2[jm] * MU(j, k) + dx2[j] * MU(jm, k)) * rdmx2[j];
    mu1 = 0.5 * (dx1[im] * mxy + dx1[i] * mxy) * rdmx1[i];
    mu2 = 0.5 * (dx1[ip] * mxy + dx1[i] * mxy) * rdmx1[ip];
}

struct DVX {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = true;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt, mu1, mu2; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dv_stale_mu12(g, f, s.mu1, s.mu2);
        return s;
    }
    __device__ int lj(int l) const { return 2 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + blockIdx.y, ip = i + 1, jm = j - 1;
        const Phys &p = g.ph;
        const double *dx2 = g.m2.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const double mu1 = st.mu1, mu2 = st.mu2;
        const double u1 = (dx2[jm] * ld(f.U + c) + dx2[j] * ld(f.U + c - sj)) * rdmx2[j] * 0.5;
        const double u2 = (dx2[jm] * ld(f.U + c + 1) + dx2[j] * ld(f.U + c + 1 - sj)) * rdmx2[j] * 0.5;
        const double invRhoc = 0.5 * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + 0.25 * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const double mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + 0.25 * (u2 * rdmx1[ip]);
        const double mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + 0.25 * (-u1 * rdmx1[i]);
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACI * dt + 1.0; cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, r + 1, lj(l), 1 + blockIdx.y)] = x[0]; }
};

struct DVY {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = r + 2, k = 1 + blockIdx.y, jm = j - 1, jp = j + 1;
        const Phys &p = g.ph;
        const double *dx2 = g.m2.dx, *rdx2 = g.m2.rdx, *rdmx2 = g.m2.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const double jvp = (jm >= 2) ? 1.0 : 0.0, jvm = (jp <= g.N2) ? 1.0 : 0.0;
        const double Vc = ld(f.V + c), Vym = ld(f.V + c - sj), Vyp = ld(f.V + c + sj);
        const double v3 = 0.5 * (Vym + Vc), v4 = 0.5 * (Vc + Vyp);
        const double dvdy3 = (Vc - Vym) * rdx2[jm], dvdy4 = (Vyp - Vc) * rdx2[j];
        const double Mjk = MU(j, k), Mjmk = MU(jm, k);
        const double invRhoc = 0.5 * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACJ = ih * rdmx2[j] * (Mjk * rdx2[j] + Mjmk * rdx2[jm]) * 2.0 + 0.25 * (dvdy4 * 0.5 + dvdy3 * 0.5 - v4 * rdx2[j] + v3 * rdx2[jm]);
        const double mAPJ = (-ih * rdmx2[j] * Mjk * rdx2[j] * 2.0 + 0.25 * (v4 * rdx2[j] + dvdy4 * 0.5)) * jvp;
        const double mAMJ = (-ih * rdmx2[j] * Mjmk * rdx2[jm] * 2.0 + 0.25 * (-v3 * rdx2[jm] + dvdy3 * 0.5)) * jvm;
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACJ * dt + 1.0; cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { store_periodic(g, f.dV, li(l), r + 2, 1 + blockIdx.y, x[0]); }
};

// ---------------------------------------------------------------------------
// solvedW (:930-1272).  Stage 2 uses stale mu1, mu2 and stage 3 stale mu3,
// mu4 (last stage-1 iteration) and a stale km = N3-1 (last stage-2 iteration).
// ---------------------------------------------------------------------------
struct DWZ {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt; };
    __device__ State prepare() const { return State{g.scal[S_DT]}; }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = 1 + blockIdx.y, k = r + 1;
        const int im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
        const Phys &p = g.ph;
        const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
        const double *rdx1 = g.m1.rdx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
        const double *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
        const double *U = f.U, *V = f.V, *W = f.W, *dU = f.dU, *dV = f.dV;
        const double jwm = (j == 1) ? 0.0 : 1.0, jwp = (j == g.N2) ? 0.0 : 1.0;
        const double Wc = ld(W + c), Wzm = ld(W + c - sk), Wzp = ld(W + c + sk), Wxm = ld(W + c - 1), Wxp = ld(W + c + 1);
        const double Wym = ld(W + c - sj), Wyp = ld(W + c + sj);
        const double Uc = ld(U + c), Uzm = ld(U + c - sk), Uxp = ld(U + c + 1), Uxpzm = ld(U + c + 1 - sk);
        const double Vc = ld(V + c), Vzm = ld(V + c - sk), Vyp = ld(V + c + sj), Vypzm = ld(V + c + sj - sk);
        const double dUc = ld(dU + c), dUzm = ld(dU + c - sk), dUxp = ld(dU + c + 1), dUxpzm = ld(dU + c + 1 - sk);
        const double dVc = ld(dV + c), dVzm = ld(dV + c - sk), dVyp = ld(dV + c + sj), dVypzm = ld(dV + c + sj - sk);
        const double Mjk = MU(j, k), Mjkm = MU(j, km), Mjmk = MU(jm, k), Mjmkm = MU(jm, km), Mjpk = MU(jp, k), Mjpkm = MU(jp, km);
        const double iRjk = IR(j, k), iRjkm = IR(j, km);
        const double w5 = 0.5 * (Wc + Wzm), w6 = 0.5 * (Wc + Wzp);
        const double u1 = (dx3[km] * Uc + dx3[k] * Uzm) * rdmx3[k] * 0.5;
        const double u2 = (dx3[km] * Uxp + dx3[k] * Uxpzm) * rdmx3[k] * 0.5;
        const double v3 = (dx3[km] * Vc + dx3[k] * Vzm) * rdmx3[k] * 0.5;
        const double v4 = (dx3[km] * Vyp + dx3[k] * Vypzm) * rdmx3[k] * 0.5;
        const double dwdx1 = (Wc - Wxm) * rdmx1[i], dwdx2 = (Wxp - Wc) * rdmx1[ip];
        const double dwdy3 = (Wc - Wym) * rdmx2[j], dwdy4 = (Wyp - Wc) * rdmx2[jp];
        const double dwdz5 = (Wc - Wzm) * rdx3[km], dwdz6 = (Wzp - Wc) * rdx3[k];
        const double dudz1 = (Uc - Uzm) * rdmx3[k], dudz2 = (Uxp - Uxpzm) * rdmx3[k];
        const double dvdz3 = (Vc - Vzm) * rdmx3[k], dvdz4 = (Vyp - Vypzm) * rdmx3[k];
        const double ddudz1 = (dUc - dUzm) * rdmx3[k], ddudz2 = (dUxp - dUxpzm) * rdmx3[k];
        const double ddvdz3 = (dVc - dVzm) * rdmx3[k], ddvdz4 = (dVyp - dVypzm) * rdmx3[k];
        const double ddu1 = (dx3[km] * dUc + dx3[k] * dUzm) * rdmx3[k] * 0.5;
        const double ddu2 = (dx3[km] * dUxp + dx3[k] * dUxpzm) * rdmx3[k] * 0.5;
        const double ddv3 = (dx3[km] * dVc + dx3[k] * dVzm) * rdmx3[k] * 0.5 * jwm;
        const double ddv4 = (dx3[km] * dVyp + dx3[k] * dVypzm) * rdmx3[k] * 0.5 * jwp;
        const double mxz = 0.5 * (dx3[km] * Mjk + dx3[k] * Mjkm) * rdmx3[k];   // mua = muc = mub (x)
        const double mu1 = 0.5 * (dx1[im] * mxz + dx1[i] * mxz) * rdmx1[i];
        const double mu2 = 0.5 * (dx1[ip] * mxz + dx1[i] * mxz) * rdmx1[ip];
        const double mua = 0.5 * (dx3[km] * Mjmk + dx3[k] * Mjmkm) * rdmx3[k];
        const double mub = 0.5 * (dx3[km] * Mjpk + dx3[k] * Mjpkm) * rdmx3[k];
        const double mu3 = 0.5 * (dx2[jm] * mxz + dx2[j] * mua) * rdmx2[j];
        const double mu4 = 0.5 * (dx2[jp] * mxz + dx2[j] * mub) * rdmx2[jp];
        const double invRhoc = 0.5 * (dx3[km] * iRjk + dx3[k] * iRjkm) * rdmx3[k];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double vw1 = (mu2 * dwdx2 - mu1 * dwdx1) * rdx1[i];
        const double vw2 = (mu4 * dwdy4 - mu3 * dwdy3) * rdx2[j];
        const double vw3 = (Mjk * dwdz6 - Mjkm * dwdz5) * rdmx3[k];
        const double vw31 = (mu2 * dudz2 - mu1 * dudz1) * rdx1[i];
        const double vw32 = (mu4 * dvdz4 - mu3 * dvdz3) * rdx2[j];
        double rhs = ih * (vw1 + vw2 + 2.0 * vw3 + vw31 + vw32);
        rhs = rhs - p.Cmp * invRhoc * (ld(f.P + c) - ld(f.P + c - sk)) * rdmx3[k];
        double zbc_dn = 0.25 * v3 * rdmx2[j] * p.Wbt - 0.25 * dwdy3 * (dx3[km] * p.Vbt + dx3[k] * p.Vbt) * rdmx3[k] * 0.5;
        double zbc_up = -0.25 * v4 * rdmx2[jp] * p.Wup - 0.25 * dwdy4 * (dx3[km] * p.Vup + dx3[k] * p.Vup) * rdmx3[k] * 0.5;
        zbc_dn = zbc_dn + ih * rdx2[j] * mu3 * rdmx2[jp] * p.Wbt;
        zbc_up = zbc_up + ih * rdx2[j] * mu4 * rdmx2[j] * p.Wup;
        zbc_dn = zbc_dn - ih * rdx2[j] * mu3 * rdmx3[k] * (p.Vbt - p.Vbt);
        zbc_up = zbc_up + ih * rdx2[j] * mu4 * rdmx3[k] * (p.Vup - p.Vup);
        rhs = rhs + (1.0 - jwm) * zbc_dn + (1.0 - jwp) * zbc_up;
        const double mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + 0.25 * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const double mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + 0.25 * (u2 * rdmx1[ip]);
        const double mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + 0.25 * (-u1 * rdmx1[i]);
        const double mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + 0.25 * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const double mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + 0.25 * (v4 * rdmx2[jp])) * jwp;
        const double mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + 0.25 * (-v3 * rdmx2[j])) * jwm;
        const double mACK = ih * rdmx3[k] * (Mjk * rdx3[k] + Mjkm * rdx3[km]) * 2.0 + 0.25 * (-w6 * rdx3[k] + w5 * rdx3[km] + 0.5 * dwdz6 + 0.5 * dwdz5);
        const double mAPK = -ih * rdmx3[k] * Mjk * rdx3[k] * 2.0 + 0.25 * (w6 * rdx3[k] + 0.5 * dwdz6);
        const double mAMK = -ih * rdmx3[k] * Mjkm * rdx3[km] * 2.0 + 0.25 * (-w5 * rdx3[km] + 0.5 * dwdz5);
        rhs = rhs - (mAPI * Wxp + mACI * Wc + mAMI * Wxm + mAPJ * Wyp + mACJ * Wc + mAMJ * Wym + mAPK * Wzp + mACK * Wc + mAMK * Wzm);
        rhs = rhs - (0.25 * (u2 * dwdx2 + u1 * dwdx1) - ih * rdx1[i] * (mu2 * dudz2 - mu1 * dudz1));
        rhs = rhs - (0.25 * (v3 * jwm * dwdy3 + v4 * jwp * dwdy4) - ih * rdx2[j] * (mu4 * dvdz4 * jwp - mu3 * dvdz3 * jwm));
        rhs = rhs - (0.25 * (ddu2 * dwdx2 + ddu1 * dwdx1) - ih * rdx1[i] * (mu2 * ddudz2 - mu1 * ddudz1));
        rhs = rhs - (0.25 * (ddv3 * jwm * dwdy3 + ddv4 * jwp * dwdy4) - ih * rdx2[j] * (mu4 * ddvdz4 * jwp - mu3 * ddvdz3 * jwm));
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACK * dt + 1.0; cf.c = mAPK * dt; cf.a = mAMK * dt; cf.d[0] = rhs * dt;
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, li(l), 1 + blockIdx.y, r + 1)] = x[0]; }
};

// mu1..mu4 of solvedW's last stage-1 iteration (i = N1, j = N2, k = N3).
__device__ __forceinline__ void dw_stale_mu(const Grid &g, const Fields &f, double &mu1, double &mu2, double &mu3, double &mu4)
{
    const int i = g.N1, j = g.N2, k = g.N3, im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1, km = k - 1;
    const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx;
    const double *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const double mxz = 0.5 * (dx3[km] * MU(j, k) + dx3[k] * MU(j, km)) * rdmx3[k];
    mu1 = 0.5 * (dx1[im] * mxz + dx1[i] * mxz) * rdmx1[i];
    mu2 = 0.5 * (dx1[ip] * mxz + dx1[i] * mxz) * rdmx1[ip];
    const double mua = 0.5 * (dx3[km] * MU(jm, k) + dx3[k] * MU(jm, km)) * rdmx3[k];
    const double mub = 0.5 * (dx3[km] * MU(jp, k) + dx3[k] * MU(jp, km)) * rdmx3[k];
    mu3 = 0.5 * (dx2[jm] * mxz + dx2[j] * mua) * rdmx2[j];
    mu4 = 0.5 * (dx2[jp] * mxz + dx2[j] * mub) * rdmx2[jp];
}

struct DWX {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = true;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt, mu1, mu2, mu3, mu4; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dw_stale_mu(g, f, s.mu1, s.mu2, s.mu3, s.mu4);
        return s;
    }
    __device__ int lj(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return lj(l) <= g.N2; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = r + 1, j = lj(l), k = 1 + blockIdx.y, ip = i + 1, km = k - 1;
        const Phys &p = g.ph;
        const double *dx3 = g.m3.dx, *rdx1 = g.m1.rdx, *rdmx1 = g.m1.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sk = (long long)g.P1 * g.P2;
        const double mu1 = st.mu1, mu2 = st.mu2, mu3 = st.mu3, mu4 = st.mu4;
        (void)mu1; (void)mu2; (void)mu3; (void)mu4;
        const double u1 = (dx3[km] * ld(f.U + c) + dx3[k] * ld(f.U + c - sk)) * rdmx3[k] * 0.5;
        const double u2 = (dx3[km] * ld(f.U + c + 1) + dx3[k] * ld(f.U + c + 1 - sk)) * rdmx3[k] * 0.5;
        const double invRhoc = 0.5 * (dx3[km] * IR(j, k) + dx3[k] * IR(j, km)) * rdmx3[k];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACI = ih * rdx1[i] * (mu2 * rdmx1[ip] + mu1 * rdmx1[i]) + 0.25 * (-u2 * rdmx1[ip] + u1 * rdmx1[i]);
        const double mAPI = -ih * rdx1[i] * mu2 * rdmx1[ip] + 0.25 * (u2 * rdmx1[ip]);
        const double mAMI = -ih * rdx1[i] * mu1 * rdmx1[i] + 0.25 * (-u1 * rdmx1[i]);
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACI * dt + 1.0; cf.c = mAPI * dt; cf.a = mAMI * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { f.R[ix(g, r + 1, lj(l), 1 + blockIdx.y)] = x[0]; }
};

struct DWY {
    static constexpr int NRHS = 1;
    static constexpr bool CONTIG = false;
    Grid g; Fields f; int TL;
    __device__ bool skip() const { return blown(g); }
    struct State { double dt, mu1, mu2, mu3, mu4; };
    __device__ State prepare() const
    {
        State s;
        s.dt = g.scal[S_DT];
        dw_stale_mu(g, f, s.mu1, s.mu2, s.mu3, s.mu4);
        return s;
    }
    __device__ int li(int l) const { return 1 + blockIdx.x * TL + l; }
    __device__ bool line_ok(int l) const { return li(l) <= g.N1; }
    __device__ Coef<1> build(int l, int r, const State &st) const
    {
        const int i = li(l), j = r + 1, k = 1 + blockIdx.y, jp = j + 1, km = g.N3 - 1;
        const Phys &p = g.ph;
        const double *dx3 = g.m3.dx, *rdx2 = g.m2.rdx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
        const long long c = ix(g, i, j, k), sj = g.P1;
        const double jwm = (j == 1) ? 0.0 : 1.0, jwp = (j == g.N2) ? 0.0 : 1.0;
        const double mu1 = st.mu1, mu2 = st.mu2, mu3 = st.mu3, mu4 = st.mu4;
        (void)mu1; (void)mu2; (void)mu3; (void)mu4;
        const long long ckm = ix(g, i, j, km);
        const double v3 = (dx3[km] * ld(f.V + c) + dx3[k] * ld(f.V + ckm)) * rdmx3[k] * 0.5;
        const double v4 = (dx3[km] * ld(f.V + c + sj) + dx3[k] * ld(f.V + ckm + sj)) * rdmx3[k] * 0.5;
        const double invRhoc = 0.5 * (dx3[km] * IR(j, k) + dx3[k] * IR(j, km)) * rdmx3[k];
        const double ih = 0.5 * p.Cmu * invRhoc;
        const double mACJ = ih * rdx2[j] * (mu4 * rdmx2[jp] + mu3 * rdmx2[j]) + 0.25 * (-v4 * rdmx2[jp] + v3 * rdmx2[j]);
        const double mAPJ = (-ih * rdx2[j] * mu4 * rdmx2[jp] + 0.25 * (v4 * rdmx2[jp])) * jwp;
        const double mAMJ = (-ih * rdx2[j] * mu3 * rdmx2[j] + 0.25 * (-v3 * rdmx2[j])) * jwm;
        const double dt = st.dt;
        Coef<1> cf;
        cf.b = mACJ * dt + 1.0; cf.c = mAPJ * dt; cf.a = mAMJ * dt; cf.d[0] = ld(f.R + c);
        return cf;
    }
    __device__ void emit(int l, int r, const double *x, const State &st) const { store_periodic(g, f.dW, li(l), r + 1, 1 + blockIdx.y, x[0]); }
};

void launch_solve_du(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    LinePlan pz = make_line_plan(g.N3, true, cx.tl_strided), px = make_line_plan(g.N1, true, cx.tl_contig);
    LinePlan py = make_line_plan(g.N2, false, cx.tl_strided);
    launch_lines(DUZ{g, cx.f, pz.TL}, pz, dim3((g.N1 + pz.TL - 1) / pz.TL, g.N2), s, K_DU_Z, cx);
    launch_lines(DUX{g, cx.f, px.TL}, px, dim3((g.N2 + px.TL - 1) / px.TL, g.N3), s, K_DU_X, cx);
    launch_lines(DUY{g, cx.f, py.TL}, py, dim3((g.N1 + py.TL - 1) / py.TL, g.N3), s, K_DU_Y, cx);
}

void launch_solve_dv(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    LinePlan pz = make_line_plan(g.N3, true, cx.tl_strided), px = make_line_plan(g.N1, true, cx.tl_contig);
    LinePlan py = make_line_plan(g.N2 - 1, false, cx.tl_strided);
    launch_lines(DVZ{g, cx.f, pz.TL}, pz, dim3((g.N1 + pz.TL - 1) / pz.TL, g.N2 - 1), s, K_DV_Z, cx);
    launch_lines(DVX{g, cx.f, px.TL}, px, dim3((g.N2 - 1 + px.TL - 1) / px.TL, g.N3), s, K_DV_X, cx);
    launch_lines(DVY{g, cx.f, py.TL}, py, dim3((g.N1 + py.TL - 1) / py.TL, g.N3), s, K_DV_Y, cx);
}

void launch_solve_dw(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    LinePlan pz = make_line_plan(g.N3, true, cx.tl_strided), px = make_line_plan(g.N1, true, cx.tl_contig);
    LinePlan py = make_line_plan(g.N2, false, cx.tl_strided);
    launch_lines(DWZ{g, cx.f, pz.TL}, pz, dim3((g.N1 + pz.TL - 1) / pz.TL, g.N2), s, K_DW_Z, cx);
    launch_lines(DWX{g, cx.f, px.TL}, px, dim3((g.N2 + px.TL - 1) / px.TL, g.N3), s, K_DW_X, cx);
    launch_lines(DWY{g, cx.f, py.TL}, py, dim3((g.N1 + py.TL - 1) / py.TL, g.N3), s, K_DW_Y, cx);
}

// ---------------------------------------------------------------------------
// blockLdV (:1278-1356): dV -= dt*M23 dW, j = 2..N2, then ghost(dV).
// ---------------------------------------------------------------------------
__global__ void blockld_v_kernel(Grid g, Fields f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 2 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const int jm = j - 1, km = k - 1, kp = k + 1;
    const double *dx2 = g.m2.dx, *dx3 = g.m3.dx, *rdx3 = g.m3.rdx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
    const double dWc = ld(f.dW + c), dWym = ld(f.dW + c - sj), dWzp = ld(f.dW + c + sk), dWzpym = ld(f.dW + c + sk - sj);
    const double dwm5 = (dx2[jm] * dWc + dx2[j] * dWym) * rdmx2[j] * 0.5;
    const double dwm6 = (dx2[jm] * dWzp + dx2[j] * dWzpym) * rdmx2[j] * 0.5;
    const double ddwdy5 = (dWc - dWym) * rdmx2[j], ddwdy6 = (dWzp - dWzpym) * rdmx2[j];
    const double Vc = ld(f.V + c);
    const double dvdz5 = (Vc - ld(f.V + c - sk)) * rdmx3[k], dvdz6 = (ld(f.V + c + sk) - Vc) * rdmx3[kp];
    const double invRhoc = 0.5 * (dx2[jm] * IR(j, k) + dx2[j] * IR(jm, k)) * rdmx2[j];
    const double mua = 0.5 * (dx2[jm] * MU(j, km) + dx2[j] * MU(jm, km)) * rdmx2[j];
    const double muc = 0.5 * (dx2[jm] * MU(j, k) + dx2[j] * MU(jm, k)) * rdmx2[j];
    const double mub = 0.5 * (dx2[jm] * MU(j, kp) + dx2[j] * MU(jm, kp)) * rdmx2[j];
    const double mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
    const double mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
    const double dt = g.scal[S_DT];
    const double v = f.dV[c] - dt * (0.25 * (dwm5 * dvdz5 + dwm6 * dvdz6) - 0.5 * g.ph.Cmu * invRhoc * rdx3[k] * (mu6 * ddwdy6 - mu5 * ddwdy5));
    store_periodic(g, f.dV, i, j, k, v);
}

void launch_blockld_v(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    probe_begin(cx, K_BLOCKLDV, s);
    blockld_v_kernel<<<dim3((g.N1 + 127) / 128, g.N2 - 1, g.N3), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_BLOCKLDV, s);
    record_launch_error("blockld_v");
}

// blockLdU (:1362-1460): dU -= dt*(M12 dV + M13 dW), j = 1..N2 (no ghost
// update follows in the driver; only interior dU is read afterwards).
__global__ void blockld_u_kernel(Grid g, Fields f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const int im = i - 1, jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
    const double *dx1 = g.m1.dx, *dx2 = g.m2.dx, *dx3 = g.m3.dx, *rdx2 = g.m2.rdx, *rdx3 = g.m3.rdx;
    const double *rdmx1 = g.m1.rdmx, *rdmx2 = g.m2.rdmx, *rdmx3 = g.m3.rdmx;
    const long long c = ix(g, i, j, k), sj = g.P1, sk = (long long)g.P1 * g.P2;
    const double jum = (j == 1) ? 0.0 : 1.0, jup = (j == g.N2) ? 0.0 : 1.0;
    const double Mjk = MU(j, k), iRjk = IR(j, k);
    const double invRhoc = 0.5 * (dx1[im] * iRjk + dx1[i] * iRjk) * rdmx1[i];
    const double dVc = ld(f.dV + c), dVxm = ld(f.dV + c - 1), dVyp = ld(f.dV + c + sj), dVxmyp = ld(f.dV + c - 1 + sj);
    const double dvm3 = (dx1[i] * dVxm + dx1[im] * dVc) * rdmx1[i] * 0.5 * jum;
    const double dvm4 = (dx1[i] * dVxmyp + dx1[im] * dVyp) * rdmx1[i] * 0.5 * jup;
    const double Uc = ld(f.U + c);
    const double dudy3 = (Uc - ld(f.U + c - sj)) * rdmx2[j], dudy4 = (ld(f.U + c + sj) - Uc) * rdmx2[jp];
    const double dvmdx3 = (dVc - dVxm) * rdmx1[i] * jum, dvmdx4 = (dVyp - dVxmyp) * rdmx1[i] * jup;
    double mua = 0.5 * (dx1[im] * MU(jm, k) + dx1[i] * MU(jm, k)) * rdmx1[i];
    const double muc = 0.5 * (dx1[im] * Mjk + dx1[i] * Mjk) * rdmx1[i];
    double mub = 0.5 * (dx1[im] * MU(jp, k) + dx1[i] * MU(jp, k)) * rdmx1[i];
    const double mu3 = 0.5 * (dx2[jm] * muc + dx2[j] * mua) * rdmx2[j];
    const double mu4 = 0.5 * (dx2[jp] * muc + dx2[j] * mub) * rdmx2[jp];
    const double dWc = ld(f.dW + c), dWxm = ld(f.dW + c - 1), dWzp = ld(f.dW + c + sk), dWxmzp = ld(f.dW + c - 1 + sk);
    const double dwm5 = (dx1[i] * dWxm + dx1[im] * dWc) * rdmx1[i] * 0.5;
    const double dwm6 = (dx1[i] * dWxmzp + dx1[im] * dWzp) * rdmx1[i] * 0.5;
    const double dudz5 = (Uc - ld(f.U + c - sk)) * rdmx3[k], dudz6 = (ld(f.U + c + sk) - Uc) * rdmx3[kp];
    const double dwmdx5 = (dWc - dWxm) * rdmx1[i], dwmdx6 = (dWzp - dWxmzp) * rdmx1[i];
    mua = 0.5 * (dx1[im] * MU(j, km) + dx1[i] * MU(j, km)) * rdmx1[i];
    mub = 0.5 * (dx1[im] * MU(j, kp) + dx1[i] * MU(j, kp)) * rdmx1[i];
    const double mu5 = 0.5 * (dx3[km] * muc + dx3[k] * mua) * rdmx3[k];
    const double mu6 = 0.5 * (dx3[kp] * muc + dx3[k] * mub) * rdmx3[kp];
    const double dt = g.scal[S_DT], Cmu = g.ph.Cmu;
    f.dU[c] = f.dU[c]
        - dt * (0.25 * (dvm4 * dudy4 + dvm3 * dudy3) - 0.5 * Cmu * invRhoc * rdx2[j] * (mu4 * dvmdx4 - mu3 * dvmdx3))
        - dt * (0.25 * (dwm6 * dudz6 + dwm5 * dudz5) - 0.5 * Cmu * invRhoc * rdx3[k] * (mu6 * dwmdx6 - mu5 * dwmdx5));
}

void launch_blockld_u(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    probe_begin(cx, K_BLOCKLDU, s);
    blockld_u_kernel<<<dim3((g.N1 + 127) / 128, g.N2, g.N3), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_BLOCKLDU, s);
    record_launch_error("blockld_u");
}

// Standalone mpi_momentum_pseudoupdateUVW (:178-208) + ghost(U,V,W): writes the
// second buffers; the caller swaps them in.  The step normally fuses this into
// the pressure right-hand side (tcs_pressure.cu).
__global__ void pseudo_update_kernel(Grid g, Fields f)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > g.N1 || blown(g)) return;
    const long long c = ix(g, i, j, k);
    const double vmask = (j == 1) ? 0.0 : 1.0;     // dble(2 - j_indexS) on the lower plane
    store_periodic(g, f.Un, i, j, k, f.U[c] + f.dU[c]);
    store_periodic(g, f.Vn, i, j, k, f.V[c] + f.dV[c] * vmask);
    store_periodic(g, f.Wn, i, j, k, f.W[c] + f.dW[c]);
}

void launch_pseudo_update(const Ctx &cx, cudaStream_t s)
{
    const Grid &g = cx.g;
    probe_begin(cx, K_PSEUDO, s);
    pseudo_update_kernel<<<dim3((g.N1 + 127) / 128, g.N2, g.N3), 128, 0, s>>>(g, cx.f);
    probe_end(cx, K_PSEUDO, s);
    record_launch_error("pseudo_update");
}

#undef MU
#undef IR

} // namespace tcs
