"""The U-momentum z sweep evaluates the right-hand side of
module_solve_momentum.f90:281-420 (stage 1 of mpi_momentum_solvedU) in a
reduced form: the explicit operator minus the three implicit operators
applied to U collapses in x and z (and in y away from the walls) to
4 ih vu1 + 2 ih (vu3 + vu13) - (u1 dudx1 + u2 dudx2)/2 - (w5 dudz5 + w6 dudz6)/2
(+ 2 ih (vu2 + vu12) - (v3 dudy3 + v4 dudy4)/2 on interior planes).  The x
part relies on Mu being constant along i, which is the reference's own
row-wise assignment of Mu (module_solve_momentum.f90:165, 168).  This checks
the identity on random stencil values: the reference's expression (as the
oracle restates it) against the kernel's reduced one, for an interior plane
and for both wall-adjacent planes, where the kernel keeps the reference's
y terms."""
import numpy as np


def forms(v, jum, jup):
    (dx1m, dx1, dmx1, dx2m, dx2, dx2p, dmx2, dmx2p, dx3m, dx3, dx3p, dmx3, dmx3p,
     Uc, Uxm, Uxp, Uym, Uyp, Uzm, Uzp, Vc, Vxm, Vyp, Vxmyp, Wc, Wxm, Wzp, Wxmzp,
     Mjk, Mjmk, Mjpk, Mjkm, Mjkp, iRjk, Pc, Pxm, Tcv, Txm,
     Cmu, Cmp, Cmt, a12pera11, DeltaT, Ubt, Uup, Vbt, Vup) = v
    # Mu and invRho are constant along i (row-wise), so Mu(i) = Mu(im) = Mjk etc.
    u1, u2 = 0.5 * (Uxm + Uc), 0.5 * (Uxp + Uc)
    v3 = 0.5 * (dx1m * Vc + dx1 * Vxm) / dmx1
    v4 = 0.5 * (dx1m * Vyp + dx1 * Vxmyp) / dmx1
    w5 = 0.5 * (dx1m * Wc + dx1 * Wxm) / dmx1
    w6 = 0.5 * (dx1m * Wzp + dx1 * Wxmzp) / dmx1
    dudx1, dudx2 = (Uc - Uxm) / dx1m, (Uxp - Uc) / dx1
    dudy3, dudy4 = (Uc - Uym) / dmx2, (Uyp - Uc) / dmx2p
    dudz5, dudz6 = (Uc - Uzm) / dmx3, (Uzp - Uc) / dmx3p
    dvdx3, dvdx4 = (Vc - Vxm) / dmx1, (Vyp - Vxmyp) / dmx1
    dwdx5, dwdx6 = (Wc - Wxm) / dmx1, (Wzp - Wxmzp) / dmx1
    mua = 0.5 * (dx1m * Mjmk + dx1 * Mjmk) / dmx1
    muc = 0.5 * (dx1m * Mjk + dx1 * Mjk) / dmx1
    mub = 0.5 * (dx1m * Mjpk + dx1 * Mjpk) / dmx1
    mu3 = 0.5 * (dx2m * muc + dx2 * mua) / dmx2
    mu4 = 0.5 * (dx2p * muc + dx2 * mub) / dmx2p
    mua = 0.5 * (dx1m * Mjkm + dx1 * Mjkm) / dmx1
    mub = 0.5 * (dx1m * Mjkp + dx1 * Mjkp) / dmx1
    mu5 = 0.5 * (dx3m * muc + dx3 * mua) / dmx3
    mu6 = 0.5 * (dx3p * muc + dx3 * mub) / dmx3p
    invRhoc = 0.5 * (dx1m * iRjk + dx1 * iRjk) / dmx1
    ih = 0.5 * Cmu * invRhoc
    vu1 = (Mjk * dudx2 - Mjk * dudx1) / dmx1
    vu2 = (mu4 * dudy4 - mu3 * dudy3) / dx2
    vu3 = (mu6 * dudz6 - mu5 * dudz5) / dx3
    vu12 = (mu4 * dvdx4 - mu3 * dvdx3) / dx2
    vu13 = (mu6 * dwdx6 - mu5 * dwdx5) / dx3
    Tc = 0.5 * (dx1m * Tcv + dx1 * Txm) / dmx1
    body = -Cmp * invRhoc * (Pc - Pxm) / dmx1 + Cmt * (Tc + a12pera11 * (Tc * Tc) * DeltaT) * invRhoc
    ubc_dn = 0.25 * v3 / dmx2 * Ubt - 0.25 * dudy3 * (dx1 * Vbt + dx1m * Vbt) / dmx1 * 0.5
    ubc_up = -0.25 * v4 / dmx2p * Uup - 0.25 * dudy4 * (dx1 * Vup + dx1m * Vup) / dmx1 * 0.5
    ubc_dn = ubc_dn + ih / dx2 * mu3 / dmx2 * Ubt - ih / dx2 * mu3 / dmx1 * (Vbt - Vbt)
    ubc_up = ubc_up + ih / dx2 * mu4 / dmx2p * Uup + ih / dx2 * mu4 / dmx1 * (Vup - Vup)
    mACI = ih / dmx1 * (Mjk / dx1 + Mjk / dx1m) * 2.0 + 0.25 * (dudx2 * 0.5 + dudx1 * 0.5 - u2 / dx1 + u1 / dx1m)
    mAPI = -ih / dmx1 * Mjk / dx1 * 2.0 + 0.25 * (u2 / dx1 + dudx2 * 0.5)
    mAMI = -ih / dmx1 * Mjk / dx1m * 2.0 + 0.25 * (-u1 / dx1m + dudx1 * 0.5)
    mACJ = ih / dx2 * (mu4 / dmx2p + mu3 / dmx2) + 0.25 * (-v4 / dmx2p + v3 / dmx2)
    mAPJ = (-ih / dx2 * mu4 / dmx2p + 0.25 * (v4 / dmx2p)) * jup
    mAMJ = (-ih / dx2 * mu3 / dmx2 + 0.25 * (-v3 / dmx2)) * jum
    mACK = ih / dx3 * (mu6 / dmx3p + mu5 / dmx3) + 0.25 * (-w6 / dmx3p + w5 / dmx3)
    mAPK = -ih / dx3 * mu6 / dmx3p + 0.25 * (w6 / dmx3p)
    mAMK = -ih / dx3 * mu5 / dmx3 + 0.25 * (-w5 / dmx3)
    # the reference (module_solve_momentum.f90:281-420, as the oracle restates it)
    full = ih * (2.0 * vu1 + vu2 + vu3 + vu12 + vu13) + body + (1.0 - jum) * ubc_dn + (1.0 - jup) * ubc_up
    implicit = (mAPI * Uxp + mACI * Uc + mAMI * Uxm + mAPJ * Uyp + mACJ * Uc + mAMJ * Uym
                + mAPK * Uzp + mACK * Uc + mAMK * Uzm)
    full = full - implicit
    full = full - (0.25 * (v4 * jup * dudy4 + v3 * jum * dudy3) - ih / dx2 * (mu4 * dvdx4 * jup - mu3 * dvdx3 * jum))
    full = full - (0.25 * (w6 * dudz6 + w5 * dudz5) - ih / dx3 * (mu6 * dwdx6 - mu5 * dwdx5))
    # the kernel's reduced form (DUZ in csrc/tcs_momentum.cu)
    red = 4.0 * ih * vu1 + 2.0 * ih * (vu3 + vu13) - 0.5 * (u1 * dudx1 + u2 * dudx2) - 0.5 * (w5 * dudz5 + w6 * dudz6) + body
    if jum == 1.0 and jup == 1.0:
        red = red + 2.0 * ih * (vu2 + vu12) - 0.5 * (v3 * dudy3 + v4 * dudy4)
    else:
        red = (red + ih * (vu2 + vu12) + (1.0 - jum) * ubc_dn + (1.0 - jup) * ubc_up
               - (mAPJ * Uyp + mACJ * Uc + mAMJ * Uym)
               - (0.25 * (v4 * jup * dudy4 + v3 * jum * dudy3) - ih / dx2 * (mu4 * dvdx4 * jup - mu3 * dvdx3 * jum)))
    scale = sum(abs(t) for t in (mAPI * Uxp, mACI * Uc, mAPK * Uzp, mACK * Uc, mACJ * Uc, ih * vu1, ih * vu3, body))
    return full, red, scale


def test_reduced_u_momentum_rhs_matches_reference_expression():
    rng = np.random.default_rng(17)
    worst = 0.0
    for _ in range(500):
        metrics = rng.uniform(0.5, 2.0, 13)
        vel = rng.uniform(-1.0, 1.0, 15)
        mu = rng.uniform(0.5, 2.0, 6)
        pt = rng.uniform(-1.0, 1.0, 4)
        consts = rng.uniform(0.5, 2.0, 5)
        bcs = rng.uniform(-1.0, 1.0, 4)
        v = np.concatenate([metrics, vel, mu, pt, consts, bcs])
        for jum, jup in ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0)):
            full, red, scale = forms(v, jum, jup)
            worst = max(worst, abs(full - red) / scale)
    assert worst < 1e-13, worst


def test_identity_needs_the_row_wise_viscosity():
    # with Mu(i) != Mu(im) the x part does not collapse: the check is not vacuous
    rng = np.random.default_rng(5)
    v = np.concatenate([rng.uniform(0.5, 2.0, 13), rng.uniform(-1.0, 1.0, 15), rng.uniform(0.5, 2.0, 6),
                        rng.uniform(-1.0, 1.0, 4), rng.uniform(0.5, 2.0, 5), rng.uniform(-1.0, 1.0, 4)])
    full, red, scale = forms(v, 1.0, 1.0)
    # the explicit viscous x term with Mu(im) = Mu(i) - 0.3: 2 ih vu1 gains 2 ih 0.3 dudx1 / dmx1,
    # while the implicit rows (which use Mu(i) only) do not change
    dx1m, dx1, dmx1, Uc, Uxm, iRjk, Cmu = v[0], v[1], v[2], v[13], v[14], v[33], v[38]
    ih = 0.5 * Cmu * (0.5 * (dx1m * iRjk + dx1 * iRjk) / dmx1)
    delta = ih * 2.0 * 0.3 * (Uc - Uxm) / dx1m / dmx1
    assert abs((full + delta) - red) / scale > 1e-6
