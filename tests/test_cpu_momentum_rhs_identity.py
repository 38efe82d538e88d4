"""The momentum z sweeps evaluate their right-hand sides in a reduced form,
checked here for U, V and W (the V and W forms add the dU and dV cross terms).  The
U-momentum z sweep evaluates the right-hand side of
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


def forms_w(v, jwm, jwp):
    """solvedW stage 1 (module_solve_momentum.f90:988-1130, as the oracle
    restates it) against the reduced form of the W-momentum z sweep (DWZ in
    csrc/tcs_momentum.cu), with the dU and dV cross terms of the reference."""
    (dx1m, dx1, dx1p, dmx1, dmx1p, dx2m, dx2, dx2p, dmx2, dmx2p, dx3m, dx3, dmx3,
     Wc, Wxm, Wxp, Wym, Wyp, Wzm, Wzp, Uc, Uzm, Uxp, Uxpzm, Vc, Vzm, Vyp, Vypzm,
     dUc, dUzm, dUxp, dUxpzm, dVc, dVzm, dVyp, dVypzm, Pc, Pzm,
     Mjk, Mjkm, Mjmk, Mjmkm, Mjpk, Mjpkm, iRjk, iRjkm, Cmu, Cmp, Vbt, Vup, Wbt, Wup) = v
    w5, w6 = 0.5 * (Wc + Wzm), 0.5 * (Wc + Wzp)
    u1 = (dx3m * Uc + dx3 * Uzm) / dmx3 * 0.5
    u2 = (dx3m * Uxp + dx3 * Uxpzm) / dmx3 * 0.5
    v3 = (dx3m * Vc + dx3 * Vzm) / dmx3 * 0.5
    v4 = (dx3m * Vyp + dx3 * Vypzm) / dmx3 * 0.5
    dwdx1, dwdx2 = (Wc - Wxm) / dmx1, (Wxp - Wc) / dmx1p
    dwdy3, dwdy4 = (Wc - Wym) / dmx2, (Wyp - Wc) / dmx2p
    dwdz5, dwdz6 = (Wc - Wzm) / dx3m, (Wzp - Wc) / dx3
    dudz1, dudz2 = (Uc - Uzm) / dmx3, (Uxp - Uxpzm) / dmx3
    dvdz3, dvdz4 = (Vc - Vzm) / dmx3, (Vyp - Vypzm) / dmx3
    ddudz1, ddudz2 = (dUc - dUzm) / dmx3, (dUxp - dUxpzm) / dmx3
    ddvdz3, ddvdz4 = (dVc - dVzm) / dmx3, (dVyp - dVypzm) / dmx3
    ddu1 = (dx3m * dUc + dx3 * dUzm) / dmx3 * 0.5
    ddu2 = (dx3m * dUxp + dx3 * dUxpzm) / dmx3 * 0.5
    ddv3 = (dx3m * dVc + dx3 * dVzm) / dmx3 * 0.5 * jwm
    ddv4 = (dx3m * dVyp + dx3 * dVypzm) / dmx3 * 0.5 * jwp
    # Mu constant along i (row-wise): Mu(im) = Mu(i) = Mu(ip)
    mxz = 0.5 * (dx3m * Mjk + dx3 * Mjkm) / dmx3
    mu1 = 0.5 * (dx1m * mxz + dx1 * mxz) / dmx1
    mu2 = 0.5 * (dx1p * mxz + dx1 * mxz) / dmx1p
    mua = 0.5 * (dx3m * Mjmk + dx3 * Mjmkm) / dmx3
    mub = 0.5 * (dx3m * Mjpk + dx3 * Mjpkm) / dmx3
    mu3 = 0.5 * (dx2m * mxz + dx2 * mua) / dmx2
    mu4 = 0.5 * (dx2p * mxz + dx2 * mub) / dmx2p
    invRhoc = 0.5 * (dx3m * iRjk + dx3 * iRjkm) / dmx3
    ih = 0.5 * Cmu * invRhoc
    vw1 = (mu2 * dwdx2 - mu1 * dwdx1) / dx1
    vw2 = (mu4 * dwdy4 - mu3 * dwdy3) / dx2
    vw3 = (Mjk * dwdz6 - Mjkm * dwdz5) / dmx3
    vw31 = (mu2 * dudz2 - mu1 * dudz1) / dx1
    vw32 = (mu4 * dvdz4 - mu3 * dvdz3) / dx2
    press = -Cmp * invRhoc * (Pc - Pzm) / dmx3
    zbc_dn = 0.25 * v3 / dmx2 * Wbt - 0.25 * dwdy3 * (dx3m * Vbt + dx3 * Vbt) / dmx3 * 0.5
    zbc_up = -0.25 * v4 / dmx2p * Wup - 0.25 * dwdy4 * (dx3m * Vup + dx3 * Vup) / dmx3 * 0.5
    zbc_dn = zbc_dn + ih / dx2 * mu3 / dmx2p * Wbt - ih / dx2 * mu3 / dmx3 * (Vbt - Vbt)
    zbc_up = zbc_up + ih / dx2 * mu4 / dmx2 * Wup + ih / dx2 * mu4 / dmx3 * (Vup - Vup)
    mACI = ih / dx1 * (mu2 / dmx1p + mu1 / dmx1) + 0.25 * (-u2 / dmx1p + u1 / dmx1)
    mAPI = -ih / dx1 * mu2 / dmx1p + 0.25 * (u2 / dmx1p)
    mAMI = -ih / dx1 * mu1 / dmx1 + 0.25 * (-u1 / dmx1)
    mACJ = ih / dx2 * (mu4 / dmx2p + mu3 / dmx2) + 0.25 * (-v4 / dmx2p + v3 / dmx2)
    mAPJ = (-ih / dx2 * mu4 / dmx2p + 0.25 * (v4 / dmx2p)) * jwp
    mAMJ = (-ih / dx2 * mu3 / dmx2 + 0.25 * (-v3 / dmx2)) * jwm
    mACK = ih / dmx3 * (Mjk / dx3 + Mjkm / dx3m) * 2.0 + 0.25 * (-w6 / dx3 + w5 / dx3m + 0.5 * dwdz6 + 0.5 * dwdz5)
    mAPK = -ih / dmx3 * Mjk / dx3 * 2.0 + 0.25 * (w6 / dx3 + 0.5 * dwdz6)
    mAMK = -ih / dmx3 * Mjkm / dx3m * 2.0 + 0.25 * (-w5 / dx3m + 0.5 * dwdz5)
    full = ih * (vw1 + vw2 + 2.0 * vw3 + vw31 + vw32) + press + (1.0 - jwm) * zbc_dn + (1.0 - jwp) * zbc_up
    full = full - (mAPI * Wxp + mACI * Wc + mAMI * Wxm + mAPJ * Wyp + mACJ * Wc + mAMJ * Wym
                   + mAPK * Wzp + mACK * Wc + mAMK * Wzm)
    full = full - (0.25 * (u2 * dwdx2 + u1 * dwdx1) - ih / dx1 * (mu2 * dudz2 - mu1 * dudz1))
    full = full - (0.25 * (v3 * jwm * dwdy3 + v4 * jwp * dwdy4) - ih / dx2 * (mu4 * dvdz4 * jwp - mu3 * dvdz3 * jwm))
    full = full - (0.25 * (ddu2 * dwdx2 + ddu1 * dwdx1) - ih / dx1 * (mu2 * ddudz2 - mu1 * ddudz1))
    full = full - (0.25 * (ddv3 * jwm * dwdy3 + ddv4 * jwp * dwdy4) - ih / dx2 * (mu4 * ddvdz4 * jwp - mu3 * ddvdz3 * jwm))
    red = (2.0 * ih * (vw1 + vw31) + 4.0 * ih * vw3 - 0.5 * (u1 * dwdx1 + u2 * dwdx2) - 0.5 * (w5 * dwdz5 + w6 * dwdz6)
           - 0.25 * (ddu1 * dwdx1 + ddu2 * dwdx2) + ih / dx1 * (mu2 * ddudz2 - mu1 * ddudz1) + press)
    if jwm == 1.0 and jwp == 1.0:
        red = (red + 2.0 * ih * (vw2 + vw32) - 0.5 * (v3 * dwdy3 + v4 * dwdy4)
               - 0.25 * (ddv3 * dwdy3 + ddv4 * dwdy4) + ih / dx2 * (mu4 * ddvdz4 - mu3 * ddvdz3))
    else:
        red = (red + ih * (vw2 + vw32) + (1.0 - jwm) * zbc_dn + (1.0 - jwp) * zbc_up - (mAPJ * Wyp + mACJ * Wc + mAMJ * Wym)
               - (0.25 * (v3 * jwm * dwdy3 + v4 * jwp * dwdy4) - ih / dx2 * (mu4 * dvdz4 * jwp - mu3 * dvdz3 * jwm))
               - (0.25 * (ddv3 * jwm * dwdy3 + ddv4 * jwp * dwdy4) - ih / dx2 * (mu4 * ddvdz4 * jwp - mu3 * ddvdz3 * jwm)))
    scale = sum(abs(t) for t in (mAPI * Wxp, mACI * Wc, mAPK * Wzp, mACK * Wc, mACJ * Wc, ih * vw1, ih * vw3, press))
    return full, red, scale


def test_reduced_w_momentum_rhs_matches_reference_expression():
    rng = np.random.default_rng(23)
    worst = 0.0
    for _ in range(500):
        v = np.concatenate([rng.uniform(0.5, 2.0, 13), rng.uniform(-1.0, 1.0, 25), rng.uniform(0.5, 2.0, 8),
                            rng.uniform(0.5, 2.0, 2), rng.uniform(-1.0, 1.0, 4)])
        for jwm, jwp in ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0)):
            full, red, scale = forms_w(v, jwm, jwp)
            worst = max(worst, abs(full - red) / scale)
    assert worst < 1e-13, worst


def forms_v(v, jvm, jvp):
    """solvedV stage 1 (module_solve_momentum.f90:626-780, as the oracle
    restates it) against the reduced form of the V-momentum z sweep (DVZ in
    csrc/tcs_momentum.cu), with the reference's dU cross terms; jvm, jvp are
    jS_BC(j+1) and jS_BC(j-1)."""
    (dx1m, dx1, dx1p, dmx1, dmx1p, dx2m, dx2, dmx2, dx3m, dx3, dx3p, dmx3, dmx3p,
     Vc, Vym, Vyp, Vxm, Vxp, Vzm, Vzp, Uc, Uym, Uxp, Uxpym, Wc, Wym, Wzp, Wzpym,
     dUc, dUym, dUxp, dUxpym, Pc, Pym,
     Mjk, Mjmk, Mjkm, Mjmkm, Mjkp, Mjmkp, iRjk, iRjmk, Cmu, Cmp, Vbt, Vup) = v
    v3, v4 = 0.5 * (Vym + Vc), 0.5 * (Vc + Vyp)
    u1 = (dx2m * Uc + dx2 * Uym) / dmx2 * 0.5
    u2 = (dx2m * Uxp + dx2 * Uxpym) / dmx2 * 0.5
    w5 = (dx2m * Wc + dx2 * Wym) / dmx2 * 0.5
    w6 = (dx2m * Wzp + dx2 * Wzpym) / dmx2 * 0.5
    ddu1 = (dx2m * dUc + dx2 * dUym) / dmx2 * 0.5
    ddu2 = (dx2m * dUxp + dx2 * dUxpym) / dmx2 * 0.5
    dvdx1, dvdx2 = (Vc - Vxm) / dmx1, (Vxp - Vc) / dmx1p
    dvdy3, dvdy4 = (Vc - Vym) / dx2m, (Vyp - Vc) / dx2
    dvdz5, dvdz6 = (Vc - Vzm) / dmx3, (Vzp - Vc) / dmx3p
    dudy1, dudy2 = (Uc - Uym) / dmx2, (Uxp - Uxpym) / dmx2
    dwdy5, dwdy6 = (Wc - Wym) / dmx2, (Wzp - Wzpym) / dmx2
    ddudy1, ddudy2 = (dUc - dUym) / dmx2, (dUxp - dUxpym) / dmx2
    # Mu constant along i (row-wise): the three x-neighbour averages coincide
    mxy = 0.5 * (dx2m * Mjk + dx2 * Mjmk) / dmx2
    mu1 = 0.5 * (dx1m * mxy + dx1 * mxy) / dmx1
    mu2 = 0.5 * (dx1p * mxy + dx1 * mxy) / dmx1p
    mua = 0.5 * (dx2m * Mjkm + dx2 * Mjmkm) / dmx2
    mub = 0.5 * (dx2m * Mjkp + dx2 * Mjmkp) / dmx2
    mu5 = 0.5 * (dx3m * mxy + dx3 * mua) / dmx3
    mu6 = 0.5 * (dx3p * mxy + dx3 * mub) / dmx3p
    invRhoc = 0.5 * (dx2m * iRjk + dx2 * iRjmk) / dmx2
    ih = 0.5 * Cmu * invRhoc
    vv1 = (mu2 * dvdx2 - mu1 * dvdx1) / dx1
    vv2 = (Mjk * dvdy4 - Mjmk * dvdy3) / dmx2
    vv3 = (mu6 * dvdz6 - mu5 * dvdz5) / dx3
    vv21 = (mu2 * dudy2 - mu1 * dudy1) / dx1
    vv23 = (mu6 * dwdy6 - mu5 * dwdy5) / dx3
    press = -Cmp * invRhoc * (Pc - Pym) / dmx2
    vbc_dn = 0.25 / dx2m * v3 * Vbt - 0.25 * 0.5 * dvdy3 * Vbt + ih / dmx2 * Mjmk / dx2m * Vbt * 2.0
    vbc_up = -0.25 / dx2 * v4 * Vup - 0.25 * 0.5 * dvdy4 * Vup + ih / dmx2 * Mjk / dx2 * Vup * 2.0
    mACI = ih / dx1 * (mu2 / dmx1p + mu1 / dmx1) + 0.25 * (-u2 / dmx1p + u1 / dmx1)
    mAPI = -ih / dx1 * mu2 / dmx1p + 0.25 * (u2 / dmx1p)
    mAMI = -ih / dx1 * mu1 / dmx1 + 0.25 * (-u1 / dmx1)
    mACJ = ih / dmx2 * (Mjk / dx2 + Mjmk / dx2m) * 2.0 + 0.25 * (dvdy4 * 0.5 + dvdy3 * 0.5 - v4 / dx2 + v3 / dx2m)
    mAPJ = (-ih / dmx2 * Mjk / dx2 * 2.0 + 0.25 * (v4 / dx2 + dvdy4 * 0.5)) * jvp
    mAMJ = (-ih / dmx2 * Mjmk / dx2m * 2.0 + 0.25 * (-v3 / dx2m + dvdy3 * 0.5)) * jvm
    mACK = ih / dx3 * (mu6 / dmx3p + mu5 / dmx3) + 0.25 * (-w6 / dmx3p + w5 / dmx3)
    mAPK = -ih / dx3 * mu6 / dmx3p + 0.25 * (w6 / dmx3p)
    mAMK = -ih / dx3 * mu5 / dmx3 + 0.25 * (-w5 / dmx3)
    full = ih * (vv1 + 2.0 * vv2 + vv3 + vv21 + vv23) + press + (1.0 - jvm) * vbc_dn + (1.0 - jvp) * vbc_up
    full = full - (mAPI * Vxp + mACI * Vc + mAMI * Vxm + mAPJ * Vyp + mACJ * Vc + mAMJ * Vym
                   + mAPK * Vzp + mACK * Vc + mAMK * Vzm)
    full = full - (0.25 * (u2 * dvdx2 + u1 * dvdx1) - ih / dx1 * (mu2 * dudy2 - mu1 * dudy1))
    full = full - (0.25 * (w6 * dvdz6 + w5 * dvdz5) - ih / dx3 * (mu6 * dwdy6 - mu5 * dwdy5))
    full = full - (0.25 * (ddu2 * dvdx2 + ddu1 * dvdx1) - ih / dx1 * (mu2 * ddudy2 - mu1 * ddudy1))
    red = (2.0 * ih * (vv1 + vv21 + vv3 + vv23) - 0.5 * (u1 * dvdx1 + u2 * dvdx2) - 0.5 * (w5 * dvdz5 + w6 * dvdz6)
           - 0.25 * (ddu1 * dvdx1 + ddu2 * dvdx2) + ih / dx1 * (mu2 * ddudy2 - mu1 * ddudy1) + press)
    if jvp != 0.0 and jvm != 0.0:
        red = red + 4.0 * ih * vv2 - 0.5 * (v3 * dvdy3 + v4 * dvdy4)
    else:
        red = red + 2.0 * ih * vv2 + (1.0 - jvm) * vbc_dn + (1.0 - jvp) * vbc_up - (mAPJ * Vyp + mACJ * Vc + mAMJ * Vym)
    scale = sum(abs(t) for t in (mAPI * Vxp, mACI * Vc, mAPK * Vzp, mACK * Vc, mACJ * Vc, ih * vv1, ih * vv2, press))
    return full, red, scale


def test_reduced_v_momentum_rhs_matches_reference_expression():
    rng = np.random.default_rng(29)
    worst = 0.0
    for _ in range(500):
        v = np.concatenate([rng.uniform(0.5, 2.0, 13), rng.uniform(-1.0, 1.0, 21), rng.uniform(0.5, 2.0, 8),
                            rng.uniform(0.5, 2.0, 2), rng.uniform(-1.0, 1.0, 2)])
        for jvm, jvp in ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0)):
            full, red, scale = forms_v(v, jvm, jvp)
            worst = max(worst, abs(full - red) / scale)
    assert worst < 1e-13, worst
