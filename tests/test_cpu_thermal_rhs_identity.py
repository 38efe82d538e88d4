"""The thermal z sweep evaluates the right-hand side of
module_solve_thermal.f90:236-361 in a reduced form (the dK/dT products and
the dh*Tc*dv terms of the explicit operator and of the implicit operators
applied to T cancel).  This checks the identity itself on random stencil
values: the reference's expression (as the oracle and the kernel's wall
planes write it) against the reduced one, for an interior plane and for both
wall-adjacent planes, where the kernel keeps the reference's y terms."""
import numpy as np


def reference_rhs(v, jem, jep):
    (dx1, dx1m, dx1p, rdmx1, rdmx1p, rdx1, dx2, dx2m, dx2p, rdmx2, rdmx2p, rdx2,
     dx3, dx3m, dx3p, rdmx3, rdmx3p, rdx3, Tc, Txm, Txp, Tym, Typ, Tzm, Tzp,
     Kc, Kxm, Kxp, Kym, Kyp, Kzm, Kzp, dKc, dKxm, dKxp, dKym, dKyp, dKzm, dKzp,
     Uc, Uxp, Vc, Vyp, Wc, Wzp, irc, dirc, Ct, Tup, Tbt) = v
    h, dh = 0.5 * Ct * irc, 0.5 * Ct * dirc
    e1 = (dx1 * Txm + dx1m * Tc) * (0.5 * rdmx1); e2 = (dx1p * Tc + dx1 * Txp) * (0.5 * rdmx1p)
    e3 = (dx2 * Tym + dx2m * Tc) * (0.5 * rdmx2); e4 = (dx2p * Tc + dx2 * Typ) * (0.5 * rdmx2p)
    e5 = (dx3 * Tzm + dx3m * Tc) * (0.5 * rdmx3); e6 = (dx3p * Tc + dx3 * Tzp) * (0.5 * rdmx3p)
    dedx1, dedx2 = (Tc - Txm) * rdmx1, (Txp - Tc) * rdmx1p
    dedy3, dedy4 = (Tc - Tym) * rdmx2, (Typ - Tc) * rdmx2p
    dedz5, dedz6 = (Tc - Tzm) * rdmx3, (Tzp - Tc) * rdmx3p
    rhs = -0.5 * ((Uc * dedx1 + Uxp * dedx2) * 0.5 + (Vc * dedy3 + Vyp * dedy4) * 0.5 + (Wc * dedz5 + Wzp * dedz6) * 0.5)
    kPP1 = 0.5 * rdmx1 * (dx1 * Kxm + dx1m * Kc); kPP2 = 0.5 * rdmx1p * (dx1p * Kc + dx1 * Kxp)
    kPP3 = 0.5 * rdmx2 * (dx2 * Kym + dx2m * Kc); kPP4 = 0.5 * rdmx2p * (dx2p * Kc + dx2 * Kyp)
    kPP5 = 0.5 * rdmx3 * (dx3 * Kzm + dx3m * Kc); kPP6 = 0.5 * rdmx3p * (dx3p * Kc + dx3 * Kzp)
    dkPP1 = 0.5 * rdmx1 * (dx1 * dKxm + dx1m * dKc); dkPP2 = 0.5 * rdmx1p * (dx1p * dKc + dx1 * dKxp)
    dkPP3 = 0.5 * rdmx2 * (dx2 * dKym + dx2m * dKc); dkPP4 = 0.5 * rdmx2p * (dx2p * dKc + dx2 * dKyp)
    dkPP5 = 0.5 * rdmx3 * (dx3 * dKzm + dx3m * dKc); dkPP6 = 0.5 * rdmx3p * (dx3p * dKc + dx3 * dKzp)
    ve1 = (kPP2 * dedx2 - kPP1 * dedx1 - e2 * dkPP2 * dedx2 + e1 * dkPP1 * dedx1) * rdx1
    ve2 = (kPP4 * dedy4 - kPP3 * dedy3 - e4 * dkPP4 * dedy4 + e3 * dkPP3 * dedy3) * rdx2
    ve3 = (kPP6 * dedz6 - kPP5 * dedz5 - e6 * dkPP6 * dedz6 + e5 * dkPP5 * dedz5) * rdx3
    dv = (kPP2 * dedx2 - kPP1 * dedx1) * rdx1 + (kPP4 * dedy4 - kPP3 * dedy3) * rdx2 + (kPP6 * dedz6 - kPP5 * dedz5) * rdx3
    rhs = rhs + h * (ve1 + ve2 + ve3) - dh * Tc * dv
    ebc_up = -0.25 * Vyp * rdmx2p * Tup + h * rdx2 * kPP4 * rdmx2p * Tup + h * rdx2 * dkPP4 * dedy4 * Tup
    ebc_dn = 0.25 * Vc * rdmx2 * Tbt + h * rdx2 * kPP3 * rdmx2 * Tbt - h * rdx2 * dkPP3 * dedy3 * Tbt
    rhs = rhs + (1.0 - jem) * ebc_dn + (1.0 - jep) * ebc_up
    eACK = h * rdx3 * (kPP6 * rdmx3p + kPP5 * rdmx3 - dx3p * (0.5 * rdmx3p) * dkPP6 * dedz6 + dx3m * (0.5 * rdmx3) * dkPP5 * dedz5) + (-0.25 * Wzp * rdmx3p + 0.25 * Wc * rdmx3)
    eAPK = -h * rdx3 * (kPP6 * rdmx3p + dx3 * (0.5 * rdmx3p) * dkPP6 * dedz6) + 0.25 * Wzp * rdmx3p
    eAMK = -h * rdx3 * (kPP5 * rdmx3 - dx3 * (0.5 * rdmx3) * dkPP5 * dedz5) - 0.25 * Wc * rdmx3
    eACI = h * rdx1 * (kPP2 * rdmx1p + kPP1 * rdmx1 - dx1p * (0.5 * rdmx1p) * dkPP2 * dedx2 + dx1m * (0.5 * rdmx1) * dkPP1 * dedx1) + (0.25 * Uc * rdmx1 - 0.25 * Uxp * rdmx1p)
    eAPI = -h * rdx1 * (kPP2 * rdmx1p + dx1 * (0.5 * rdmx1p) * dkPP2 * dedx2) + 0.25 * Uxp * rdmx1p
    eAMI = -h * rdx1 * (kPP1 * rdmx1 - dx1 * (0.5 * rdmx1) * dkPP1 * dedx1) - 0.25 * Uc * rdmx1
    eACJ = h * rdx2 * (kPP4 * rdmx2p + kPP3 * rdmx2 - dx2p * (0.5 * rdmx2p) * dkPP4 * dedy4 * jep + dx2m * (0.5 * rdmx2) * dkPP3 * dedy3 * jem) + (0.25 * Vc * rdmx2 - 0.25 * Vyp * rdmx2p)
    eAPJ = (-h * rdx2 * (kPP4 * rdmx2p + dx2 * (0.5 * rdmx2p) * dkPP4 * dedy4) + 0.25 * Vyp * rdmx2p) * jep
    eAMJ = (-h * rdx2 * (kPP3 * rdmx2 - dx2 * (0.5 * rdmx2) * dkPP3 * dedy3) - 0.25 * Vc * rdmx2) * jem
    full = rhs - (eAPK * Tzp + eACK * Tc + eAMK * Tzm + eAPJ * Typ + eACJ * Tc + eAMJ * Tym
                  + eAPI * Txp + eACI * Tc + eAMI * Txm - dh * Tc * dv)
    # the reduced form of the kernel
    fx, fz = kPP2 * dedx2 - kPP1 * dedx1, kPP6 * dedz6 - kPP5 * dedz5
    red = 2 * h * (fx * rdx1 + fz * rdx3) - 0.5 * (Uc * dedx1 + Uxp * dedx2) - 0.5 * (Wc * dedz5 + Wzp * dedz6)
    if jem == 1.0 and jep == 1.0:
        red = red + 2 * h * (kPP4 * dedy4 - kPP3 * dedy3) * rdx2 - 0.5 * (Vc * dedy3 + Vyp * dedy4)
    else:
        red = (red - 0.25 * (Vc * dedy3 + Vyp * dedy4) + h * ve2 + (1 - jem) * ebc_dn + (1 - jep) * ebc_up
               - (eAPJ * Typ + eACJ * Tc + eAMJ * Tym))
    scale = sum(abs(t) for t in (eAPK * Tzp, eACK * Tc, eAPI * Txp, eACI * Tc, h * ve1, h * ve3, dh * Tc * dv, rhs))
    return full, red, scale


def test_reduced_thermal_rhs_matches_reference_expression():
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(500):
        metrics = rng.uniform(0.5, 2.0, 18)
        fields = rng.uniform(-1.0, 1.0, 7)
        K = rng.uniform(0.5, 2.0, 7)
        dK = rng.uniform(-1.0, 1.0, 7)
        vel = rng.uniform(-1.0, 1.0, 6)
        rest = rng.uniform(0.5, 2.0, 5)
        v = np.concatenate([metrics, fields, K, dK, vel, rest])
        for jem, jep in ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0)):
            full, red, scale = reference_rhs(v, jem, jep)
            worst = max(worst, abs(full - red) / scale)
    assert worst < 1e-13, worst
