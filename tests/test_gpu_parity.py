"""CUDA path vs the CPU oracle, through the C ABI (needs a B200).

Tolerances (FP64 plain form): every stage <= 1e-10 relative L2 against the
oracle from identical inputs (typically 1e-14..1e-11; the near-singular
lowest pressure modes set the upper end); the full 100-step run of the 64^3 constant-
property case <= 1e-10 relative L2 on u, v, w, T, p and on the Nusselt and
kinetic-energy series (the parity bar of the FP64 form); the
PaScaL_TDMA interface is bit-exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STAGE_TOL = 1e-10
RUN_TOL = 1e-10


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return d / nb if nb > 0 else d


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


def _pair(tcs, oracle_mod, **cfg):
    g = tcs.Solver(**cfg)
    o = oracle_mod.Oracle(**{k: v for k, v in g.config.items() if k not in ("device", "precision")})
    return g, o


def _check_fields(g, o, names, tol=STAGE_TOL, where=""):
    for n in names:
        a, b = g.get(n), o.get(n)
        assert np.all(np.isfinite(a)), f"{where}: {n} not finite"
        e = rel_l2(a, b)
        print(f"{where:28s} {n:7s} rel L2 {e:.2e}")
        assert e <= tol, f"{where}: {n} rel L2 {e:.3e} > {tol:.1e}"


CASES = [
    dict(n1m=32, n2m=24, n3m=16, property_set=0),
    dict(n1m=48, n2m=20, n3m=40, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, top_wall_mode=1),
    dict(n1m=30, n2m=17, n3m=24, property_set=2, Pr=7.0, Ra=1e5, dtStart=5e-4, uniform1=0, gamma1=1.2),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_stage_by_stage_parity(tcs, oracle_mod, case):
    g, o = _pair(tcs, oracle_mod, **CASES[case])
    _check_fields(g, o, ["T", "U", "V", "W", "P"], tol=0.0, where="initial")
    for step in range(3):
        w = f"step {step}"
        g.thermal_solver(); o.stage("thermal"); o.stage("ghost_T")
        _check_fields(g, o, ["T"], where=w + " thermal")
        g.momentum_coeffi(); o.stage("mom_coeffi")
        _check_fields(g, o, ["Mu", "invRho"], where=w + " mom_coeffi")
        g.momentum_solvedU(); o.stage("dU")
        _check_fields(g, o, ["dU"], where=w + " solvedU")
        g.momentum_solvedV(); o.stage("dV")
        _check_fields(g, o, ["dV"], where=w + " solvedV")
        g.momentum_solvedW(); o.stage("dW")
        _check_fields(g, o, ["dW"], where=w + " solvedW")
        g.momentum_blockLdV(); o.stage("blockLdV")
        _check_fields(g, o, ["dV"], where=w + " blockLdV")
        g.momentum_blockLdU(); o.stage("blockLdU")
        _check_fields(g, o, ["dU"], where=w + " blockLdU")
        g.momentum_pseudoupdateUVW(); g.pressure_RHS(); g.pressure_Poisson_FFT2()
        o.stage("pseudo"); o.stage("prhs"); o.stage("poisson")
        _check_fields(g, o, ["U", "V", "W", "dP"], where=w + " pseudo+poisson")
        g.pressure_Projection(); o.stage("project")
        _check_fields(g, o, ["U", "V", "W", "P", "dPhat", "dP0"], where=w + " projection")
        div = g.post_div(); cfl, dt = g.post_cfl(); o.stage("post")
        so = o.scalars()
        assert abs(div - so["maxDivU"]) <= 1e-12 + 1e-9 * abs(so["maxDivU"]), (div, so["maxDivU"])
        assert rel_l2(cfl, so["CFL"]) < 1e-12 and rel_l2(dt, so["dt"]) < 1e-12


def test_poisson_fft1_equals_fft2(tcs, oracle_mod):
    # mpi_pressure_Poisson_FFT1 (transpose scheme 1) and _FFT2 compute the same
    # arithmetic on one rank: from identical inputs the two entry points give
    # bit-identical dP, which matches the oracle's Poisson stage at the bar
    cfg = dict(n1m=30, n2m=17, n3m=24, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, top_wall_mode=1)
    a, o = _pair(tcs, oracle_mod, **cfg)
    b = tcs.Solver(**cfg)
    a.step(2); b.step(2); o.step(2)
    for s in (a, b):
        s.thermal_solver(); s.momentum_coeffi(); s.momentum_solvedU(); s.momentum_solvedV()
        s.momentum_solvedW(); s.momentum_blockLdV(); s.momentum_blockLdU()
        s.momentum_pseudoupdateUVW(); s.pressure_RHS()
    a.pressure_Poisson_FFT2()
    b.pressure_Poisson_FFT1()
    np.testing.assert_array_equal(b.get("dP"), a.get("dP"))
    for st in ("thermal", "ghost_T", "mom_coeffi", "dU", "dV", "dW", "blockLdV", "blockLdU", "pseudo", "prhs", "poisson"):
        o.stage(st)
    _check_fields(b, o, ["dP"], where="Poisson_FFT1")
    b.pressure_Projection(); a.pressure_Projection()
    np.testing.assert_array_equal(b.get("U"), a.get("U"))


def _run_compare(tcs, oracle_mod, steps, **cfg):
    g, o = _pair(tcs, oracle_mod, **cfg)
    g.step(steps)
    hd = o.step(steps)
    hg = g.history(0, steps)
    out = {n: rel_l2(g.get(n)[1:-1, 1:-1, 1:-1], o.get(n)[1:-1, 1:-1, 1:-1]) for n in ("U", "V", "W", "T", "P")}
    for col, n in ((4, "Nu_bot"), (5, "Nu_top"), (6, "KE")):
        out[n] = rel_l2(hg[:, col], hd[:, col])
    out["dt"] = rel_l2(hg[:, 0], hd[:, 0])
    return out, g, o


def test_long_lines_match_oracle(tcs, oracle_mod):
    # 512-row z and y lines (16 rows per lane; the z and y sweeps in their
    # one-block-per-SM form), water properties: whole steps against the oracle
    err, g, _ = _run_compare(tcs, oracle_mod, 3, n1m=16, n2m=512, n3m=512, gamma2=2.0, property_set=1, Pr=7.0,
                             Ra=1e7, DeltaT=10.0, dtStart=5e-5, fixed_dt=1, seed=2)
    print({k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= RUN_TOL, f"{k}: rel L2 {v:.3e}"
    g.set_tuning("long_lines", 4)
    assert g.tuning()["long_lines"] == 4


def test_one_line_per_thread_y_solver_matches_oracle(tcs, oracle_mod):
    # the FP64 y sweeps and the modal solves on the plain Thomas elimination
    # with one line per thread (y_solver 4); 150 lines along x leave the last
    # block of 128 lines part-filled, water properties
    cfg = dict(n1m=150, n2m=40, n3m=24, gamma2=1.5, property_set=1, Pr=7.0, Ra=1e7, DeltaT=10.0,
               dtStart=2e-4, fixed_dt=1, seed=5)
    g, o = _pair(tcs, oracle_mod, **cfg)
    g.set_tuning("y_solver", 4)
    g.step(12)
    hd = o.step(12)
    hg = g.history(0, 12)
    err = {n: rel_l2(g.get(n)[1:-1, 1:-1, 1:-1], o.get(n)[1:-1, 1:-1, 1:-1]) for n in ("U", "V", "W", "T", "P")}
    for col, n in ((4, "Nu_bot"), (5, "Nu_top"), (6, "KE")):
        err[n] = rel_l2(hg[:, col], hd[:, col])
    print({k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= RUN_TOL, f"{k}: rel L2 {v:.3e}"


def test_64cube_constant_properties_100_steps(tcs, oracle_mod):
    # The plain FP64 Rayleigh-Benard channel case: 64^3, Ra=1e5, Pr=0.71, dt=1e-3, seed 0.
    err, g, _ = _run_compare(tcs, oracle_mod, 100, n1m=64, n2m=64, n3m=64, Ra=1e5, Pr=0.71,
                             dtStart=1e-3, fixed_dt=1, seed=0, property_set=0)
    print({k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= RUN_TOL, f"{k}: rel L2 {v:.3e}"
    assert g.scalars()["step"] == 100


def test_water_fixed_dt_run(tcs, oracle_mod):
    # Temperature-dependent water properties (non-Oberbeck-Boussinesq terms, row-wise Mu/invRho,
    # sequential dPhat reads in the projection), top wall ghost as on a multi-rank y split.
    err, _, _ = _run_compare(tcs, oracle_mod, 40, n1m=32, n2m=32, n3m=32, property_set=1, Pr=7.0,
                             Ra=1e7, DeltaT=10.0, dtStart=2e-4, fixed_dt=1, seed=1, top_wall_mode=1)
    print({k: f"{v:.2e}" for k, v in err.items()})
    for k, v in err.items():
        assert v <= RUN_TOL, f"{k}: rel L2 {v:.3e}"


def test_adaptive_dt_run(tcs, oracle_mod):
    # The reference's CFL-adaptive dt (module_post.f90:222-226), started from a
    # shear flow U = W = 0.05 sin(pi y) so that the CFL limit sets a moderate dt.
    cfg = dict(n1m=32, n2m=32, n3m=32, property_set=0, Ra=1e5, Pr=0.71, dtStart=1e-3, fixed_dt=0,
               MaxCFL=0.3, seed=1, top_wall_mode=1)
    g, o = _pair(tcs, oracle_mod, **cfg)
    x2 = g.metric("x2")
    yc = 0.5 * (x2[:-1] + x2[1:])
    for n in ("U", "W"):
        a = g.get(n)
        a[:, 1:-1, :] = 0.05 * np.sin(np.pi * yc[1:])[None, :, None]
        g.set(n, a); o.set(n, a)
    g.step(20)
    hd = o.step(20)
    hg = g.history(0, 20)
    assert 1e-3 < hg[1, 0] < 1.0 and np.ptp(hg[1:, 0]) > 0    # dt really adapts
    errs = {n: rel_l2(g.get(n)[1:-1, 1:-1, 1:-1], o.get(n)[1:-1, 1:-1, 1:-1]) for n in ("U", "V", "W", "T", "P")}
    errs["dt"] = rel_l2(hg[:, 0], hd[:, 0])
    errs["KE"] = rel_l2(hg[:, 6], hd[:, 6])
    print({k: f"{v:.2e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v <= RUN_TOL, f"{k}: rel L2 {v:.3e}"


def test_snapshot_restore_replays_identically(tcs):
    g = tcs.Solver(n1m=24, n2m=16, n3m=20, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4)
    g.step(2)
    g.snapshot()
    g.step(3)
    a = {n: g.get(n) for n in ("T", "U", "V", "W", "P", "dPhat")}
    g.restore()
    g.step(3)
    for n, v in a.items():
        np.testing.assert_array_equal(g.get(n), v, err_msg=n)


def test_blowup_step_matches_oracle(tcs, oracle_mod):
    # Water properties with CFL-adaptive dt blow up once dt jumps to dtMax: both
    # implementations must stop at the same step with the BLOW UP status.
    cfg = dict(n1m=32, n2m=32, n3m=32, property_set=1, Pr=7.0, Ra=1e7, DeltaT=10.0, dtStart=2e-4,
               fixed_dt=0, MaxCFL=0.5, seed=1, top_wall_mode=1)
    g, o = _pair(tcs, oracle_mod, **cfg)
    with pytest.raises(FloatingPointError) as eo:
        o.step(40)
    ostep = int(str(eo.value).split()[-1])
    with pytest.raises(tcs.TcsError) as eg:
        g.step(40)
    assert eg.value.code == 4
    assert g.scalars()["blowup"] == ostep


def test_driver_sequence_matches_graph_step(tcs):
    cfg = dict(n1m=32, n2m=16, n3m=24, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4)
    a = tcs.Solver(**cfg)
    b = tcs.Solver(**cfg)
    for _ in range(4):
        a.driver_step()
    b.step(4)
    for n in ("T", "U", "V", "W", "P", "dPhat", "dP0"):
        np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
    np.testing.assert_array_equal(a.history(0, 4), b.history(0, 4))


def test_graph_and_eager_steps_identical(tcs):
    cfg = dict(n1m=24, n2m=16, n3m=20)
    a = tcs.Solver(**cfg)
    b = tcs.Solver(**cfg)
    b.use_graph(False)
    a.step(5); b.step(5)
    for n in ("T", "U", "V", "W", "P"):
        np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)


@pytest.mark.parametrize("n_row", [3, 7, 64, 255])
@pytest.mark.parametrize("cyclic", [False, True])
def test_tdma_interface_bitexact_host(tcs, oracle_mod, n_row, cyclic):
    rng = np.random.default_rng(n_row + 10 * cyclic)
    n_sys = 333
    ratio = 0.45 if n_row < 10 else 0.3        # weakly dominant: the one-rank closure is visible
    A = rng.uniform(-1, 1, (n_row, n_sys)) * ratio
    C = rng.uniform(-1, 1, (n_row, n_sys)) * ratio
    B = 1.0 + rng.uniform(0, 1, (n_row, n_sys))
    D = rng.uniform(-1, 1, (n_row, n_sys))
    ref = oracle_mod.tdma_many(A, B, C, D, cyclic=cyclic)
    plan = tcs.TdmaPlan(n_sys)
    Ag, Bg, Cg, Dg = A.copy(), B.copy(), C.copy(), D.copy()
    (plan.many_solve_cycle if cyclic else plan.many_solve)(Ag, Bg, Cg, Dg, n_sys, n_row)
    np.testing.assert_array_equal(Dg, ref)
    np.testing.assert_array_equal(Bg, B)


def test_tdma_interface_device_pointers(tcs, oracle_mod):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    n_sys, n_row = 4096, 96
    A = rng.uniform(-0.3, 0.3, (n_row, n_sys)); C = rng.uniform(-0.3, 0.3, (n_row, n_sys))
    B = 1.0 + rng.uniform(0, 1, (n_row, n_sys)); D = rng.uniform(-1, 1, (n_row, n_sys))
    ref = oracle_mod.tdma_many(A, B, C, D, cyclic=True)
    t = [torch.tensor(x, device="cuda") for x in (A, B, C, D)]
    plan = tcs.TdmaPlan(n_sys)
    plan.many_solve_cycle(*t, n_sys, n_row)
    np.testing.assert_array_equal(t[3].cpu().numpy(), ref)


def test_tdma_plan_rejects_multirank(tcs):
    with pytest.raises(tcs.TcsError):
        tcs.TdmaPlan(16, myrank=0, nprocs=2)


def test_blowup_is_reported_and_freezes_fields(tcs, oracle_mod):
    # Temperatures far outside the property polynomials' range make the
    # non-Boussinesq terms leave a divergence >= 1e-3 after projection
    # (main.f90:208-212); the fields then stay at the state of that step.
    cfg = dict(n1m=16, n2m=16, n3m=16, property_set=1, Pr=7.0, Ra=1e6, dtStart=1e-3)
    g, o = _pair(tcs, oracle_mod, **cfg)
    T = g.get("T")
    rng = np.random.default_rng(0)
    T[1:-1, 1:-1, 1:-1] = rng.uniform(-5.0, 5.0, T[1:-1, 1:-1, 1:-1].shape)
    g.set("T", T)
    o.set("T", T)
    with pytest.raises(FloatingPointError):
        o.step(5)
    with pytest.raises(tcs.TcsError) as ei:
        g.step(5)
    assert ei.value.code == 4
    s = g.scalars()
    assert s["blowup"] == 1.0 and s["step"] == 0
    T1 = g.get("T")
    with pytest.raises(tcs.TcsError):
        g.step(1)
    np.testing.assert_array_equal(g.get("T"), T1)


def test_unsupported_fft_size_is_rejected(tcs):
    with pytest.raises(tcs.TcsError) as ei:
        tcs.Solver(n1m=14, n2m=8, n3m=8)      # 14 = 2 * 7: no radix-7 FFT
    assert ei.value.code == 3
