"""Ensembles (tcs_ensemble_*): independent cases of uneven sizes, properties
and precisions advanced together by one CUDA graph per step must give, case
by case, exactly what each case gives when stepped alone, in both forms (the
batched one: one multi-case launch per line sweep; one branch per case) and
in the auto mode that measures both (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    dict(n1m=32, n2m=24, n3m=20, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, seed=3),
    dict(n1m=48, n2m=16, n3m=30, property_set=0, Pr=0.71, Ra=1e5, dtStart=1e-3, seed=4, precision=1),
    dict(n1m=24, n2m=40, n3m=36, property_set=2, Pr=7.0, Ra=2e5, dtStart=5e-4, seed=5),
    dict(n1m=40, n2m=32, n3m=24, property_set=1, Pr=7.0, Ra=1e7, dtStart=2e-4, seed=6, precision=1),
]


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


@pytest.mark.parametrize("batched", [True, False, None])
def test_ensemble_matches_cases_stepped_alone(tcs, batched):
    # None (auto) runs both forms within these 5 steps
    alone = [tcs.Solver(**c) for c in CASES]
    grouped = [tcs.Solver(**c) for c in CASES]
    for s in alone:
        s.step(5)
    ens = tcs.Ensemble(grouped, batched=batched)
    assert len(ens) == len(CASES)
    assert ens.step(3) == 0
    assert ens.step(2) == 0          # the second graph state, then a cached one
    for a, b in zip(alone, grouped):
        for n in ("T", "U", "V", "W", "P", "dPhat", "dP0"):
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
        np.testing.assert_array_equal(a.history(0, 5), b.history(0, 5))
        assert b.scalars()["step"] == 5


@pytest.mark.parametrize("batched", [True, False])
def test_ensemble_reports_blown_cases(tcs, batched):
    good = tcs.Solver(**CASES[0])
    bad = tcs.Solver(n1m=16, n2m=16, n3m=16, property_set=1, Pr=7.0, Ra=1e6, dtStart=1e-3)
    T = bad.get("T")
    T[1:-1, 1:-1, 1:-1] = np.random.default_rng(0).uniform(-5.0, 5.0, T[1:-1, 1:-1, 1:-1].shape)
    bad.set("T", T)
    ens = tcs.Ensemble([good, bad], batched=batched)
    assert ens.step(3) == 1
    assert good.scalars()["step"] == 3 and good.scalars()["blowup"] == 0
    assert bad.scalars()["blowup"] == 1


def test_ensemble_rejects_repeated_case(tcs):
    s = tcs.Solver(**CASES[0])
    with pytest.raises(tcs.TcsError):
        tcs.Ensemble([s, s])


def test_batched_ensemble_more_cases_than_one_launch_holds(tcs):
    # 24 FP64 cases: more than one multi-case launch's parameter block holds,
    # so every sweep is split over several launches; two sizes, so the items
    # of the longer lines come first.
    cfgs = [dict(n1m=16, n2m=12 + 4 * (i % 2), n3m=(10, 12, 16)[i % 3], property_set=1, Pr=7.0, Ra=1e6,
                 dtStart=5e-4, seed=10 + i) for i in range(24)]
    alone = [tcs.Solver(**c) for c in cfgs]
    grouped = [tcs.Solver(**c) for c in cfgs]
    for s in alone:
        s.step(3)
    ens = tcs.Ensemble(grouped)
    assert ens.step(3) == 0
    for a, b in zip(alone, grouped):
        for n in ("T", "U", "V", "W", "P"):
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)


def test_ensemble_switch_between_forms(tcs):
    alone = [tcs.Solver(**c) for c in CASES[:2]]
    grouped = [tcs.Solver(**c) for c in CASES[:2]]
    for s in alone:
        s.step(4)
    ens = tcs.Ensemble(grouped, batched=True)
    ens.step(1)
    assert ens.form()[0] == 1
    ens.set_batched(False)
    ens.step(2)
    assert ens.form()[0] == 0
    ens.set_batched(True)
    ens.step(1)
    for a, b in zip(alone, grouped):
        for n in ("T", "U", "W", "P", "dPhat"):
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)


def test_ensemble_auto_picks_a_form(tcs):
    alone = [tcs.Solver(**c) for c in CASES]
    grouped = [tcs.Solver(**c) for c in CASES]
    for s in alone:
        s.step(10)
    ens = tcs.Ensemble(grouped)
    ens.step(7)
    assert ens.form()[0] == -1                       # still measuring
    ens.step(3)
    form, ms_br, ms_bat = ens.form()
    assert form in (0, 1) and ms_br > 0 and ms_bat > 0
    assert form == (1 if ms_bat < ms_br else 0)
    for a, b in zip(alone, grouped):
        for n in ("T", "U", "V", "W", "P"):
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
