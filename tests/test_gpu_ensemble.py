"""Ensembles (tcs_ensemble_*): independent cases of uneven sizes, properties
and precisions advanced together by one CUDA graph per step must give, case
by case, exactly what each case gives when stepped alone (needs a B200)."""
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


def test_ensemble_matches_cases_stepped_alone(tcs):
    alone = [tcs.Solver(**c) for c in CASES]
    grouped = [tcs.Solver(**c) for c in CASES]
    for s in alone:
        s.step(5)
    ens = tcs.Ensemble(grouped)
    assert len(ens) == len(CASES)
    assert ens.step(3) == 0
    assert ens.step(2) == 0          # the second graph state, then a cached one
    for a, b in zip(alone, grouped):
        for n in ("T", "U", "V", "W", "P", "dPhat", "dP0"):
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
        np.testing.assert_array_equal(a.history(0, 5), b.history(0, 5))
        assert b.scalars()["step"] == 5


def test_ensemble_reports_blown_cases(tcs):
    good = tcs.Solver(**CASES[0])
    bad = tcs.Solver(n1m=16, n2m=16, n3m=16, property_set=1, Pr=7.0, Ra=1e6, dtStart=1e-3)
    T = bad.get("T")
    T[1:-1, 1:-1, 1:-1] = np.random.default_rng(0).uniform(-5.0, 5.0, T[1:-1, 1:-1, 1:-1].shape)
    bad.set("T", T)
    ens = tcs.Ensemble([good, bad])
    assert ens.step(3) == 1
    assert good.scalars()["step"] == 3 and good.scalars()["blowup"] == 0
    assert bad.scalars()["blowup"] == 1


def test_ensemble_rejects_repeated_case(tcs):
    s = tcs.Solver(**CASES[0])
    with pytest.raises(tcs.TcsError):
        tcs.Ensemble([s, s])
