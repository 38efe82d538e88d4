"""The CUDA path against the golden fixtures of tests/golden (needs a B200):
the PaScaL_TDMA interface against dense-solve known answers, and the time
step against the oracle's stored short runs at the parity bar of the FP64
form (1e-10 relative L2 on the fields and the Nusselt, kinetic-energy and dt
series)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RUNS = ["rb16_water_oracle.npz", "rb16_glycerol_oracle.npz"]
TOL = 1e-10
I = (slice(1, -1),) * 3


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


@pytest.mark.parametrize("cyclic", [0, 1])
def test_tdma_interface_matches_dense_fixture(tcs, cyclic):
    z = load("tdma_dense.npz")
    A, B, C, D, X = (z[f"{n}{cyclic}"].copy() for n in "ABCDX")
    n_row, n_sys = D.shape
    plan = tcs.TdmaPlan(n_sys)
    (plan.many_solve_cycle if cyclic else plan.many_solve)(A, B, C, D, n_sys, n_row)
    plan.destroy()
    assert np.max(np.abs(D - X)) <= 1e-13 * np.max(np.abs(X))


@pytest.mark.parametrize("name", RUNS)
def test_time_step_matches_run_fixture(tcs, name):
    z = load(name)
    s = tcs.Solver(**json.loads(str(z["config"])))
    steps = int(z["steps"])
    assert s.step(steps) == steps
    h = s.history(0, steps)
    want = z["series"]
    for col, n in ((0, "dt"), (4, "Nu_bot"), (5, "Nu_top"), (6, "KE")):
        assert rel_l2(h[:, col], want[:, col]) <= TOL, n
    assert np.all(np.abs(h[:, 2] - want[:, 2]) <= 1e-12 + 1e-9 * np.abs(want[:, 2])), (h[:, 2], want[:, 2])
    for f in ("T", "U", "V", "W", "P"):
        e = rel_l2(s.get(f)[I], z[f][I])
        assert e <= TOL, (f, e)
    s.close()
