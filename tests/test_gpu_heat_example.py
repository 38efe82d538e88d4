"""The PaScaL_TDMA heat example (PaScaL_TDMA/examples) driven through the
library's PaScaL_TDMA entry points from host arrays, as the example's Fortran
driver calls them: a plan created and destroyed around every sweep, one plane
of lines (or one line) per call.  It must equal the same driver on the oracle
bit for bit, and follow the example's closed-form answer (needs a B200)."""
import numpy as np
import pytest

from heat_example import HeatExample, OraclePlan

pytestmark = pytest.mark.gpu

DIMS = (16, 12, 10)
STEPS = 12


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


@pytest.fixture(scope="module")
def oracle_run(oracle_mod):
    h = HeatExample(*DIMS)
    for _ in range(STEPS):
        h.step_many(lambda n_sys: OraclePlan(oracle_mod, n_sys))
    return h


@pytest.mark.parametrize("nonblocking", [False, True])
def test_many_plan_example_matches_oracle_and_closed_form(tcs, oracle_run, nonblocking):
    h = HeatExample(*DIMS)
    for _ in range(STEPS):
        h.step_many(lambda n_sys: tcs.TdmaPlan(n_sys), nonblocking=nonblocking)
    np.testing.assert_array_equal(h.theta, oracle_run.theta)
    assert np.max(np.abs(h.interior() - h.expected(STEPS))) <= 1e-14


def test_single_plan_example_matches_oracle(tcs, oracle_run):
    h = HeatExample(*DIMS)
    for _ in range(STEPS):
        h.step_single(lambda: tcs.TdmaPlanSingle())
    np.testing.assert_array_equal(h.theta, oracle_run.theta)
