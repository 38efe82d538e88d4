"""The PaScaL_TDMA heat example (PaScaL_TDMA/examples) driven through the
oracle's PaScaL_TDMA solves: the whole example against its closed-form
answer, and its many-system and single-system drivers against each other."""
import numpy as np
import pytest

from heat_example import HeatExample, OraclePlan

DIMS = (16, 12, 10)
STEPS = 20


@pytest.fixture(scope="module")
def many_run(oracle_mod):
    h = HeatExample(*DIMS)
    for _ in range(STEPS):
        h.step_many(lambda n_sys: OraclePlan(oracle_mod, n_sys))
    return h


def test_closed_form_factor_is_a_real_decay():
    h = HeatExample(*DIMS)
    g = h.mode_factor()
    assert 0.5 < g < 1.0, g


def test_initial_field_and_walls():
    h = HeatExample(*DIMS)
    np.testing.assert_array_equal(h.theta[:, 0, :], h.theta_hot)
    np.testing.assert_array_equal(h.theta[:, h.NY, :], h.theta_cold)
    # periodic ghosts after the initial ghost update (main.f90 of the example)
    np.testing.assert_array_equal(h.theta[:, :, 0], h.theta[:, :, h.NX - 1])
    np.testing.assert_array_equal(h.theta[0], h.theta[h.NZ - 1])
    np.testing.assert_allclose(h.interior(), h.expected(0), rtol=0, atol=1e-15)


def test_many_driver_follows_the_closed_form(many_run):
    h = many_run
    got, want = h.interior(), h.expected(STEPS)
    amp = h.mode_factor() ** STEPS
    err = np.max(np.abs(got - want))
    assert err <= 1e-14, (err, amp)
    # the mode did decay, so the check is not trivially met by the linear profile
    assert np.max(np.abs(got - h.expected(0))) > 0.5


def test_single_driver_equals_many_driver(oracle_mod, many_run):
    s = HeatExample(*DIMS)
    for _ in range(STEPS):
        s.step_single(lambda: OraclePlan(oracle_mod))
    np.testing.assert_array_equal(s.theta, many_run.theta)
