"""The golden fixtures of tests/golden (made by tests/golden/make_golden.py):
the dense-solve known answers for PaScaL_TDMA systems and the oracle's short
runs, which the oracle must reproduce bit for bit."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RUNS = ["rb16_water_oracle.npz", "rb16_glycerol_oracle.npz"]


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def residual(A, B, C, X, D, cyclic):
    R = B * X - D
    R[1:] += A[1:] * X[:-1]
    R[:-1] += C[:-1] * X[1:]
    if cyclic:
        R[0] += A[0] * X[-1]
        R[-1] += C[-1] * X[0]
    return np.max(np.abs(R))


@pytest.mark.parametrize("cyclic", [0, 1])
def test_dense_fixture_solves_its_systems(cyclic):
    z = load("tdma_dense.npz")
    A, B, C, D, X = (z[f"{n}{cyclic}"] for n in "ABCDX")
    assert residual(A, B, C, X, D, cyclic) <= 1e-14


@pytest.mark.parametrize("cyclic", [0, 1])
def test_oracle_tdma_matches_dense_fixture(oracle_mod, cyclic):
    z = load("tdma_dense.npz")
    A, B, C, D, X = (z[f"{n}{cyclic}"] for n in "ABCDX")
    got = oracle_mod.tdma_many(A, B, C, D, cyclic=bool(cyclic))
    assert np.max(np.abs(got - X)) <= 1e-13 * np.max(np.abs(X))


@pytest.mark.parametrize("name", RUNS)
def test_oracle_reproduces_run_fixture(oracle_mod, name):
    z = load(name)
    o = oracle_mod.Oracle(**json.loads(str(z["config"])))
    series = o.step(int(z["steps"]))
    np.testing.assert_array_equal(series, z["series"])
    for f in ("T", "U", "V", "W", "P"):
        np.testing.assert_array_equal(o.get(f), z[f], err_msg=f)
