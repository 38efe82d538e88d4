"""The allocation-free PaScaL_TDMA entry point (tcs_tdma_many_solve_noalloc).

It serves callers that may not allocate device memory when they solve; it
stages host arrays through a fixed device array compiled into libtcs.  This
file is collected last so that a run stopping at the first failure has run
every other test first.  The check: through the C ABI, two calls in a row
(different sizes and both closures, so the second call finds the first call's
data still in the shared array) give exactly what the plan-based entry point
gives -- the tridiagonal interface is bit-exact in every other test too.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(rng, n_sys, n_row):
    A = rng.uniform(-0.4, 0.4, (n_row, n_sys))
    C = rng.uniform(-0.4, 0.4, (n_row, n_sys))
    B = 1.0 + rng.uniform(0.0, 1.0, (n_row, n_sys))
    D = rng.uniform(-1.0, 1.0, (n_row, n_sys))
    return A, B, C, D


def test_noalloc_matches_plan_entry_on_two_calls():
    import pascal_tcs_b200 as P
    for call, (n_sys, n_row, cyclic) in enumerate(((700, 91, False), (313, 64, True))):
        rng = np.random.default_rng(11 + call)
        A, B, C, D = _systems(rng, n_sys, n_row)
        ref = [x.copy() for x in (A, B, C, D)]
        plan = P.TdmaPlan(n_sys)
        (plan.many_solve_cycle if cyclic else plan.many_solve)(*ref, n_sys, n_row)
        plan.destroy()
        got = [x.copy() for x in (A, B, C, D)]
        P.tdma_many_solve_noalloc(*got, n_sys, n_row, cyclic=cyclic)
        for name, g, r in zip("ABCD", got, ref):
            np.testing.assert_array_equal(g, r, err_msg=f"call {call}: {name}")


def test_noalloc_rejects_oversize_batch():
    import pascal_tcs_b200 as P
    n_row = 8
    n_sys = P.TDMA_NOALLOC_MAX_ELEMS // n_row + 1
    z = np.zeros((n_row, n_sys))
    with pytest.raises(P.TcsError) as ei:
        P.tdma_many_solve_noalloc(z, z + 1.0, z.copy(), z.copy(), n_sys, n_row)
    assert ei.value.code == 3
