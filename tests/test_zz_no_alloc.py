"""The allocation-free PaScaL_TDMA entry point (tcs_tdma_many_solve_noalloc).

It serves callers that may not allocate device memory when they solve: a host
application that owns the device memory budget, a path where a cudaMalloc or
cudaFree would synchronise the device, or a Fortran driver that hands over host
arrays and creates no plans.  It stages the arrays through a fixed device
array compiled into libtcs.  This file is collected last, so that a run that
stops at the first failure has run every other test first.

The checks, all through the C ABI:
  * two calls in a row (different sizes and both closures, so the second call
    finds the first call's data still in the shared array) give exactly what
    the plan-based entry point gives;
  * two calls in a row on the dense-solve golden systems match the dense
    solutions to 1e-13, the bar of the plan-based entry point's golden test;
  * in a fresh process, calls before and after a cudaDeviceReset (a new device
    context, in which the array's address is looked up again) both match;
  * an oversized batch is refused with TCS_ERR_UNSUPPORTED.
"""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "tdma_dense.npz")


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


def test_noalloc_matches_dense_golden_on_two_calls():
    import pascal_tcs_b200 as P
    z = np.load(GOLDEN)
    for cyclic in (0, 1):
        A, B, C, D, X = (z[f"{n}{cyclic}"].copy() for n in "ABCDX")
        n_row, n_sys = D.shape
        P.tdma_many_solve_noalloc(A, B, C, D, n_sys, n_row, cyclic=bool(cyclic))
        assert np.max(np.abs(D - X)) <= 1e-13 * np.max(np.abs(X)), (cyclic, np.max(np.abs(D - X)))


_AFTER_RESET = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    import pascal_tcs_b200 as P
    z = np.load({golden!r})

    def solve(cyclic):
        A, B, C, D, X = (z[n + str(cyclic)].copy() for n in "ABCDX")
        P.tdma_many_solve_noalloc(A, B, C, D, D.shape[1], D.shape[0], cyclic=bool(cyclic))
        return float(np.max(np.abs(D - X)) / np.max(np.abs(X)))

    e0 = solve(0)
    # the CUDA runtime libtcs runs on: reset the device (a new primary context)
    cudart = [l.split()[-1] for l in open("/proc/self/maps") if "libcudart" in l][0]
    rt = ctypes.CDLL(cudart)
    assert rt.cudaDeviceReset() == 0
    e1 = solve(1)
    e2 = solve(0)
    print(e0, e1, e2)
    sys.exit(0 if max(e0, e1, e2) <= 1e-13 else 1)
""")


def test_noalloc_after_device_reset_in_fresh_process():
    code = _AFTER_RESET.format(root=ROOT, golden=GOLDEN)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


def test_noalloc_rejects_oversize_batch():
    import pascal_tcs_b200 as P
    n_row = 8
    n_sys = P.TDMA_NOALLOC_MAX_ELEMS // n_row + 1
    z = np.zeros((n_row, n_sys))
    with pytest.raises(P.TcsError) as ei:
        P.tdma_many_solve_noalloc(z, z + 1.0, z.copy(), z.copy(), n_sys, n_row)
    assert ei.value.code == 3
