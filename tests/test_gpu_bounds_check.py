"""The bounds-check build (libtcs_bc.so, compiled with -DTCS_BOUNDS_CHECK):
every field, 2-D table, spectrum and shared-memory row index the kernels form
is checked on the device; an out-of-range index is counted and its access
redirected to a valid cell, never made.  It stands in for a memory checker
(the reference's own debug builds use the compiler's array checks,
Makefile.inc:6-11).  The test runs that build in a fresh process over uneven
sizes, both precisions, stretched and uniform grids, long lines, every
launch-shape knob family, the per-routine driver sequence, an ensemble in
both forms and a 26-case batched ensemble whose sweeps split over two
multi-case launches, the restart files and planes, and the PaScaL_TDMA interface, and
requires zero recorded violations (needs a B200)."""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_BC = os.path.join(ROOT, "pascal_tcs_b200", "libtcs_bc.so")

SCRIPT = textwrap.dedent("""
    import sys, tempfile
    import numpy as np
    sys.path.insert(0, {root!r})
    import pascal_tcs_b200 as P
    assert P.bounds_checked(), "not the bounds-check build"
    counts = {{}}
    cases = [
        dict(n1m=16, n2m=12, n3m=10, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, seed=5),
        dict(n1m=30, n2m=17, n3m=24, property_set=2, Pr=7.0, Ra=1e5, dtStart=5e-4, uniform1=0, gamma1=1.2,
             top_wall_mode=1),
        dict(n1m=48, n2m=20, n3m=40, property_set=0),
        dict(n1m=16, n2m=512, n3m=512, gamma2=2.0, property_set=1, Pr=7.0, Ra=1e7, dtStart=5e-5, seed=2),
    ]
    for ci, cfg in enumerate(cases):
        for prec in (0, 1):
            g = P.Solver(precision=prec, **cfg)
            g.step(2)
            g.driver_step()
            with tempfile.TemporaryDirectory() as d:
                g.write_continue(d)
                g.read_continue(d)
            g.plane(1, 3); g.plane(2, 1); g.plane(3, cfg["n3m"])
            counts[f"case{{ci}} prec{{prec}}"] = g.bounds_violations()
            g.close()
    for knob, v in (("lanes", 4), ("tl_strided", 2), ("tl_contig", 1), ("tl_modal", 1), ("fft_lines_x", 1),
                    ("fft_lines_z", 8), ("long_lines", 4), ("y_solver", 4), ("mixed_rows", 4), ("ifft_lines_x", 8)):
        for prec in ((0, 1) if knob in ("y_solver", "mixed_rows") else (0,)):
            g = P.Solver(n1m=150 if knob == "y_solver" else 48, n2m=32, n3m=40, property_set=1, Pr=7.0, Ra=1e6,
                         dtStart=5e-4, precision=prec)
            g.set_tuning(knob, v)
            g.step(2)
            counts[f"{{knob}}={{v}} prec{{prec}}"] = g.bounds_violations()
            g.close()
    ens = [P.Solver(n1m=n1, n2m=n2, n3m=n3, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, precision=prec)
           for (n1, n2, n3, prec) in ((16, 24, 20, 0), (32, 16, 12, 0), (24, 20, 16, 1), (20, 12, 30, 1))]
    e = P.Ensemble(ens)
    for form in (1, 0):
        e.set_batched(form)
        e.step(2)
    for k, s in enumerate(ens):
        counts[f"ensemble case {{k}}"] = s.bounds_violations()
    # 24 uneven cases per precision: more than one multi-case launch's parameter
    # block holds (21 FP64 or 24 FP32 problems), so each batched sweep is split
    g = P.Solver(n1m=36, n2m=20, n3m=64, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4)
    g.set_tuning("z_staging", 2)
    g.step(2)
    counts["z_staging=2"] = g.bounds_violations()
    g.close()
    rng = np.random.default_rng(3)
    for prec in (0, 1):
        big = [P.Solver(n1m=int(rng.choice([16, 20, 24])), n2m=int(rng.choice([12, 16, 24])),
                        n3m=int(rng.choice([16, 20, 30])), property_set=int(k % 2), Pr=7.0, Ra=1e6, dtStart=5e-4,
                        seed=k, precision=prec) for k in range(26)]
        e2 = P.Ensemble(big)
        e2.set_batched(1)
        e2.step(3)
        for k, s in enumerate(big):
            counts[f"ensemble26 prec{{prec}} case {{k}}"] = s.bounds_violations()
        e2.close()
        for s in big:
            s.close()
    rng = np.random.default_rng(1)
    for cyclic in (False, True):
        A = rng.uniform(-0.3, 0.3, (64, 500)); C = rng.uniform(-0.3, 0.3, (64, 500))
        B = 1.0 + rng.uniform(0, 1, (64, 500)); D = rng.uniform(-1, 1, (64, 500))
        plan = P.TdmaPlan(500)
        (plan.many_solve_cycle if cyclic else plan.many_solve)(A, B, C, D, 500, 64)
        plan.destroy()
    bad = {{k: v for k, v in counts.items() if v}}
    print(counts)
    sys.exit(1 if bad else 0)
""")


def test_bounds_check_build_records_no_violation():
    if not os.path.exists(LIB_BC):
        from pascal_tcs_b200 import build
        build.build(bounds_check=True)
    env = dict(os.environ, TCS_LIBRARY=LIB_BC)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], capture_output=True, text=True, env=env,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-4000:]
