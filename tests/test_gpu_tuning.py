"""The autotuner (tcs_autotune) and the launch-shape knobs it sets (needs a B200):
tuning leaves the case's state as it was, every knob setting gives the same
results to rounding, and a tuned shape is served from the cache."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(n1m=48, n2m=32, n3m=40, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, seed=7)


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


def test_autotune_keeps_state_and_caches(tcs, tmp_path):
    cache = str(tmp_path / "tune.txt")
    g = tcs.Solver(**CFG)
    g.step(2)
    before = {n: g.get(n) for n in ("T", "U", "V", "W", "P", "dPhat", "dP0")}
    step0 = g.scalars()["step"]
    knobs, hit = g.autotune(trial_steps=2, cache_path=cache)
    assert not hit
    assert set(knobs) == set(tcs.tcs.TUNING)
    assert g.scalars()["step"] == step0
    for n, v in before.items():
        np.testing.assert_array_equal(g.get(n), v, err_msg=n)
    h = tcs.Solver(**CFG)
    knobs2, hit2 = h.autotune(cache_path=cache)
    assert hit2 and knobs2 == knobs
    with open(cache) as f:
        assert len(f.read().split()) == 4 + len(knobs)


@pytest.mark.parametrize("knob,value", [("lanes", 8), ("lanes", 16), ("tl_strided", 2), ("tl_contig", 16),
                                        ("tl_modal", 1), ("fft_lines_x", 1), ("fft_lines_z", 8),
                                        ("long_lines", 1), ("long_lines", 4), ("y_solver", 2), ("y_solver", 4),
                                        ("ifft_lines_x", 8), ("mixed_rows", 4)])
def test_every_knob_setting_gives_the_same_step(tcs, knob, value):
    a, b = tcs.Solver(**CFG), tcs.Solver(**CFG)
    b.set_tuning(knob, value)
    assert b.tuning()[knob] == value
    a.step(3); b.step(3)
    for n in ("T", "U", "V", "W", "P"):
        x, y = a.get(n), b.get(n)
        assert np.linalg.norm(x - y) <= 1e-12 * np.linalg.norm(x), n


@pytest.mark.parametrize("precision", [0, 1])
def test_long_line_forms_are_bit_identical(tcs, precision):
    # 512-row z and y lines: the one-block-per-SM form (z sweeps by default, y
    # sweeps too with long_lines = 4) runs the same arithmetic per line as the
    # usual form, so every setting gives the same bits
    cfg = dict(n1m=16, n2m=512, n3m=512, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, seed=4, precision=precision)
    runs = []
    for v in (1, 2, 4):
        g = tcs.Solver(**cfg)
        g.set_tuning("long_lines", v)
        g.step(2)
        runs.append({n: g.get(n) for n in ("T", "U", "V", "W", "P")})
        g.close()
    for r in runs[1:]:
        for n, x in runs[0].items():
            np.testing.assert_array_equal(r[n], x, err_msg=n)


@pytest.mark.parametrize("knob,value", [("y_solver", 2), ("y_solver", 4), ("mixed_rows", 2), ("mixed_rows", 4),
                                        ("mixed_rows", 8)])
def test_solver_knobs_in_the_mixed_form(tcs, knob, value):
    # y_solver 2: the y sweeps' FP32-built rows eliminated in FP64 with one line
    # per thread instead of the FP32 elimination and its refinement; 4: the
    # modal pressure solves (FP64 rows in both forms) too.  mixed_rows 2 / 4:
    # the x (and z) sweeps' FP32-built rows eliminated in FP64 on the
    # partitioned solver.  Both runs store their fields in FP32 and each lies
    # within a few 1e-6 of the FP64 form, so they agree to the mixed form's 1e-5
    # bar (measured: V 2.3e-6 apart after 3 steps, V being the smallest
    # component here).
    cfg = dict(CFG, precision=1)
    a, b = tcs.Solver(**cfg), tcs.Solver(**cfg)
    b.set_tuning(knob, value)
    assert b.tuning()[knob] == value
    a.step(3); b.step(3)
    for n in ("T", "U", "V", "W", "P"):
        x, y = a.get(n), b.get(n)
        assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(x), n
    with pytest.raises(tcs.TcsError) as ei:
        b.set_tuning(knob, 16)
    assert ei.value.code == 1
    b.set_tuning(knob, 1)                           # the partitioned FP32 eliminations again (frees any scratch)
    b.step(1); a.step(1)
    assert np.linalg.norm(a.get("P") - b.get("P")) <= 1e-5 * np.linalg.norm(a.get("P"))


def test_tma_staged_dwz_gives_the_same_bits(tcs):
    # solvedW's z sweep with its inputs staged by TMA (z_staging 2) runs the same
    # arithmetic on the same values as the global-load form: the same bits, over
    # whole water steps, on a grid whose N3 is two passes of 64 planes and whose
    # last x block is part-filled (N1 = 36)
    cfg = dict(n1m=36, n2m=24, n3m=128, property_set=1, Pr=7.0, Ra=1e6, DeltaT=10.0, dtStart=5e-4, seed=9)
    a, b = tcs.Solver(**cfg), tcs.Solver(**cfg)
    b.set_tuning("z_staging", 2)
    assert b.tuning()["z_staging"] == 2
    a.step(3); b.step(3)
    for n in ("T", "U", "V", "W", "P", "dW"):
        np.testing.assert_array_equal(b.get(n), a.get(n), err_msg=n)
    # refused where it cannot run: the FP32 form, N3 not a multiple of 64, odd N1
    for bad in (dict(cfg, precision=1), dict(cfg, n3m=96), dict(cfg, n1m=45)):
        g = tcs.Solver(**bad)
        with pytest.raises(tcs.TcsError) as ei:
            g.set_tuning("z_staging", 2)
        assert ei.value.code == 1
        g.close()
