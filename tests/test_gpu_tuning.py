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
                                        ("tl_modal", 1), ("fft_lines_x", 1), ("fft_lines_z", 8)])
def test_every_knob_setting_gives_the_same_step(tcs, knob, value):
    a, b = tcs.Solver(**CFG), tcs.Solver(**CFG)
    b.set_tuning(knob, value)
    assert b.tuning()[knob] == value
    a.step(3); b.step(3)
    for n in ("T", "U", "V", "W", "P"):
        x, y = a.get(n), b.get(n)
        assert np.linalg.norm(x - y) <= 1e-12 * np.linalg.norm(x), n
