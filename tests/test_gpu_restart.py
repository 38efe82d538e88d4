"""Restart files and planes straight from the device, and the PaScaL_TDMA
single-system and nonblocking entry points (needs a B200)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(n1m=32, n2m=24, n3m=20, property_set=1, Pr=7.0, Ra=1e6, dtStart=5e-4, seed=3)
I = (slice(1, -1),) * 3


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    P.load()
    return P


# field -> continue file: the names module_post.f90 writes and reads (:1336-1340, :1443-1447)
CONT = {"U": "cont_U.bin", "V": "cont_V.bin", "W": "cont_W.bin", "P": "cont_P.bin", "T": "cont_THETA.bin",
        "dPhat": "cont_dPhat.bin", "dP0": "cont_dP0.bin"}


def test_continue_files_have_the_reference_layout(tcs, tmp_path):
    g = tcs.Solver(**CFG)
    g.step(3)
    g.write_continue(str(tmp_path))
    n = CFG["n1m"] * CFG["n2m"] * CFG["n3m"]
    assert not (tmp_path / "cont_T.bin").exists()
    for f, name in CONT.items():
        a = np.fromfile(tmp_path / name, dtype=np.float64)
        assert a.size == n
        # (n1m, n2m, n3m) interior, i fastest: numpy (k, j, i) order
        np.testing.assert_array_equal(a.reshape(CFG["n3m"], CFG["n2m"], CFG["n1m"]), g.get(f)[I], err_msg=f)
    td = np.fromfile(tmp_path / "cont_time.bin", dtype=np.float64)
    s = g.scalars()
    assert td.tolist() == [s["time"], s["dt"]]


@pytest.mark.parametrize("precision", [0, 1])
def test_resume_from_continue_files_is_bit_continuous(tcs, tmp_path, precision):
    a = tcs.Solver(precision=precision, **CFG)
    a.step(3)
    a.write_continue(str(tmp_path))
    a.step(2)
    b = tcs.Solver(precision=precision, **CFG)
    assert b.read_continue(str(tmp_path))
    assert b.scalars()["time"] == pytest.approx(3 * CFG["dtStart"], rel=1e-12)
    b.step(2)
    for f in ("T", "U", "V", "W", "P", "dPhat", "dP0"):
        np.testing.assert_array_equal(b.get(f)[I], a.get(f)[I], err_msg=f)


def test_reads_files_written_by_the_reference_names(tcs, tmp_path):
    # continue files written field by field under the reference's names (as
    # mpi_Post_FileOut_Continue_Post_Reassembly_IO does), without the dPhat/dP0
    # extras: the reader takes them and reports the missing pressure history
    src = tcs.Solver(**CFG)
    src.step(2)
    for f in ("U", "V", "W", "P", "T"):
        np.ascontiguousarray(src.get(f)[I]).tofile(tmp_path / CONT[f])
    s = src.scalars()
    np.array([s["time"], s["dt"]]).tofile(tmp_path / "cont_time.bin")
    b = tcs.Solver(**CFG)
    assert not b.read_continue(str(tmp_path))
    for f in ("U", "V", "W", "P", "T"):
        np.testing.assert_array_equal(b.get(f)[I], src.get(f)[I], err_msg=f)
    assert b.scalars()["time"] == s["time"]
    # a temperature file under this library's earlier name is still read
    os.rename(tmp_path / "cont_THETA.bin", tmp_path / "cont_T.bin")
    c = tcs.Solver(**CFG)
    c.read_continue(str(tmp_path))
    np.testing.assert_array_equal(c.get("T")[I], src.get("T")[I])


def test_resume_without_pressure_history_is_reported(tcs, tmp_path):
    a = tcs.Solver(**CFG)
    a.step(2)
    a.write_continue(str(tmp_path))
    os.remove(tmp_path / "cont_dPhat.bin")
    b = tcs.Solver(**CFG)
    assert not b.read_continue(str(tmp_path))
    np.testing.assert_array_equal(b.get("U")[I], a.get("U")[I])


def test_planes_match_whole_fields(tcs):
    g = tcs.Solver(precision=1, **CFG)
    g.step(2)
    names = ("U", "V", "W", "P", "T")
    full = {f: g.get(f) for f in names}
    k = (CFG["n3m"] + 1 - 1) // 2          # the X-Y plane of module_post.f90:302
    xy = g.plane(3, k, names)
    xz = g.plane(2, 3, names)              # the X-Z plane at j = 3 (:334)
    yz = g.plane(1, 5, names)
    for q, f in enumerate(names):
        np.testing.assert_array_equal(xy[q], full[f][k, :, :])
        np.testing.assert_array_equal(xz[q], full[f][:, 3, :])
        np.testing.assert_array_equal(yz[q], full[f][:, :, 5])


@pytest.mark.parametrize("cyclic", [False, True])
def test_tdma_single_and_nonblocking_bitexact(tcs, oracle_mod, cyclic):
    rng = np.random.default_rng(11 + cyclic)
    n_row = 37
    A = rng.uniform(-0.4, 0.4, n_row); C = rng.uniform(-0.4, 0.4, n_row)
    B = 1.0 + rng.uniform(0, 1, n_row); D = rng.uniform(-1, 1, n_row)
    ref = oracle_mod.tdma_many(A[:, None].copy(), B[:, None].copy(), C[:, None].copy(), D[:, None].copy(), cyclic=cyclic)[:, 0]
    plan = tcs.TdmaPlanSingle()
    a, b, c, d = A.copy(), B.copy(), C.copy(), D.copy()
    (plan.single_solve_cycle if cyclic else plan.single_solve)(a, b, c, d, n_row)
    np.testing.assert_array_equal(d, ref)
    n_sys = 50
    AA = rng.uniform(-0.4, 0.4, (n_row, n_sys)); CC = rng.uniform(-0.4, 0.4, (n_row, n_sys))
    BB = 1.0 + rng.uniform(0, 1, (n_row, n_sys)); DD = rng.uniform(-1, 1, (n_row, n_sys))
    ref2 = oracle_mod.tdma_many(AA, BB, CC, DD, cyclic=cyclic)
    many = tcs.TdmaPlan(n_sys)
    x = [m.copy() for m in (AA, BB, CC, DD)]
    (many.many_solve_cycle_nonblocking if cyclic else many.many_solve_nonblocking)(*x, n_sys, n_row)
    np.testing.assert_array_equal(x[3], ref2)
