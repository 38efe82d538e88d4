"""Host-side checks that need no GPU: the C-ABI library loads and exports every
symbol include/tcs.h declares, argument validation happens before any CUDA
call, and the multi-process timing path of bench.py (replicas, max over ranks)
works over gloo with two ranks."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def tcs():
    import pascal_tcs_b200 as P
    from pascal_tcs_b200 import build
    build.build()
    P.load()
    return P


def test_library_exports_every_declared_symbol(tcs):
    hdr = open(os.path.join(ROOT, "include", "tcs.h")).read()
    declared = set(re.findall(r"\b(tcs_[a-zA-Z_0-9]+)\s*\(", hdr))
    L = tcs.load()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(tcs.EXPORTS)


def test_tuning_knobs_follow_the_header(tcs):
    # the Python binding addresses knobs by their index in include/tcs.h's
    # TCS_TUNE_* enum: the two lists must agree name for name and in order,
    # and every line of the committed tune cache must carry at most that many
    # knob columns (older lines may stop early; the library keeps the rest)
    hdr = open(os.path.join(ROOT, "include", "tcs.h")).read()
    body = re.search(r"enum\s*\{\s*(TCS_TUNE_TL_STRIDED[^}]*)\}", hdr).group(1)
    names = [n.strip().split("=")[0].strip() for n in body.split(",") if n.strip()]
    assert names[-1] == "TCS_TUNE_COUNT"
    assert [n[len("TCS_TUNE_"):].lower() for n in names[:-1]] == tcs.tcs.TUNING
    with open(os.path.join(ROOT, "pascal_tcs_b200", "tune_cache.txt")) as f:
        for line in f:
            v = line.split()
            if v:
                assert 4 + 7 <= len(v) <= 4 + len(tcs.tcs.TUNING), line
                assert all(int(x) > 0 for x in v[:3] + v[4:]) and v[3] in ("0", "1"), line


def test_kernel_names(tcs):
    names = tcs.kernel_names()
    assert len(names) == len(set(names)) and "thermal_z" in names and "projection" in names


def test_stage_timers_follow_the_reference_labels(tcs):
    # main.f90:55-72: the 18 timer labels, and every kernel of the time loop
    # under the timer of the routine whose work it does
    ref = ["Thermal coeff", "Thermal solve", "Momentum coeff", "Momentum solvedU", "Momentum solvedV",
           "Momentum solvedW", "Momentum blockLdV", "Momentum blockLdU", "Momentum updatePseudoUVW", "Pressure RHS",
           "Pressure PoissonSolve", "Pressure projection", "Update GhostCell", "Clean coeff", "Post div",
           "Post CFL", "Misc operation", "File write"]
    assert tcs.timer_names() == ["[Main] " + r for r in ref]
    m = tcs.timer_of_kernel()
    assert set(m) == set(tcs.kernel_names())
    want = {"thermal_z": "Thermal solve", "du_y": "Momentum solvedU", "dv_x": "Momentum solvedV",
            "dw_z": "Momentum solvedW", "momentum_coeffi": "Momentum coeff", "blockld_v": "Momentum blockLdV",
            "blockld_u": "Momentum blockLdU", "pseudo_update": "Momentum updatePseudoUVW", "prhs_fftx": "Pressure RHS",
            "fftz_fwd": "Pressure PoissonSolve", "modal_tdma": "Pressure PoissonSolve", "ifftx": "Pressure PoissonSolve",
            "projection": "Pressure projection", "post": "Post div", "tdma_api": None}
    for k, v in want.items():
        assert m[k] == (None if v is None else "[Main] " + v), k
    L = tcs.load()
    assert L.tcs_timer_of_kernel(-1) == -1 and L.tcs_timer_name(0) is None and L.tcs_timer_name(19) is None


@pytest.mark.parametrize("cfg,code", [(dict(n1m=2), 1), (dict(n1m=14), 3), (dict(n3m=22), 3)])
def test_create_rejects_bad_configuration_without_touching_the_gpu(tcs, cfg, code):
    with pytest.raises(tcs.TcsError) as ei:
        tcs.Solver(**cfg)
    assert ei.value.code == code


def test_tdma_plan_rejects_multirank_without_gpu(tcs):
    with pytest.raises(tcs.TcsError) as ei:
        tcs.TdmaPlan(8, myrank=1, nprocs=4)
    assert ei.value.code == 3


def _gloo_worker(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    import sys
    sys.path.insert(0, ROOT)
    import bench
    t = bench.dist_max(1.0 + rank, ws)         # per-rank replica time
    bench.dist_barrier(ws)
    q.put((rank, t))
    dist.destroy_process_group()


def test_two_rank_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.0, 1: 2.0}
    assert all(p.exitcode == 0 for p in ps)


def test_ensemble_cases_and_lpt_sharding():
    import bench
    cases = bench.ensemble_cases(48, 0)
    assert len(cases) == 48
    assert all(c[a] in (64, 96, 128, 160, 192) for c in cases for a in ("n1m", "n2m", "n3m"))
    assert all(1e5 <= c["Ra"] <= 1e7 for c in cases)
    assert {c["property_set"] for c in cases} <= {0, 1} and [c["seed"] for c in cases] == list(range(48))
    assert bench.ensemble_cases(48, 0) == cases                       # seeded
    cells = lambda c: c["n1m"] * c["n2m"] * c["n3m"]
    for ws in (1, 2, 3, 8):
        shards = [bench.lpt_shard(cases, ws, r) for r in range(ws)]
        assert sorted(c["seed"] for s in shards for c in s) == list(range(48))
        loads = [sum(cells(c) for c in s) for s in shards]
        assert max(loads) - min(loads) <= max(cells(c) for c in cases)    # LPT bound


def _lpt_rank(rank, ws, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    mine = bench.lpt_shard(bench.ensemble_cases(48, 1), ws, rank)
    import torch
    t = torch.tensor([float(sum(c["n1m"] * c["n2m"] * c["n3m"] for c in mine)), float(len(mine))])
    dist.all_reduce(t)
    out[rank] = (t[0].item(), t[1].item())
    dist.destroy_process_group()


def test_lpt_sharding_two_gloo_ranks_cover_all_cases():
    import multiprocessing as mp
    import bench
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = 29000 + os.getpid() % 1000
        ps = [ctx.Process(target=_lpt_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
        assert all(p.exitcode == 0 for p in ps)
        total = sum(c["n1m"] * c["n2m"] * c["n3m"] for c in bench.ensemble_cases(48, 1))
        assert out[0] == out[1] == (float(total), 48.0)


def test_tune_shape_parser():
    from pascal_tcs_b200 import tune
    assert tune.parse("256x128x64:1") == dict(n1m=256, n2m=128, n3m=64, precision=1)
    assert tune.parse("64x64x64") == dict(n1m=64, n2m=64, n3m=64, precision=0)


def test_reference_arm_restarts_before_blowup():
    # The water cases blow up in the reference algorithm after about 8 steps
    # from the seeded state: the reference arm restarts from that state every
    # RESET_EVERY steps (as the GPU arm does) and times only the steps.
    import bench

    class FakeOracle:
        made = 0

        def __init__(self):
            FakeOracle.made += 1
            self.n = 0

        def step(self, k):
            self.n += k
            if self.n > 8:
                raise FloatingPointError("blow up")

    el = bench.oracle_steps(FakeOracle, 20, 8, warmup=3)
    assert el >= 0.0
    assert FakeOracle.made == 1 + (3 + 20) // 8
    FakeOracle.made = 0
    bench.oracle_steps(FakeOracle, 5, 0)          # no reset period: one oracle
    assert FakeOracle.made == 1
