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


def test_kernel_names(tcs):
    names = tcs.kernel_names()
    assert len(names) == len(set(names)) and "thermal_z" in names and "projection" in names


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
