"""The N-GPU replica logic of bench.py, on CPU: world size 2 with the gloo backend.

Each rank does independent work; the timed regions are bracketed by barriers and reduced with the
maximum over ranks, rates are whole-job totals, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from pigfem_b200 import replicas
    assert replicas.dist_env() == (world, rank, rank)
    assert replicas.init("gloo", rank, timeout_s=60)
    replicas.barrier()
    # rank r "took" 10 + r ms and 7 - r ms on two timed regions
    mx = replicas.max_over_ranks([10.0 + rank, 7.0 - rank])
    tot = replicas.sum_over_ranks([1.0 + rank])
    rate = replicas.aggregate_rate(1000.0, world, mx[0])
    replicas.finish()
    out.put((rank, mx, tot, rate))


def test_max_over_ranks_and_rates_gloo_world_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, tot, rate in res:
        assert mx == [11.0, 7.0]          # the slowest rank per region
        assert tot == [3.0]
        assert rate == pytest.approx(2 * 1000.0 / 11e-3)


def test_single_rank_is_local():
    sys.path.insert(0, ROOT)
    from pigfem_b200 import replicas
    assert replicas.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert replicas.aggregate_rate(100.0, 1, 10.0) == pytest.approx(1e4)


def test_reference_arm_prints_on_rank_0_only():
    """Under torchrun every rank runs bench.py --impl reference; ranks other than 0 exit 0 silently."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
