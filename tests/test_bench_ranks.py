"""The multi-rank logic of bench.py (replicas: no data-path collective, the
timed region is the max over ranks) with two gloo ranks on the CPU."""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    import bench
    env = bench.dist_env()
    t = [1.5, 2.5, 0.5][rank]
    m = bench.max_over_ranks(t, ws)
    bench.rank_barrier(ws)
    q.put((rank, env, m, bench.replica_throughput(ws, 100.0, m)))
    dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_ranks_time_the_slowest_and_sum_the_work(ws):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = max([1.5, 2.5, 0.5][:ws])
    for rank, env, m, thr in out:
        assert env == (ws, rank, rank)
        assert m == slowest
        assert thr == pytest.approx(ws * 100.0 / slowest)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup, gpus = 2, 3, 2

    assert bench.run_reference_arm(A()) == 0
    assert capsys.readouterr().out == ""


def test_shape_option_sets_the_named_launch_shapes():
    """bench --shape: every key of a tuner result it names becomes one
    pd_set_option call with the matching option; other keys are ignored."""
    sys.path.insert(0, ROOT)
    import bench
    import pdmtel_b200 as P

    class Ctx:
        def __init__(self):
            self.calls = []

        def set_option(self, opt, v):
            self.calls.append((opt, v))

    c = Ctx()
    out = bench.apply_shape(c, {"tile": 261, "gather_sell": 1, "gather_stencil": 1,
                                "force_stencil": 3, "trials": 27})
    assert sorted(c.calls) == sorted([(P.OPT_TILE, 261), (P.OPT_GATHER_SELL, 1), (P.OPT_GATHER_STENCIL, 1),
                                      (P.OPT_FORCE_STENCIL, 3)])
    assert out["applied"] and out["tile"] == 261
