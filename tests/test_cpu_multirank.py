"""Multi-rank host logic of bench.py on CPU: two gloo ranks, as torchrun
would start them (one process per GPU on a B200 node).

Every rank propagates its own population (weak scaling, no collective on
the data path); the only collectives are the max-over-ranks reductions of
the timings. These tests check that reduction, the whole-job rate formula,
that the ranks' populations are independent, and that the reference arm
runs on rank 0 alone."""
import importlib
import importlib.util
import io
import os
import socket
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        dev_ms = [3.0, 7.5][rank]  # rank 1 is the slow one
        t_max = b.max_over_ranks(dev_ms, dist, "cpu")
        rate = b.whole_job_rate(world, 4096, 10, t_max * 1e-3)
        out.put((rank, t_max, rate, b.rank_seeds(rank)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, t_max, rate, seeds in res:
        assert t_max == 7.5
        assert rate == pytest.approx(2 * 4096 * 10 / 7.5e-3)
    assert res[0][3] != res[1][3]  # independent configuration and walker streams


def test_single_rank_needs_no_process_group():
    b = _bench()
    assert b.max_over_ranks(4.25) == 4.25
    assert b.whole_job_rate(1, 100, 3, 0.5) == 600.0


def test_rank_populations_differ(tmp_path):
    """make_config with the two ranks' seeds draws different walkers."""
    b = _bench()
    s0, _ = b.rank_seeds(0)
    s1, _ = b.rank_seeds(1)
    tables = importlib.import_module("2degas_b200.tables")
    cfg = tables.CONFIGS[b.CONFIG]
    x = []
    for s in (s0, s1):
        d = tables.make_run(str(tmp_path / f"r{s}"), "c", nconf=4, seed=s, **cfg)
        x.append(sorted(open(os.path.join(d, f)).read() for f in os.listdir(d) if ".x.0" in f))
    assert x[0] and x[0] != x[1]


def test_reference_arm_runs_on_rank_zero_only():
    b = _bench()

    class A:
        steps, warmup = 1, 3

    buf = io.StringIO()
    with redirect_stdout(buf):
        assert b.reference_arm(A, 1, 2) == 0
    assert buf.getvalue() == ""
