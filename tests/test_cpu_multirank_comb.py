"""branch2's comb across ranks (reptation.f:2162-2273) on CPU: the plan of
qmc2d_comb_plan (host code of the library), the exchange of
2degas_b200/multirank.py over two gloo ranks, and an independent
line-by-line transcription of the reference's multi-rank branch2
(tests/branch2_ref.py:
the comb with the shared rannyu2 stream, the send/receive loop, prov_dest).

Walker records here are small host arrays whose first entry names the
walker; a walker's DMC weight is a function of that name and of the
generation, so it travels with the walker. Checks:
- one rank: the plan is the oracle's single-population branch2 on the same
  uniforms;
- two gloo ranks, three generations: every rank ends with exactly the
  records the transcription puts there, slot by slot;
- after the first generation the two ranks together hold the same walkers,
  with the same multiplicities, as the oracle's branch2 of the concatenated
  population."""
import importlib
import os
import socket

import numpy as np

from branch2_ref import transcribed_branch2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEED = 0xC0B1
NCONF, L = 24, 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def weight(ids, gen):
    w = np.exp(0.8 * np.sin(1.7 * ids + 0.9 * gen))
    return np.where((ids == 3) & (gen == 0), 12.0, w)  # one weight above wmult = 10


def start_records(rank):
    ids = rank * NCONF + np.arange(NCONF, dtype=np.float64)
    rec = np.zeros((NCONF, L))
    rec[:, 0] = ids
    rec[:, 1:] = ids[:, None] * np.array([0.5, -1.25, 3.0, 0.125])
    return rec


def comb_uniforms(oracle, gen, n):
    return np.array([oracle.philox_uniform2(SEED, c, 0xFFFFFFFF, gen, 1)[0] for c in range(n)])


class FakePop:
    """The population interface of multirank.dmc_generations on host arrays."""

    def __init__(self, lib, recs):
        self.lib, self.recs, self.gen = lib, recs, 0
        self.nw, self.record_len = recs.shape

    def weights(self, *a):
        w = weight(self.recs[:, 0], self.gen)
        self.gen += 1
        return w

    def pack(self, slots):
        import torch

        return torch.tensor(self.recs[slots])

    def empty(self, n):
        import torch

        return torch.empty((n, self.record_len), dtype=torch.float64)

    def unpack(self, slots, buf):
        self.recs[slots] = buf.numpy()

    def resample(self, src):
        self.recs = self.recs[src].copy()


def _rank_main(rank, world, port, ngen, out):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        q = importlib.import_module("2degas_b200")
        mr = importlib.import_module("2degas_b200.multirank")
        pop = FakePop(q.load_library(), start_records(rank))
        mr.dmc_generations(pop, dist, ngen, 1, 0.1, 0.0, 2.0, 50, SEED)
        out.put((rank, pop.recs))
    finally:
        dist.destroy_process_group()


def _two_ranks(ngen):
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, ngen, qu)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(qu.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    return [res[0], res[1]]


def test_one_rank_plan_is_the_oracle_comb(q, oracle_cls, n26):
    mr = importlib.import_module("2degas_b200.multirank")
    o = oracle_cls(n26)
    rng = np.random.default_rng(3)
    for gen in range(4):
        w = rng.uniform(0.2, 3.0, 64)
        w[5] = 14.0
        src, sends, recvs, ncap = mr.comb_plan(q.load_library(), w, 1, 64, SEED, gen, 0)
        mult_o, src_o, used, ncap_o = o.branch2(w, comb_uniforms(o, gen, 64))
        assert not sends and not recvs
        assert ncap == ncap_o == 1
        assert np.array_equal(src, src_o)


def test_two_gloo_ranks_follow_the_reference(oracle_cls, n26):
    o = oracle_cls(n26)
    ngen = 3
    got = _two_ranks(ngen)
    want = [start_records(0), start_records(1)]
    for gen in range(ngen):
        w = [weight(r[:, 0], gen) for r in want]
        want = transcribed_branch2(want, w, comb_uniforms(o, gen, 2 * NCONF))
    for r in range(2):
        assert got[r].shape == (NCONF, L)
        assert np.array_equal(got[r], want[r]), r
    # an exchange happened: some walker left its rank
    assert any(int(v) // NCONF != r for r in range(2) for v in got[r][:, 0])


def test_first_generation_equals_one_population(oracle_cls, n26):
    o = oracle_cls(n26)
    got = _two_ranks(1)
    ids = np.concatenate([start_records(0)[:, 0], start_records(1)[:, 0]])
    mult_o, src_o, _, _ = o.branch2(weight(ids, 0), comb_uniforms(o, 0, 2 * NCONF))
    both = np.sort(np.concatenate([got[0][:, 0], got[1][:, 0]]))
    assert np.array_equal(both, np.sort(ids[src_o]))
    assert np.array_equal(np.bincount(both.astype(int), minlength=2 * NCONF), mult_o)
