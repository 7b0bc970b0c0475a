"""DMC across ranks on one GPU without ranks that wait on one another:
- with one rank, 2degas_b200/multirank.py's generations (weights on the
  device, the host plan of qmc2d_comb_plan, qmc2d_population_resample)
  give the walkers, sign and age that qmc2d_dmc gives, walker for walker;
- two handles in one process stand in for two ranks: their weights are
  gathered on the host, each handle's plan is computed, the records it
  sends are packed on the device (qmc2d_records_pack) and unpacked into the
  other handle (qmc2d_records_unpack), then each resamples. Every slot of
  both populations must hold the record that the line-by-line
  transcription of the reference's multi-rank branch2 (tests/branch2_ref.py;
  reptation.f:2162-2258) puts there, over three generations."""
import importlib

import numpy as np
import pytest

from branch2_ref import transcribed_branch2

pytestmark = pytest.mark.gpu

SEED = 0xD0C0B1


def records(h):
    p = h.population_get()
    return np.concatenate([p["x"], p["g"], p["h"], p["p"], p["s"][:, None], p["age"][:, None]],
                          axis=1)


def test_one_rank_equals_qmc2d_dmc(q, n26, n26_configs):
    import torch

    mr = importlib.import_module("2degas_b200.multirank")
    nw, ngen, delta, et = 32, 3, 0.05, -0.43
    with q.Handle(n26, capacity=nw, seed=SEED) as a, q.Handle(n26, capacity=nw, seed=SEED) as b:
        a.population_set(n26_configs[:nw])
        b.population_set(n26_configs[:nw])
        a.dmc(ngen, 1, delta, et, 5.0, 1000)
        pop = mr.HandleRecords(b, torch.device("cuda"))
        mr.dmc_generations(pop, None, ngen, 1, delta, et, 5.0, 1000, SEED, device="cuda")
        ra, rb = records(a), records(b)
    assert np.array_equal(ra, rb)


def test_two_handles_exchange_as_the_reference(q, oracle_cls, n26, n26_configs):
    import torch

    mr = importlib.import_module("2degas_b200.multirank")
    o = oracle_cls(n26)
    nw, ngen, delta, et = 24, 3, 0.05, -0.43
    comb_seed = 0xC0B1
    lib = q.load_library()
    with q.Handle(n26, capacity=nw, seed=SEED) as h0, \
            q.Handle(n26, capacity=nw, seed=SEED + 1) as h1:
        hs = [h0, h1]
        h0.population_set(n26_configs[:nw])
        h1.population_set(n26_configs[nw:2 * nw])
        L = h0.record_len()
        moved = 0
        for gen in range(ngen):
            w = [h.dmc_weights(1, delta, et, 5.0, 1000) for h in hs]
            before = [records(h) for h in hs]
            assert before[0].shape[1] == L
            u = np.array([o.philox_uniform2(comb_seed, c, 0xFFFFFFFF, gen, 1)[0]
                          for c in range(2 * nw)])
            want = transcribed_branch2(before, w, u)
            plans = [mr.comb_plan(lib, np.concatenate(w), 2, nw, comb_seed, gen, r)
                     for r in range(2)]
            # the exchange: rank r's k-th send to p is rank p's k-th receive from r
            for r in range(2):
                p = 1 - r
                sends = [s for (peer, s) in plans[r][1] if peer == p]
                recvs = [s for (peer, s) in plans[p][2] if peer == r]
                assert len(sends) == len(recvs)
                if sends:
                    buf = torch.empty((len(sends), L), dtype=torch.float64, device="cuda")
                    hs[r].records_pack(sends, buf.data_ptr())
                    torch.cuda.synchronize()
                    hs[p].records_unpack(recvs, buf.data_ptr())
                    moved += len(sends)
            for r in range(2):
                hs[r].population_resample(plans[r][0])
            for r in range(2):
                assert np.array_equal(records(hs[r]), want[r]), (gen, r)
        assert moved > 0
