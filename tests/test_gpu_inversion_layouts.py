"""The inversion layouts of the determinant section (qmc2d_set_inversion:
0 register-resident over every warp, 1 one warp per spin in shared memory,
2 blocks of eight pivot steps with one-warp panels) against the oracle at
1e-10, and three VMC steps in layouts 1 and 2 against the oracle's replay, on the n26 golden deck (13 + 13, u3, twist), the N = 58
benchmark deck and a polarised shell of 25."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x1A70
CASES = {
    "n58_bf": dict(n_up=29, n_down=29, rs=5.0, backflow=(0.2, 5.0, 3.0)),
    "pol25_bf": dict(n_up=25, n_down=0, rs=3.0, backflow=(0.2, 3.0, 2.0)),
}


def close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)).max()


@pytest.fixture(params=["n26"] + sorted(CASES))
def deck(request, q, tmp_path, n26, n26_configs):
    if request.param == "n26":
        return n26, n26_configs[:8]
    tables = importlib.import_module("2degas_b200.tables")
    d = tables.make_run(os.path.join(tmp_path, request.param), "c", nconf=8, seed=5,
                        **CASES[request.param])
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 8)


@pytest.mark.parametrize("layout", [0, 1, 2])
def test_layout_matches_the_oracle(q, oracle_cls, deck, layout):
    s, x = deck
    o = oracle_cls(s)
    with q.Handle(s, capacity=len(x), seed=1) as h:
        h.set_inversion(layout)
        g, hl, p, sg = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert close(p[k], po) < 1e-10
        assert close(g[k], go) < 1e-10
        assert close(hl[k], ho) < 1e-10


@pytest.mark.parametrize("layout", [1, 2])
def test_layout_vmc_replays_the_oracle(q, oracle_cls, deck, layout):
    s, x = deck
    o = oracle_cls(s)
    pop = o.population_init(x)
    blk_o, nacc_o = o.vmc_philox(pop, 3, 0.05, 1000, SEED, 0)
    with q.Handle(s, capacity=len(x), seed=SEED) as h:
        h.set_inversion(layout)
        h.population_set(x)
        h.block_reset()
        h.vmc(3, 0.05, 1000)
        got = h.population_get()
        blk, norm = h.block_get()
        cnt = h.counters()
    assert cnt["accepted"] == nacc_o
    assert close(got["x"], pop["x"]) < 1e-11
    assert close(blk, blk_o) < 1e-9
