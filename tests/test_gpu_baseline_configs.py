"""GPU parity on the decks of the benchmark configurations that the
headline DMC line does not run:

- vmc_n26_rs1 (plain VMC, N = 26 unpolarised, r_s = 1, 1000-knot u2 cut at
  L/2, eta = 0 backflow table so that the reference's determinant routine
  carries the 13 lowest plane waves per spin, 2D Ewald): evaluation at 1e-10
  against the oracle and three VMC steps of 64 walkers at the Gaussian step
  0.3 r_s (delta = 0.045 r_s^2) that replay the oracle's Philox streams;
- rmc_n26_rs10 and rmc_n58_rs10 (reptation, r_s = 10, u2 + u3 + backflow):
  evaluation at 1e-10, and 4 reptiles of 200 beads with one-bead head moves
  (mdelta = 1, tau = 0.01 r_s^2) over 300 moves, more than the ring of
  nbuf = ntau + mdelta = 201 slots, so that the ring index wraps
  (reptation_move, reptation.f:1897-2160; n_buffer :1782). Each reptile
  starts as a random walk of 200 beads with the propagator's link variance;
  a move is forced after two rejections (mage_r = 2, reptation_metropolis_test
  :1865-1895), which keeps about half the moves accepted from that start.
  Both launch shapes of the moves (qmc2d_rmc_set_launch: the pair passes in a
  kernel of their own, or whole moves in one kernel) replay it.

Every deck is read by the product and, independently, by the oracle's own
reader."""
import importlib
import os

import numpy as np
import pytest

from oracle_lib import Reptile

pytestmark = pytest.mark.gpu

SEED = 0xBA5E11E5
RTOL = 1e-10


def close(a, b):
    """|a-b| / max(|b|, 1e-3 max|b|), elementwise maximum."""
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)).max()


def _deck(q, tmp_path, name, nconf):
    tables = importlib.import_module("2degas_b200.tables")
    cfg = tables.CONFIGS[name]
    d = tables.make_run(os.path.join(tmp_path, name), "c", nconf=nconf, seed=29, **cfg)
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, nconf), cfg["rs"]


@pytest.mark.parametrize("name", ["vmc_n26_rs1", "rmc_n26_rs10", "rmc_n58_rs10"])
def test_config_deck_evaluation(q, oracle_cls, tmp_path, name):
    s, x, _ = _deck(q, tmp_path, name, 16)
    o = oracle_cls(s)
    with q.Handle(s, capacity=16, seed=1) as h:
        g, hl, p, sg = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert close(p[k], po) < RTOL, (name, k)
        assert close(g[k], go) < RTOL
        assert close(hl[k], ho) < RTOL
        assert sg[k] == so


def test_config0_vmc_replay(q, oracle_cls, tmp_path):
    s, x, rs = _deck(q, tmp_path, "vmc_n26_rs1", 64)
    delta, nstp, mage = 0.045 * rs * rs, 3, 10 ** 6
    o = oracle_cls(s)
    pop = o.population_init(x)
    blk_o, nacc_o = o.vmc_philox(pop, nstp, delta, mage, SEED, 0)
    with q.Handle(s, capacity=64, seed=SEED) as h:
        h.population_set(x)
        h.block_reset()
        h.vmc(nstp, delta, mage)
        got = h.population_get()
        blk, norm = h.block_get()
        cnt = h.counters()
    assert cnt["accepted"] == nacc_o and 0 < nacc_o < 64 * nstp
    assert norm == 64 * nstp
    assert close(got["x"], pop["x"]) < 1e-11
    assert close(got["p"], pop["p"]) < 1e-9
    assert close(blk, blk_o) < 1e-9


@pytest.mark.parametrize("split", [1, 0])
@pytest.mark.parametrize("name", ["rmc_n26_rs10", "rmc_n58_rs10"])
def test_config2_reptation_ring_wraps(q, oracle_cls, tmp_path, name, split):
    capi = importlib.import_module("2degas_b200._capi")
    nrep, ntau, mdelta, nstp, mage_r = 4, 200, 1, 300, 2
    s, x0, rs = _deck(q, tmp_path, name, nrep)
    delta, etrial = 0.01 * rs * rs, -0.27
    # each reptile starts as a random walk from one configuration, with the
    # link variance of the propagator (2 hbs2m delta = 2 delta / r_s^2)
    rng = np.random.default_rng(7)
    var = 2.0 * delta / rs ** 2
    steps = rng.normal(0.0, np.sqrt(var), size=(nrep, ntau, x0.shape[1]))
    steps[:, 0] = 0.0
    x = (x0[:, None, :] + np.cumsum(steps, axis=1)).reshape(nrep * ntau, -1)
    prm = capi.RmcParams(ntau, 1, mdelta, delta, etrial, 10 ** 6, mage_r)
    o = oracle_cls(s)
    blk_o = np.zeros(s.nprops)
    nacc_o = 0
    paths = []
    for r in range(nrep):
        rep = Reptile(o, prm)
        rep.init(x[r * ntau:(r + 1) * ntau])
        b, na = rep.run(r, SEED, 0, nstp)
        blk_o += b
        nacc_o += na
        paths.append(rep.path())
    with q.Handle(s, capacity=nrep, seed=SEED) as h:
        h.rmc_set_launch(split)
        h.rmc_init(nrep, x, ntau, 1, mdelta, delta, etrial, 10 ** 6, mage_r)
        h.block_reset()
        h.rmc(nstp)
        blk, norm = h.block_get()
        cnt = h.counters()
        for r in range(nrep):
            xg, pg = h.rmc_get_path(r, ntau)
            assert close(xg, paths[r][0]) < 1e-10, (name, r)
            assert close(pg, paths[r][1]) < 1e-9
    assert norm == nrep * nstp
    assert cnt["accepted"] == nacc_o and 0 < nacc_o < nrep * nstp
    assert close(blk, blk_o) < 1e-9
