"""Single-electron moves with Sherman-Morrison inverse updates
(qmc2d_vmc_single) on the plain Slater-Jastrow deck of the VMC benchmark
configuration (N = 26, r_s = 1, u2, eta = 0 backflow table):

- a few sweeps replay the oracle's single-electron chain on the same Philox
  streams, the oracle taking every ratio and drift from a full evaluation
  (no inverse kept), so the device's ratios, updated inverses and refreshes
  are checked against an independent route;
- after ~100 Sherman-Morrison updates without a recompute, the properties
  measured from the updated inverse equal a fresh evaluation of the same
  configurations at 1e-10, and the drift |W D - I| measured before a
  recompute stays at round-off;
- the single-electron chain's mean energy agrees with the oracle's
  all-electron chain (the reference's move, reptation.f:4617-4680) within
  their combined statistical error;
- decks with u3 or a non-zero backflow table are refused."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x51E1EC7
ERR_UNSUPPORTED = 4


def close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)).max()


@pytest.fixture
def plain(q, tmp_path):
    tables = importlib.import_module("2degas_b200.tables")
    cfg = tables.CONFIGS["vmc_n26_rs1"]
    d = tables.make_run(os.path.join(tmp_path, "c0"), "c", nconf=256, seed=41, **cfg)
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 256), 0.045 * cfg["rs"] ** 2


def test_single_sweeps_replay_the_oracle(q, oracle_cls, plain):
    s, x, delta = plain
    nw, nsweep = 12, 3
    o = oracle_cls(s)
    pop = o.population_init(x[:nw])
    blk_o, nacc_o = o.vmc_single(pop, nsweep, delta, SEED, 0)
    with q.Handle(s, capacity=nw, seed=SEED) as h:
        h.population_set(x[:nw])
        h.block_reset()
        h.vmc_single(nsweep, delta, refresh=50)
        got = h.population_get()
        blk, norm = h.block_get()
        cnt = h.counters()
    assert cnt["proposed"] == nw * nsweep * s.N
    assert cnt["accepted"] == nacc_o and 0 < nacc_o < nw * nsweep * s.N
    assert norm == nw * nsweep
    assert close(got["x"], pop["x"]) < 1e-11
    assert close(got["g"], pop["g"]) < 1e-9
    assert close(got["p"], pop["p"]) < 1e-9
    assert close(blk, blk_o) < 1e-9


def test_updated_inverse_equals_fresh_evaluation(q, plain):
    s, x, delta = plain
    nw = 32
    with q.Handle(s, capacity=nw, seed=SEED) as h:
        h.population_set(x[:nw])
        h.vmc_single(4, delta, refresh=0)  # ~100 updates per walker, no recompute
        got = h.population_get()
        g, hl, p, sg = h.compute_properties(got["x"])
        cnt = h.counters()
        assert cnt["accepted"] > 0.5 * nw * 4 * s.N
        cols = [c for c in range(s.nprops) if c != 2]  # all but the acceptance column
        assert close(got["p"][:, cols], p[:, cols]) < 1e-10
        assert close(got["g"], g) < 1e-10
        assert close(got["h"], hl) < 1e-10
        # drift of the updated inverse just before each recompute (every 50 moves)
        h.vmc_single(4, delta, refresh=50)
        drift = h.single_drift()
        assert 0.0 < drift < 1e-9, drift
        got = h.population_get()
        g, hl, p, sg = h.compute_properties(got["x"])
        assert close(got["p"][:, cols], p[:, cols]) < 1e-10


def test_single_electron_energy_matches_all_electron_chain(q, oracle_cls, plain):
    """VMC samples |psi|^2 with either move; the mean local energies of the
    device's single-electron chain and the oracle's all-electron chain agree
    within 4 combined standard errors (errors from blocks of the
    per-step population means)."""
    s, x, delta = plain
    o = oracle_cls(s)
    nw_o, nblk_o, blen_o = 48, 12, 20
    pop = o.population_init(x[:nw_o])
    o.vmc_philox(pop, 60, delta, 10 ** 6, SEED + 1, 0)  # equilibration
    e_o = []
    for b in range(nblk_o):
        blk, _ = o.vmc_philox(pop, blen_o, delta, 10 ** 6, SEED + 1, 60 + b * blen_o)
        e_o.append(blk[0] / (nw_o * blen_o))
    nw_d, nblk_d, blen_d = 256, 20, 20
    e_d = []
    with q.Handle(s, capacity=nw_d, seed=SEED + 2) as h:
        h.population_set(x[:nw_d])
        h.vmc_single(60, delta, refresh=50)  # equilibration
        for b in range(nblk_d):
            h.block_reset()
            h.vmc_single(blen_d, delta, refresh=50)
            blk, norm = h.block_get()
            e_d.append(blk[0] / norm)
    e_o, e_d = np.array(e_o), np.array(e_d)
    m_o, m_d = e_o.mean(), e_d.mean()
    err = np.sqrt(e_o.var(ddof=1) / len(e_o) + e_d.var(ddof=1) / len(e_d))
    assert abs(m_o - m_d) < 4 * err, (m_o, m_d, err)


def test_single_electron_moves_need_a_plain_determinant(q, n26, n26_configs):
    with q.Handle(n26, capacity=4, seed=1) as h:
        h.population_set(n26_configs[:4])
        with pytest.raises(q.QMCError) as e:
            h.vmc_single(1, 0.05)
        assert e.value.code == ERR_UNSUPPORTED
