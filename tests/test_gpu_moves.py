"""GPU parity of the walker moves against the CPU oracle.

The device draws its random numbers from Philox4x32-10 streams keyed by
(seed, walker slot, move index); the oracle replays the same streams, so a
few VMC steps, DMC generations and reptation moves must give the same walkers
and the same block sums up to round-off. Chains are kept short so that no
accept/reject decision sits within round-off of its threshold.
"""
import numpy as np
import pytest

from oracle_lib import Reptile
from variants import write_variant

pytestmark = pytest.mark.gpu

SEED = 0x5EED1234ABCD


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("backflow", [True, False])
def test_vmc_steps(q, oracle_cls, tmp_path, n26_configs, backflow):
    d = write_variant(tmp_path, "v", backflow=backflow, ntwists=4 if backflow else 0)
    sysobj = q.System.read(d, "v")
    nw, nstp, delta, mage = 8, 6, 0.05, 1000
    x0 = n26_configs[:nw]
    o = oracle_cls(sysobj)
    pop = o.population_init(x0)
    blk_o, nacc_o = o.vmc_philox(pop, nstp, delta, mage, SEED, 0)
    with q.Handle(sysobj, capacity=nw, seed=SEED) as h:
        h.population_set(x0)
        h.block_reset()
        h.vmc(nstp, delta, mage)
        got = h.population_get()
        blk, norm = h.block_get()
        cnt = h.counters()
    assert cnt["accepted"] == nacc_o
    assert norm == nw * nstp
    assert rel(got["x"], pop["x"]) < 1e-11
    assert rel(got["g"], pop["g"]) < 1e-9
    assert rel(got["p"][:, :14], pop["p"][:, :14]) < 1e-9
    assert np.array_equal(got["age"], pop["age"])
    assert rel(blk[:14], blk_o[:14]) < 1e-9


def test_vmc_forced_moves(q, oracle_cls, n26, n26_configs):
    """mage = 0 forces every move (move, reptation.f:4650-4653)."""
    nw = 4
    x0 = n26_configs[:nw]
    o = oracle_cls(n26)
    pop = o.population_init(x0)
    o.vmc_philox(pop, 3, 0.05, 0, SEED, 0)
    with q.Handle(n26, capacity=nw, seed=SEED) as h:
        h.population_set(x0)
        h.vmc(3, 0.05, 0)
        got = h.population_get()
        cnt = h.counters()
    # age starts at 0 == mage, a forced move has p = 1 and is accepted, so
    # age returns to 0: every move is forced
    assert cnt["forced"] == nw * 3
    assert rel(got["x"], pop["x"]) < 1e-11


@pytest.mark.parametrize("lanes,move_inv", [(8, 1), (4, 1), (16, 1), (8, 2)])
def test_dmc_generations(q, oracle_cls, n26, n26_configs, lanes, move_inv):
    nw, ngen, mmstep, delta = 32, 3, 2, 0.05
    etrial, mmult, mage = -0.43, 5.0, 1000
    x0 = n26_configs[:nw]
    o = oracle_cls(n26)
    pop = o.population_init(x0)
    blk_o, norm_o, _ = o.dmc_philox(pop, ngen, mmstep, delta, etrial, mmult, mage, SEED)
    with q.Handle(n26, capacity=nw, seed=SEED) as h:
        h.set_pair_lanes(lanes)  # lanes per particle of the pair passes
        h.set_move_inversion(move_inv)  # 2: orbitals and inversion in orb_inv_kernel
        h.population_set(x0)
        h.block_reset()
        h.dmc(ngen, mmstep, delta, etrial, mmult, mage)
        got = h.population_get()
        blk, norm = h.block_get()
    assert rel(got["x"], pop["x"]) < 1e-10
    assert rel(got["p"][:, :14], pop["p"][:, :14]) < 1e-9
    assert abs(norm - norm_o) / norm_o < 1e-10
    assert rel(blk[:14], blk_o[:14]) < 1e-9


@pytest.mark.parametrize("split,lanes", [(1, 8), (0, 8), (1, 4), (1, 16)])
def test_reptation_moves(q, oracle_cls, n26, n26_configs, split, lanes):
    from ctypes import c_double, c_int  # noqa: F401

    import importlib

    capi = importlib.import_module("2degas_b200._capi")
    nrep, ntau, mdelta, nstp = 2, 8, 2, 6
    prm = capi.RmcParams(ntau, 1, mdelta, 0.05, -0.43, 1000, 1000)
    x = n26_configs[: nrep * ntau]
    o = oracle_cls(n26)
    blk_o = np.zeros(n26.nprops)
    paths = []
    for r in range(nrep):
        rep = Reptile(o, prm)
        rep.init(x[r * ntau:(r + 1) * ntau])
        b, _ = rep.run(r, SEED, 0, nstp)
        blk_o += b
        paths.append(rep.path())
    with q.Handle(n26, capacity=nrep, seed=SEED) as h:
        h.rmc_set_launch(split)
        h.set_pair_lanes(lanes)
        h.rmc_init(nrep, x, ntau, 1, mdelta, 0.05, -0.43, 1000, 1000)
        h.block_reset()
        h.rmc(nstp)
        blk, norm = h.block_get()
        for r in range(nrep):
            xg, pg = h.rmc_get_path(r, ntau)
            assert rel(xg, paths[r][0]) < 1e-10
            assert rel(pg[:, :14], paths[r][1][:, :14]) < 1e-9
    assert norm == nrep * nstp
    assert rel(blk[:14], blk_o[:14]) < 1e-9


def test_dmc_ecut(q, n26, n26_configs):
    """qmc2d_set_dmc_ecut: a cutoff no E_L reaches changes nothing; a small
    one bounds every weight to exp(+-npnorm ecut delta) (capped at mmult)."""
    nw, ngen, delta, et = 32, 4, 0.05, -0.43
    x0 = n26_configs[:nw]
    out = {}
    for ecut in (0.0, 1e300, 1e-3):
        with q.Handle(n26, capacity=nw, seed=SEED) as h:
            h.set_dmc_ecut(ecut)
            h.population_set(x0)
            h.block_reset()
            h.dmc(ngen, 1, delta, et, 5.0, 1000)
            blk, norm = h.block_get()
            out[ecut] = (h.population_get()["x"], blk, norm)
    assert np.array_equal(out[1e300][0], out[0.0][0]) and np.array_equal(out[1e300][1], out[0.0][1])
    lim = np.exp(n26.s.npnorm * 1e-3 * delta)
    per_gen = out[1e-3][2] / (nw * ngen)
    assert 1.0 / lim <= per_gen <= lim
    with q.Handle(n26, capacity=4, seed=1) as h:
        with pytest.raises(q.QMCError):
            h.set_dmc_ecut(-1.0)
