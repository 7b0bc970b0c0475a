"""Mixed-precision pair passes (qmc2d_set_precision(QMC2D_PRECISION_MIXED)):
the u2 Jastrow and real-space Ewald pair terms in FP32, each thread's sums
compensated, everything else FP64.

Error bounds against the FP64 oracle, per configuration:

- local energy, potential and kinetic energy within 1e-6 Ry per electron;
- -ln psi within 1e-6 relative;
- drift within 1e-6 of the configuration's largest drift component.

Moves: three VMC steps in mixed precision take the same accept decisions as
the oracle's FP64 replay of the same Philox streams; a DMC run's mean energy
agrees with the FP64 path's within the runs' statistical error."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x5EED0F32
DE = 1e-6        # Ry per electron
DLNPSI = 1e-6    # relative
DDRIFT = 1e-6    # relative to the largest drift component

DECKS = {
    "n58_bf": dict(n_up=29, n_down=29, rs=5.0, backflow=(0.2, 5.0, 3.0)),
    "n26_u3_fine": dict(n_up=13, n_down=13, rs=10.0, backflow=(0.2, 10.0, 6.0), u3=True,
                        nknots=6000),
    "pol25_bf": dict(n_up=25, n_down=0, rs=3.0, backflow=(0.2, 3.0, 2.0)),
    "n26_rs1": dict(n_up=13, n_down=13, rs=1.0),
}


def _deck(q, tmp_path, name):
    if name == "n26":
        from conftest import N26
        s = q.System.read(N26, "n26")
        return s, s.read_configs(N26, ".0", 0, 16)
    tables = importlib.import_module("2degas_b200.tables")
    d = tables.make_run(os.path.join(tmp_path, name), "c", nconf=16, seed=23, **DECKS[name])
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 16)


@pytest.mark.parametrize("name", ["n26"] + sorted(DECKS))
def test_evaluation_error_against_fp64_oracle(q, oracle_cls, tmp_path, name):
    s, x = _deck(q, tmp_path, name)
    o = oracle_cls(s)
    with q.Handle(s, capacity=len(x), seed=1) as h:
        h.set_precision("mixed")
        g, hl, p, sg = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert sg[k] == so, f"{name}: sign, config {k}"
        assert abs(p[k][0] - po[0]) < DE, f"{name}: E_L, config {k}"
        assert abs(p[k][1] - po[1]) < DLNPSI * max(1.0, abs(po[1])), f"{name}: -ln psi, config {k}"
        assert abs(p[k][3] - po[3]) < DE, f"{name}: E_pot, config {k}"
        assert abs(p[k][4] - po[4]) < DE, f"{name}: E_kin, config {k}"
        assert np.abs(g[k] - go).max() < DDRIFT * np.abs(go).max(), f"{name}: drift, config {k}"


def test_fp64_is_the_default_and_restorable(q, oracle_cls, n26, n26_configs):
    x = n26_configs[:8]
    o = oracle_cls(n26)
    with q.Handle(n26, capacity=8, seed=1) as h:
        g0, _, p0, _ = h.compute_properties(x)
        h.set_precision("mixed")
        h.compute_properties(x)
        h.set_precision("fp64")
        g, hl, p, sg = h.compute_properties(x)
    assert np.array_equal(p, p0) and np.array_equal(g, g0)
    for k in range(8):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert abs(p[k][0] - po[0]) <= 1e-10 * abs(po[0])


def test_vmc_takes_the_fp64_decisions(q, oracle_cls, tmp_path):
    s, x = _deck(q, tmp_path, "n58_bf")
    nw, nstp, delta = len(x), 3, 0.02 * 25.0
    o = oracle_cls(s)
    pop = o.population_init(x)
    blk_o, nacc_o = o.vmc_philox(pop, nstp, delta, 1000, SEED, 0)
    with q.Handle(s, capacity=nw, seed=SEED) as h:
        h.set_precision("mixed")
        h.population_set(x)
        h.block_reset()
        h.vmc(nstp, delta, 1000)
        got = h.population_get()
        cnt = h.counters()
    assert cnt["accepted"] == nacc_o
    assert np.abs(got["x"] - pop["x"]).max() < 1e-6
    assert np.abs(got["p"][:, 0] - pop["p"][:, 0]).max() < DE


def test_dmc_mean_energy_within_statistical_error(q, n26, n26_configs):
    """Eight blocks of five generations of 64 walkers in each precision, the
    same seed: the block-mean energies agree within their combined error."""
    nw, nblk, ngen = 64, 8, 5
    x0 = n26_configs[:nw]
    means = {}
    for prec in ("fp64", "mixed"):
        e = []
        with q.Handle(n26, capacity=nw, seed=SEED) as h:
            h.set_precision(prec)
            h.population_set(x0)
            for _ in range(nblk):
                h.block_reset()
                h.dmc(ngen, 1, 0.05, -0.44, 5.0, 1000)
                blk, norm = h.block_get()
                e.append(blk[0] / norm)
        e = np.array(e)
        means[prec] = (e.mean(), e.std(ddof=1) / np.sqrt(nblk))
    (m1, s1), (m2, s2) = means["fp64"], means["mixed"]
    assert abs(m1 - m2) < 3.0 * np.hypot(s1, s2), means
