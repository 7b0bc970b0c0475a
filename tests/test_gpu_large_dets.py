"""Determinants beyond one CTA's shared memory (more than 45 electrons per
spin unpolarised, 49 polarised): the orbital, inversion, F and cross-term
matrices of each walker live in a per-walker block of HBM, the rest of the
walker in shared memory. Checked against the oracle at 49+49, 57 polarised,
the largest unpolarised shell, 81+81 (N=162), and 121 and 161 polarised:
the batched evaluation, VMC moves, DMC generations and reptation moves,
bit for bit in the Philox stream."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x6A7A


def close(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    same = a == b
    a, b = np.where(same, 0.0, a), np.where(same, 0.0, b)
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)).max()


@pytest.fixture(scope="module",
                params=[(49, 49, 2.0), (57, 0, 3.0), (81, 81, 5.0), (121, 0, 4.0),
                        (161, 0, 4.0)],
                ids=["n98", "pol57", "n162", "pol121", "pol161"])
def large(q, tmp_path_factory, request):
    tables = importlib.import_module("2degas_b200.tables")
    nu, nd, rs = request.param
    d = tables.make_run(str(tmp_path_factory.mktemp("large") / "d"), "c", nu, nd, rs, nconf=6,
                        seed=5, backflow=(0.2, rs, 0.6 * rs))
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 6), rs


def test_properties_match_the_oracle(q, oracle_cls, large):
    s, x, _ = large
    o = oracle_cls(s)
    with q.Handle(s, capacity=len(x), seed=1) as h:
        g, hl, p, sg = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert close(g[k], go) < 1e-9 and close(hl[k], ho) < 1e-9
        assert close(p[k], po) < 1e-9 and sg[k] == so


def test_vmc_and_dmc_match_the_oracle(q, oracle_cls, large):
    s, x, rs = large
    o = oracle_cls(s)
    delta = 0.01 * rs * rs
    ref = o.population_init(x)
    _, nacc = o.vmc_philox(ref, 2, delta, 1000, SEED, 0)
    with q.Handle(s, capacity=len(x), seed=SEED) as h:
        h.population_set(x)
        h.vmc(2, delta, 1000)
        got = h.population_get()
        assert h.counters()["accepted"] == nacc
        assert close(got["x"], ref["x"]) < 1e-10
        e0 = float(np.mean(got["p"][:, 0]))
        h.dmc(2, 1, delta, e0, 2.0, 50)
        gotd = h.population_get()
    o.dmc_philox(ref, 2, 1, delta, e0, 2.0, 50, SEED, 0, 2)
    assert close(gotd["x"], ref["x"]) < 1e-10


def test_footprint_counts_the_matrix_blocks(q, large):
    s, x, _ = large
    small = s.footprint(len(x))
    big = s.footprint(4 * len(x))
    n = max(int(v) for v in s.s.np[:s.s.ntypes])
    # at least the two spins' orbital matrices (complex, n x n) per walker
    assert big - small >= 3 * len(x) * 16 * n * n


def test_reptation_matches_the_oracle(q, oracle_cls, large):
    """Reptiles of these shells use one walker slot's determinant block each;
    with capacity 2 the 6 beads of read_path are evaluated in three launches
    of two."""
    capi = importlib.import_module("2degas_b200._capi")
    from oracle_lib import Reptile

    s, x, rs = large
    o = oracle_cls(s)
    nrep, ntau, nstp = 2, 3, 4
    delta = 0.01 * rs * rs
    rng = np.random.default_rng(3)
    st = rng.normal(0.0, np.sqrt(2.0 * delta / rs ** 2), size=(nrep, ntau, x.shape[1]))
    st[:, 0] = 0.0
    xp = (x[:nrep, None, :] + np.cumsum(st, axis=1)).reshape(nrep * ntau, -1)
    prm = capi.RmcParams(ntau, 1, 1, delta, -1.0, 1000, 2)
    paths, nacc_o = [], 0
    for r in range(nrep):
        rep = Reptile(o, prm)
        rep.init(xp[r * ntau:(r + 1) * ntau])
        _, na = rep.run(r, SEED, 0, nstp)
        nacc_o += na
        paths.append(rep.path())
    with q.Handle(s, capacity=nrep, seed=SEED) as h:
        h.rmc_init(nrep, xp, ntau, 1, 1, delta, -1.0, 1000, 2)
        h.rmc(nstp)
        assert h.counters()["accepted"] == nacc_o
        for r in range(nrep):
            xg, pg = h.rmc_get_path(r, ntau)
            assert close(xg, paths[r][0]) < 1e-10
            assert close(pg, paths[r][1]) < 1e-9
