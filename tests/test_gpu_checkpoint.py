"""Checkpoints: write_conf (reptation.f:2504) and restart (reptation.f:4439)
through the C-ABI. A restart must continue the same random-stream chain: a
run interrupted by restart_write / restart_read in a fresh handle ends where
the uninterrupted run ends."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DELTA = 0.05


def test_write_conf_round_trip(q, n26, n26_configs, tmp_path):
    x0 = n26_configs[:16]
    with q.Handle(n26, capacity=16, seed=11) as h:
        h.population_set(x0)
        h.vmc(3, DELTA, 10 ** 9)
        x = h.population_get()["x"]
        h.write_conf(tmp_path, rank=0)
    back = n26.read_configs(tmp_path, ".0", 0, 16)
    assert back.shape == x.shape
    assert np.array_equal(back, x)  # %.17E text round-trips doubles exactly


def test_restart_continues_the_chain(q, n26, n26_configs, tmp_path):
    x0 = n26_configs[:16]
    # uninterrupted: 4 + 3 VMC steps
    with q.Handle(n26, capacity=16, seed=5) as h:
        h.population_set(x0)
        h.vmc(4, DELTA, 10 ** 9)
        h.vmc(3, DELTA, 10 ** 9)
        x_ref = h.population_get()["x"]
    # interrupted after 4 steps: restart files, a fresh handle with another seed
    st = q.Stats(n26)
    with q.Handle(n26, capacity=16, seed=5) as h:
        h.population_set(x0)
        h.block_reset()
        h.vmc(4, DELTA, 10 ** 9)
        blk, norm = h.block_get()
        st.add_block(blk, norm)
        h.restart_write(st, 1, "vmc", tmp_path, "n26")
    st2 = q.Stats(n26)
    with q.Handle(n26, capacity=16, seed=999) as h:
        iblk, etrial = h.restart_read(st2, "vmc", tmp_path, "n26")
        h.vmc(3, DELTA, 10 ** 9)
        x_new = h.population_get()["x"]
    assert iblk == 1
    m1, e1, n1, b1 = st.get()
    m2, e2, n2, b2 = st2.get()
    np.testing.assert_allclose(m2, m1, rtol=1e-15)
    assert (n2, b2) == (n1, b1)
    assert etrial == pytest.approx(m1[0], rel=1e-15)
    # the re-evaluated walkers continue the same Philox chain
    np.testing.assert_allclose(x_new, x_ref, rtol=0, atol=1e-9)


def test_update_twist_matches_a_fresh_handle(q, n26, n26_configs):
    """A handle moved to twist (2, 3) evaluates like one created there."""
    x = n26_configs[:8]
    with q.Handle(n26, capacity=8, seed=1) as h:
        n26.set_twist(2, 3)
        h.update_twist()
        g1, hl1, p1, s1 = h.compute_properties(x)
    with q.Handle(n26, capacity=8, seed=1) as h2:
        g2, hl2, p2, s2 = h2.compute_properties(x)
    n26.set_twist(1, 1)
    assert np.array_equal(g1, g2) and np.array_equal(p1, p2)


def test_tabc_visits_the_grid_in_order(q, n26, n26_configs):
    x0 = n26_configs[:8]
    seen = []
    with q.Handle(n26, capacity=8, seed=2) as h:
        h.population_set(x0)
        done = q.tabc(h, lambda hh, i, j: (hh.vmc(1, DELTA, 10 ** 9), seen.append((i, j))),
                      ntheta=2)
        # resume after a restart stored at twist (1, 2), block 1: next twist
        rest = q.tabc(h, lambda hh, i, j: None, ntheta=2, resume=(1, 2, 1))
    n26.set_twist(1, 1)
    assert done == seen == [(1, 1), (1, 2), (2, 1), (2, 2)]
    assert rest == [(2, 1), (2, 2)]


def _state_line(path):
    """The stream-state line of a .res file: seed words, move, generation and
    reptation counters."""
    lines = open(path).read().splitlines()
    for ln in lines[2:]:
        f = ln.split()
        if len(f) == 8 and all(t.lstrip("-").isdigit() for t in f):
            return [int(t) for t in f]
    raise AssertionError("no state line")


def test_reptation_restart_rebuilds_the_paths(q, n26, n26_configs, tmp_path):
    """restart(1) of a reptation run, then restart(0) + read_path in a fresh
    handle: the same paths, every bead evaluated again to the same values,
    and the reptation counter carried on."""
    nrep, ntau = 3, 8
    prm = (ntau, 1, 2, 0.05, -0.43, 1000, 1000)
    x0 = n26_configs[: nrep * ntau]
    st = q.Stats(n26)
    with q.Handle(n26, capacity=nrep, seed=21) as h:
        h.rmc_init(nrep, x0, *prm)
        h.block_reset()
        h.rmc(4)
        blk, norm = h.block_get()
        st.add_block(blk, norm)
        h.restart_write(st, 1, "rmc", tmp_path, "n26")
        paths = [h.rmc_get_path(r, ntau) for r in range(nrep)]
    assert _state_line(tmp_path / "n26.res")[4] == 4
    st2 = q.Stats(n26)
    out = tmp_path / "again"
    out.mkdir()
    with q.Handle(n26, capacity=nrep, seed=999) as h:
        iblk = h.restart_read_rmc(st2, tmp_path, "n26", *prm)
        assert iblk == 1
        for r in range(nrep):
            xr, pr = h.rmc_get_path(r, ntau)
            assert np.array_equal(xr, paths[r][0])
            keep = [i for i in range(14) if i != 2]  # jacc is recomputed, as read_path does
            np.testing.assert_allclose(pr[:, keep], paths[r][1][:, keep], rtol=1e-12, atol=1e-14)
        h.rmc(2)
        h.restart_write(st2, 2, "rmc", out, "n26")
    assert _state_line(out / "n26.res")[4] == 6
    m1, _, n1, b1 = st.get()
    m2, _, n2, b2 = st2.get()
    np.testing.assert_allclose(m2, m1, rtol=1e-15)
    assert (n2, b2) == (n1, b1)


def test_reptation_restart_needs_whole_paths(q, n26, n26_configs, tmp_path):
    st = q.Stats(n26)
    with q.Handle(n26, capacity=16, seed=3) as h:
        h.population_set(n26_configs[:10])
        h.restart_write(st, 1, "vmc", tmp_path, "n26")
    with q.Handle(n26, capacity=4, seed=3) as h:
        with pytest.raises(q.QMCError):
            h.restart_read_rmc(q.Stats(n26), tmp_path, "n26", 8, 1, 2, 0.05, -0.43, 1000, 1000)
