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
