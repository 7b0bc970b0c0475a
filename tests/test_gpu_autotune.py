"""Pair-kernel launch choices (qmc2d_set_launch, qmc2d_set_pair_lanes) and
their autotuner (qmc2d_autotune): every choice of walker groups per CTA and
pair-row staging gives the same walkers bit for bit, lanes per particle 4
and 16 give them to round-off (the partner sums meet in another order), and
tuning leaves the population and the random streams where they were. The
autotuner also picks the inversion layout (qmc2d_set_inversion), whose
choices agree to round-off: bit for bit when it keeps the defaults, to
1e-12 otherwise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DELTA = 0.05


def _run(q, s, x, seed, launch=None, tune=False, nstp=3, lanes=None):
    with q.Handle(s, capacity=len(x), seed=seed) as h:
        h.population_set(x)
        if launch:
            h.set_launch(*launch)
        if lanes:
            h.set_pair_lanes(lanes)
            assert h.get_pair_lanes() == lanes
        got = None
        if tune:
            before = h.population_get()
            got = h.autotune() + (h.get_launch()[2], h.get_pair_lanes())
            after = h.population_get()
            assert np.array_equal(before["x"], after["x"])
        h.vmc(nstp, DELTA, 10 ** 9)
        return h.population_get(), got


@pytest.mark.parametrize("launch", [(1, 0), (1, 1), (2, 1), (2, 0)])
def test_every_launch_choice_gives_the_same_walkers(q, n26, n26_configs, launch):
    ref, _ = _run(q, n26, n26_configs, 7)
    got, _ = _run(q, n26, n26_configs, 7, launch=launch)
    assert np.array_equal(got["x"], ref["x"]) and np.array_equal(got["p"], ref["p"])


@pytest.mark.parametrize("lanes", [4, 16])
def test_pair_lanes_agree_to_round_off(q, n26, n26_configs, lanes):
    ref, _ = _run(q, n26, n26_configs, 7)
    got, _ = _run(q, n26, n26_configs, 7, lanes=lanes)
    assert np.allclose(got["x"], ref["x"], rtol=1e-12, atol=0)
    assert np.allclose(got["p"], ref["p"], rtol=1e-10, atol=1e-12)


def test_autotune_picks_a_choice_and_changes_nothing(q, n26, n26_configs):
    ref, _ = _run(q, n26, n26_configs, 9)
    got, (g, st, ms, inv, lanes) = _run(q, n26, n26_configs, 9, tune=True)
    assert g in (1, 2) and st in (0, 1) and inv in (0, 1, 2) and lanes in (4, 8, 16) and ms > 0
    if inv == 0 and lanes == 8:
        assert np.array_equal(got["x"], ref["x"]) and np.array_equal(got["p"], ref["p"])
    else:
        assert np.allclose(got["x"], ref["x"], rtol=1e-12, atol=0)
        assert np.allclose(got["p"], ref["p"], rtol=1e-10, atol=1e-12)


def test_autotune_scope_keeps_the_choices_outside_it(q, n26, n26_configs):
    with q.Handle(n26, capacity=len(n26_configs), seed=4) as h:
        h.population_set(n26_configs)
        h.set_pair_lanes(16)
        h.set_inversion(1)
        h.set_autotune_scope(1)  # the walker groups and staging only
        h.autotune()
        assert h.get_pair_lanes() == 16 and h.get_launch()[2] == 1
        with pytest.raises(q.QMCError):
            h.set_autotune_scope(8)


def test_set_launch_rejects_bad_choices(q, n26, n26_configs):
    with q.Handle(n26, capacity=4, seed=1) as h:
        with pytest.raises(q.QMCError):
            h.set_launch(3, 0)
        with pytest.raises(q.QMCError):
            h.set_launch(1, 2)
        for bad in (3, 32):
            with pytest.raises(q.QMCError):
                h.set_pair_lanes(bad)
        assert h.get_pair_lanes() == 8
        with pytest.raises(q.QMCError):
            h.set_move_inversion(3)
