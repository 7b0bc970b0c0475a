"""Batched populations (qmc2d_batch_*): populations of different N,
density and polarisation advanced together through one CUDA graph per call
give the walkers, block sums and counters of the same qmc2d_vmc /
qmc2d_dmc calls made handle by handle, bit for bit, for even step counts
(graph replays only), odd ones (one more generation launched directly) and
counts beyond one graph (replays of 16 generations, the rest launched
directly), and across calls that reuse or recapture the graph."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DECKS = [  # n_up, n_down, rs, backflow, walkers
    (13, 13, 2.0, True, 64),
    (21, 0, 5.0, True, 96),
    (21, 21, 1.0, True, 160),
    (13, 13, 10.0, False, 32),
]


@pytest.fixture(scope="module")
def systems(q, tmp_path_factory):
    tables = importlib.import_module("2degas_b200.tables")
    d0 = tmp_path_factory.mktemp("batch")
    out = []
    for k, (nu, nd, rs, bf, nw) in enumerate(DECKS):
        d = tables.make_run(os.path.join(d0, f"p{k}"), "c", nu, nd, rs,
                            backflow=(0.2, rs, 0.6 * rs) if bf else None)
        out.append((q.System.read(d, "c"), rs, nw))
    return out


def _start(q, systems):
    hs = []
    for k, (s, rs, nw) in enumerate(systems):
        h = q.Handle(s, capacity=nw, seed=100 + k)
        L = s.s.el[0]
        x = np.random.default_rng(k).uniform(-L / 2, L / 2, size=(nw, 2 * s.N))
        h.population_set(x)
        h.vmc(6, 0.05 * rs * rs, 10 ** 9)
        h.block_reset()
        hs.append(h)
    return hs


def _state(h):
    p = h.population_get()
    blk, norm = h.block_get()
    return p["x"], p["p"], blk, norm, h.counters()


def _same(a, b):
    for u, v in zip(a[:4], b[:4]):
        assert np.array_equal(u, v)
    assert a[4] == b[4]


@pytest.mark.parametrize("ngen", [4, 3, 37])
def test_batch_dmc_equals_handle_by_handle(q, systems, ngen):
    taus = [0.01 * rs * rs for _, rs, _ in systems]
    et = [-0.3, -0.1, 0.4, -0.05]
    ref = _start(q, systems)
    for h, t, e in zip(ref, taus, et):
        h.dmc(ngen, 1, t, e, 2.0, 50)
    hs = _start(q, systems)
    with q.Batch(hs) as b:
        b.dmc(ngen, taus, et, 2.0, 50)
    for h, r in zip(hs, ref):
        _same(_state(h), _state(r))


def test_batch_vmc_and_graph_reuse(q, systems):
    taus = [0.05 * rs * rs for _, rs, _ in systems]
    ref = _start(q, systems)
    for h, t in zip(ref, taus):
        h.vmc(4, t, 10 ** 9)
        h.vmc(4, t, 10 ** 9)
        h.dmc(2, 1, 0.2 * t, -0.2, 2.0, 50)
        h.dmc(2, 1, 0.2 * t, -0.25, 2.0, 50)
    hs = _start(q, systems)
    with q.Batch(hs) as b:
        b.vmc(4, taus)
        b.vmc(4, taus)  # the cached graph replays
        b.dmc(2, [0.2 * t for t in taus], -0.2)
        b.dmc(2, [0.2 * t for t in taus], -0.25)  # a new trial energy: captured again
    for h, r in zip(hs, ref):
        _same(_state(h), _state(r))


@pytest.mark.parametrize("lanes", [1, 2])
def test_batch_lanes_do_not_change_results(q, systems, lanes):
    taus = [0.01 * rs * rs for _, rs, _ in systems]
    et = [-0.3, -0.1, 0.4, -0.05]
    ref = _start(q, systems)
    for h, t, e in zip(ref, taus, et):
        h.dmc(5, 1, t, e, 2.0, 50)
    hs = _start(q, systems)
    with q.Batch(hs) as b:
        b.set_lanes(lanes)
        b.dmc(5, taus, et, 2.0, 50)
    for h, r in zip(hs, ref):
        _same(_state(h), _state(r))
