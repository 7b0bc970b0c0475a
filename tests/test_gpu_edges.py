"""Edge cases on the GPU: the smallest closed shells (1+1, 5+5, 9
polarised) against the oracle, and bad configurations supplied by the host
(NaN, infinite, two same-spin electrons at one point), which must come back
as status codes and leave the handle usable."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0xED6E
ERR_SINGULAR, ERR_NONFINITE = 7, 8


def close(a, b):
    """Largest relative difference; equal entries (the nodal-distance
    property is +inf on both sides when the drift is exactly zero, as for two
    electrons beyond the u2 cutoff) count as no difference."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    same = a == b
    a, b = np.where(same, 0.0, a), np.where(same, 0.0, b)
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)).max()


@pytest.fixture(params=[(1, 1, 1.5), (5, 5, 2.0), (9, 0, 3.0)], ids=["n2", "n10", "pol9"])
def small(q, tmp_path, request):
    tables = importlib.import_module("2degas_b200.tables")
    nu, nd, rs = request.param
    d = tables.make_run(os.path.join(tmp_path, "d"), "c", nu, nd, rs, nconf=8, seed=3,
                        backflow=(0.2, rs, 0.6 * rs))
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 8), rs


def test_smallest_shells_match_the_oracle(q, oracle_cls, small):
    s, x, rs = small
    o = oracle_cls(s)
    with q.Handle(s, capacity=len(x), seed=1) as h:
        g, hl, p, sg = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert close(g[k], go) < 1e-10 and close(hl[k], ho) < 1e-10
        assert close(p[k], po) < 1e-10 and sg[k] == so
    delta = 0.02 * rs * rs
    pop = o.population_init(x)
    _, nacc = o.vmc_philox(pop, 3, delta, 1000, SEED, 0)
    with q.Handle(s, capacity=len(x), seed=SEED) as h:
        h.population_set(x)
        h.vmc(3, delta, 1000)
        got = h.population_get()
        assert h.counters()["accepted"] == nacc
    assert close(got["x"], pop["x"]) < 1e-11


def _expect(q, call, codes):
    with pytest.raises(q.QMCError) as e:
        call()
    assert e.value.code in codes, str(e.value)


def test_bad_configurations_are_status_codes(q, oracle_cls, n26, n26_configs):
    x = n26_configs[:4].copy()
    o = oracle_cls(n26)
    nan = x.copy()
    nan[1, 5] = np.nan
    inf = x.copy()
    inf[2, 0] = np.inf
    same = x.copy()
    same[3, 2:4] = same[3, 0:2]  # electrons 0 and 1 (both spin up) at one point
    with q.Handle(n26, capacity=4, seed=1) as h:
        _expect(q, lambda: h.compute_properties(nan), (ERR_NONFINITE,))
        _expect(q, lambda: h.compute_properties(inf), (ERR_NONFINITE, ERR_SINGULAR))
        _expect(q, lambda: h.compute_properties(same), (ERR_NONFINITE, ERR_SINGULAR))
        _expect(q, lambda: h.population_set(nan), (ERR_NONFINITE,))
        # the handle and its context are still good
        g, hl, p, sg = h.compute_properties(x)
        h.population_set(x)
        h.vmc(2, 0.05, 1000)
    for k in range(4):
        go, ho, po, so, _ = o.compute_properties(x[k])
        assert close(p[k], po) < 1e-10


def test_device_entry_point_reports_failed_walkers(q, n26, n26_configs):
    """compute_properties_dev is asynchronous; its status words come back
    through compute_properties_dev_status, cleared at every call."""
    import ctypes

    import torch

    x = n26_configs[:4].copy()
    x[1, 5] = np.nan
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    out = [torch.zeros(4 * k, dtype=torch.float64, device="cuda")
           for k in (2 * n26.N, n26.ntypes, n26.nprops, 1)]
    ptrs = [ctypes.c_void_p(t.data_ptr()) for t in [xd] + out]
    with q.Handle(n26, capacity=4, seed=1) as h:
        torch.cuda.synchronize()
        h.compute_properties_dev(4, *ptrs)
        _expect(q, lambda: h.compute_properties_dev_status(4), (ERR_NONFINITE,))
        xd.copy_(torch.tensor(n26_configs[:4], dtype=torch.float64))
        torch.cuda.synchronize()
        h.compute_properties_dev(4, *ptrs)
        h.compute_properties_dev_status(4)
