"""qmc2d_population_load_async: the records other than x and g arrive on a
second stream while the next move's pair kernel runs, and every later use
of the population waits for them. A chain started from asynchronously
loaded records equals the chain started from the same records loaded
synchronously (qmc2d_population_load), bit for bit; a read-back right
after the load returns the records; a second load replaces the first."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DELTA, ETRIAL, MMULT, MAGE = 0.05, -0.45, 2.0, 50


def _pinned(rec):
    import torch

    out = {}
    for k, v in rec.items():
        t = torch.empty(v.size, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = np.ascontiguousarray(v, dtype=np.float64).ravel()
        out[k] = t
    return out


def _load(h, nw, rec, asynchronous):
    pin = _pinned(rec)
    args = [pin[k].data_ptr() for k in ("x", "g", "h", "p", "s", "age")]
    if asynchronous:
        h.population_load_async_ptr(nw, *args)
    else:
        h.population_load_ptr(nw, *args)
    return pin  # the caller keeps the buffers alive until the handle syncs


def _records(q, s, x):
    with q.Handle(s, capacity=len(x), seed=3) as h:
        h.population_set(x)
        h.vmc(4, DELTA, 10 ** 9)
        return h.population_get()


@pytest.mark.parametrize("method", ["dmc", "vmc"])
def test_async_load_gives_the_synchronous_chain(q, n26, n26_configs, method):
    x = n26_configs[:48]
    rec = _records(q, n26, x)
    out = []
    for asynchronous in (False, True):
        with q.Handle(n26, capacity=len(x), seed=11) as h:
            keep = _load(h, len(x), rec, asynchronous)
            if method == "dmc":
                h.dmc(3, 1, DELTA, ETRIAL, MMULT, MAGE)
            else:
                h.vmc(3, DELTA, 10 ** 9)
            del keep
            blk, norm = h.block_get()
            out.append((h.population_get(), blk, norm))
    (a, ba, na), (b, bb, nb) = out
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(ba, bb) and na == nb


def test_read_back_and_reload(q, n26, n26_configs):
    x = n26_configs[:32]
    rec1 = _records(q, n26, x)
    rec2 = {k: v.copy() for k, v in rec1.items()}
    rec2["x"] = rec2["x"] + 0.125
    rec2["p"] = rec2["p"] * 2.0
    rec2["age"] = rec2["age"] + 7.0
    with q.Handle(n26, capacity=len(x), seed=5) as h:
        keep1 = _load(h, len(x), rec1, True)
        got = h.population_get()  # joins the side copies first
        for k in rec1:
            assert np.array_equal(got[k].ravel(), np.asarray(rec1[k]).ravel()), k
        keep2 = _load(h, len(x), rec2, True)
        got = h.population_get()
        for k in rec2:
            assert np.array_equal(got[k].ravel(), np.asarray(rec2[k]).ravel()), k
        del keep1, keep2
