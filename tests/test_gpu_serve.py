"""Serving loop on the GPU: a request's result is the same when it runs
alone and when it runs in a mix of requests admitted together (continuous
batching, one handle, stream and host thread per request), and admission
by HBM footprint keeps the device share within the budget."""
import importlib

import pytest

pytestmark = pytest.mark.gpu

serve = importlib.import_module("2degas_b200.serve")


def _requests():
    # fixed block counts (target 0, min = max) so alone and mixed runs do the same work
    kw = dict(target=0.0, block_steps=5, equil_steps=10)
    return [
        serve.Request(13, 13, 2.0, method="vmc", walkers=128, seed=11, min_blocks=4,
                      max_blocks=4, rid=0, **kw),
        serve.Request(21, 0, 5.0, method="dmc", walkers=192, seed=12, min_blocks=3,
                      max_blocks=3, rid=1, **kw),
        serve.Request(21, 21, 1.0, method="dmc", walkers=320, seed=13, min_blocks=3,
                      max_blocks=3, rid=2, **kw),
        serve.Request(13, 13, 10.0, method="dmc", walkers=64, seed=14, min_blocks=3,
                      max_blocks=3, backflow=False, rid=3, **kw),
    ]


def test_result_is_the_same_alone_and_in_the_mix(q, tmp_path):
    alone = {}
    for r in _requests():
        srv = serve.Server(hbm_bytes=8 << 30, max_slots=1, workdir=str(tmp_path / f"a{r.rid}"))
        (res,) = srv.serve([r], realtime=False)
        assert res.status == "max_blocks", res.message
        alone[r.rid] = res
    srv = serve.Server(hbm_bytes=8 << 30, max_slots=4, workdir=str(tmp_path / "mix"))
    mixed = srv.serve(_requests(), realtime=False)
    assert srv.peak_active >= 2
    for res in mixed:
        a = alone[res.rid]
        assert res.status == a.status
        assert res.block_means == a.block_means, res.rid  # bit for bit
        assert res.energy == a.energy and res.error == a.error
        assert res.moves == a.moves


def test_admission_keeps_within_the_budget(q, tmp_path):
    reqs = _requests()
    prep = [serve.prepare_request(r, str(tmp_path / "p")) for r in reqs]
    fp = sorted(p.footprint for p in prep)
    budget = fp[-1] + fp[-2] - 1  # the two largest never run together
    srv = serve.Server(hbm_bytes=budget, max_slots=4, workdir=str(tmp_path / "b"))
    res = srv.serve(_requests(), realtime=False)
    assert all(r.status == "max_blocks" for r in res), [r.message for r in res]
    assert srv.peak_used <= budget


def test_a_state_point_beyond_the_kernels_is_rejected_not_fatal(q, tmp_path):
    # 89 + 89 electrons: beyond the largest walker the library holds (162)
    big = serve.Request(89, 89, 2.0, method="vmc", walkers=64, seed=3, max_blocks=1,
                        min_blocks=1, target=0.0, rid=0)
    small = _requests()[0]
    small.rid = 1
    srv = serve.Server(hbm_bytes=8 << 30, max_slots=2, workdir=str(tmp_path))
    res = srv.serve([big, small], realtime=False)
    assert res[0].status == "rejected" and res[0].message
    assert res[1].status == "max_blocks"
