"""Serving loop host logic (no GPU): closed shells, the HBM footprint of a
handle, and admission by footprint with fake preparation and runs."""
import importlib
import threading
import time

import numpy as np
import pytest

serve = importlib.import_module("2degas_b200.serve")


def test_closed_shells():
    assert serve.closed_shells(130)[:14] == [1, 5, 9, 13, 21, 25, 29, 37, 45, 49, 57, 61, 69, 81]


def test_footprint_is_linear_in_walkers_and_counts_every_record(q, n26):
    s = n26
    N, nt, np_ = s.N, s.ntypes, s.nprops
    f = {c: s.footprint(c) for c in (512, 1024, 2048)}
    per = (f[1024] - f[512]) / 512
    assert f[2048] - f[1024] == 1024 * per
    # two populations (x, g, h, p, s, age), block sums, norm, counters,
    # weights, status, comb scratch, staging, the inverse drift record of
    # the single-electron sweeps, and the move scratch
    lib = s.lib
    recs = 2 * (4 * N + nt + np_ + 2) * 8 + (np_ + 1 + 4 + 1) * 8 + 4 + 2 * 8 + 4 * 4 \
        + (4 * N + nt + np_ + 1) * 8 + 8  # + the single-electron sweeps' drift record
    # the move scratch: per-particle sums, rho_k, (backflow) the pair values
    # of the N (N - 1) / 2 pairs i < j and, for spins of at most 32 orbitals,
    # each spin's orbitals, inverse, pivots and singular flag (A n^2 and W
    # n (n|1) complex, 2n + 1 doubles, rounded up to even), rounded up to
    # 256 bytes
    nk = s.s.nk
    pair = (14 * N + 3 + 4 * max(nk, 1) + 3) & ~3
    end = pair + 3 * (N * (N - 1) // 2)
    ns = [s.s.np[t] for t in range(nt)]
    if max(ns) <= 32:
        end = (end + 1) & ~1
        end += sum((2 * n * n + 2 * n * (n | 1) + 2 * n + 2 + 1) & ~1 for n in ns)
    scr = ((end + 31) // 32) * 32 * 8
    assert per == recs + scr
    with pytest.raises(Exception):
        s.footprint(0)


def _fake(footprints, dur=0.15):
    log = {"concurrent": [], "lock": threading.Lock(), "live": 0, "used": 0}

    def prepare(req, workdir):
        return serve.Prepared(req, None, footprints[req.rid])

    def run(p, device):
        with log["lock"]:
            log["live"] += 1
            log["used"] += p.footprint
            log["concurrent"].append((p.req.rid, log["live"], log["used"]))
        time.sleep(dur)
        with log["lock"]:
            log["live"] -= 1
            log["used"] -= p.footprint
        return dict(energy=-1.0 - p.req.rid, error=1e-5, blocks=5, moves=100, status="done")

    return prepare, run, log


def test_admission_by_footprint_first_fit():
    fp = [60, 50, 30, 80, 150]
    prepare, run, log = _fake(fp)
    reqs = [serve.Request(13, 13, 1.0, rid=i, arrival=0.01 * i) for i in range(len(fp))]
    srv = serve.Server(hbm_bytes=100, max_slots=4, prepare=prepare, run=run)
    res = srv.serve(reqs)
    assert [r.status for r in res] == ["done", "done", "done", "done", "rejected"]
    assert srv.peak_used <= 100
    assert max(u for _, _, u in log["concurrent"]) <= 100
    # request 2 (30) fits beside request 0 (60) while request 1 (50) waits
    first = {rid for rid, live, used in log["concurrent"][:2]}
    assert first == {0, 2}
    for r in res[:4]:
        assert r.t_admit >= r.t_arrival and r.t_done > r.t_admit
        assert r.energy == -1.0 - r.rid


def test_slots_bound_concurrency():
    prepare, run, log = _fake([1] * 6, dur=0.1)
    reqs = [serve.Request(13, 13, 1.0, rid=i) for i in range(6)]
    srv = serve.Server(hbm_bytes=100, max_slots=2, prepare=prepare, run=run)
    res = srv.serve(reqs, realtime=False)
    assert all(r.status == "done" for r in res)
    assert srv.peak_active == 2 and max(live for _, live, _ in log["concurrent"]) == 2


def test_hbm_determinant_requests_capped_while_small_ones_fill_in():
    prepare, run, log = _fake([1] * 6, dur=0.1)
    # 0, 2, 4: 81 orbitals per spin (determinants in HBM); 1, 3, 5: 13
    reqs = [serve.Request(81 if i % 2 == 0 else 13, 81 if i % 2 == 0 else 13, 1.0, rid=i)
            for i in range(6)]
    assert [serve.hbm_dets(r) for r in reqs] == [True, False] * 3
    srv = serve.Server(hbm_bytes=100, max_slots=4, prepare=prepare, run=run, max_hbm_dets=1)
    live_big = {"n": 0, "max": 0}
    lock = threading.Lock()

    def run_big(p, device):
        big = serve.hbm_dets(p.req)
        with lock:
            live_big["n"] += big
            live_big["max"] = max(live_big["max"], live_big["n"])
        try:
            return run(p, device)
        finally:
            with lock:
                live_big["n"] -= big

    srv.run_one = run_big
    res = srv.serve(reqs, realtime=False)
    assert all(r.status == "done" for r in res)
    assert live_big["max"] == 1
    # the small requests ran beside the first large one
    assert max(live for _, live, _ in log["concurrent"]) >= 2


def test_a_failed_run_ends_only_its_request():
    prepare, run, _ = _fake([1, 1, 1])

    def flaky(p, device):
        if p.req.rid == 1:
            raise RuntimeError("boom")
        return run(p, device)

    srv = serve.Server(hbm_bytes=10, prepare=prepare, run=flaky)
    res = srv.serve([serve.Request(13, 13, 1.0, rid=i) for i in range(3)], realtime=False)
    assert [r.status for r in res] == ["done", "error", "done"]
    assert "boom" in res[1].message


def test_poisson_stream_and_summary():
    reqs = serve.poisson_stream(200, 20.0, 7, [13, 21], [13, 21, 25])
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0) and 200 / t[-1] == pytest.approx(20.0, rel=0.2)
    assert all(r.walkers % 64 == 0 and 512 <= r.walkers <= 4096 for r in reqs)
    assert all((r.n_down == 0) or (r.n_up == r.n_down) for r in reqs)
    assert {r.method for r in reqs} == {"vmc", "dmc"}
    res = [serve.Result(i, "done", moves=10, t_arrival=0.0, t_done=float(i + 1))
           for i in range(100)]
    sm = serve.summary(res)
    assert sm["p50_s"] == pytest.approx(50.5) and sm["p99_s"] == pytest.approx(99.01)
    assert sm["walker_moves_per_s"] == pytest.approx(1000 / 100.0)


def test_requests_are_prepared_on_the_host_with_the_optimised_breakup(tmp_path):
    import importlib
    import os

    serve = importlib.import_module("2degas_b200.serve")
    small = serve.prepare_request(serve.Request(13, 13, 2.0, walkers=512, rid=0), str(tmp_path))
    large = serve.prepare_request(serve.Request(81, 81, 3.0, walkers=512, rid=1), str(tmp_path))
    assert 0 < small.footprint < large.footprint
    with open(os.path.join(small.directory, "s.v")) as fh:
        assert "fitpn" in fh.read().split("\n")[1002]
