"""Serving loop for state-point requests on one GPU.

A request names a state point (electrons per spin, r_s), a method (VMC or
DMC), a population size and a target error bar on the local energy (Ry per
electron). Requests arrive over time. Each is prepared on the host (its
spline tables and Ewald k-vectors written by `tables.make_run`, read back
as a qmc2d_system) and then waits until its device footprint
(`qmc2d_footprint`: walker records, move scratch, tables) fits the free
share of the HBM budget and a slot is free. Admission is first-fit in
arrival order: a request that does not fit yet does not hold back later,
smaller ones. Requests whose determinants live in HBM (more than
HBM_DETS_ABOVE orbitals in a spin) each fill the GPU and are bound by L2
latency; max_hbm_dets caps how many of them run at once, so that they do
not evict each other's matrices from L2, while smaller requests fill in.

An admitted request gets its own handle, hence its own CUDA stream, and its
own host thread. The library's calls release the interpreter lock, so the
kernels of all admitted requests are in flight together and overlap on the
GPU, and a request that arrives while others run starts as soon as memory
and a slot free up (continuous batching). Walkers stay resident in the
handle from the first block to the last. A request runs blocks of moves
until the error bar of its block averages (the reference's averages(3)
formula, `qmc2d_stats_*`) reaches the target, or until its block limit.

Each request's random streams come from its own seed (counter-based
Philox keyed by the seed, with counters that belong to the handle), so its
result does not depend on what else runs beside it.

The reference has no serving loop: it runs one state point per process.
"""
import math
import os
import tempfile
import threading
import time
from dataclasses import dataclass, field

import numpy as np


def closed_shells(nmax=200):
    """Electron counts per spin that fill plane-wave shells of the square
    cell: the number of integer vectors with |n|^2 <= m, for each m that is
    a sum of two squares."""
    out, m = [], 0
    while True:
        r = int(math.isqrt(m))
        cnt = sum(1 for a in range(-r, r + 1) for b in range(-r, r + 1) if a * a + b * b <= m)
        if cnt > nmax:
            return out
        if not out or cnt != out[-1]:
            out.append(cnt)
        m += 1


@dataclass
class Request:
    n_up: int
    n_down: int
    rs: float
    method: str = "dmc"          # "vmc" or "dmc"
    target: float = 1e-4         # error bar of E_L, Ry per electron
    walkers: int = 512
    seed: int = 1
    arrival: float = 0.0         # seconds after the stream starts
    backflow: bool = True
    precision: str = "fp64"      # "fp64" or "mixed" (qmc2d_set_precision)
    block_steps: int = 20
    min_blocks: int = 5
    max_blocks: int = 500
    equil_steps: int = 100
    tau: float = 0.0             # time step (Ry^-1); 0: chosen (see run_request)
    rid: int = -1

    @property
    def N(self):
        return self.n_up + self.n_down


@dataclass
class Result:
    rid: int
    status: str                  # "done", "max_blocks", "rejected" or "error"
    energy: float = float("nan")
    error: float = float("nan")
    blocks: int = 0
    moves: int = 0
    t_arrival: float = 0.0
    t_admit: float = float("nan")
    t_done: float = float("nan")
    footprint: int = 0
    message: str = ""
    block_means: list = field(default_factory=list)

    @property
    def latency(self):
        """Time to error bar: arrival to the end of the last block."""
        return self.t_done - self.t_arrival


class Prepared:
    """A request with its system on the host and its device footprint."""

    def __init__(self, req, system=None, footprint=0, directory=None):
        self.req, self.system, self.footprint, self.directory = req, system, footprint, directory


def prepare_request(req, workdir):
    """Tables and system of a request (host only) and its device footprint."""
    import importlib

    q = importlib.import_module("2degas_b200")
    tables = importlib.import_module("2degas_b200.tables")
    d = os.path.join(workdir, f"req{req.rid}")
    bf = (0.2, 1.0 * req.rs, 0.6 * req.rs) if req.backflow else None
    # the optimised Ewald breakup: the plain split at alpha = 5/L is off by
    # a few 1e-4 Ry per electron, more than the error bars served here
    tables.make_run(d, "s", req.n_up, req.n_down, req.rs, backflow=bf, ewald="fitpn")
    s = q.System.read(d, "s")
    return Prepared(req, s, s.footprint(req.walkers), d)


def run_request(p, device=0):
    """Run a prepared request to its error bar on its own handle; returns a
    dict with energy, error, blocks, moves, status and the block means."""
    import importlib

    q = importlib.import_module("2degas_b200")
    req, s = p.req, p.system
    L = s.s.el[0]
    rng = np.random.default_rng(req.seed)
    x0 = rng.uniform(-0.5 * L, 0.5 * L, size=(req.walkers, 2 * s.N))
    moves, means = 0, []
    with q.Handle(s, capacity=req.walkers, seed=req.seed, device=device) as h:
        h.set_precision(req.precision)
        h.population_set(x0)
        # Equilibration from uniform positions, in chunks of 10 VMC steps with
        # forced moves after 50 rejections (age, as the reference's mage):
        # the all-electron step is scaled after each chunk toward 50%
        # acceptance, which falls with N at a fixed step. At 0.05 r_s^2,
        # N = 50 accepted 5% of moves and one stuck walker held the DMC
        # population (the oracle shows the same).
        dv = 0.05 * req.rs * req.rs
        c0 = h.counters()
        for _ in range(max(1, req.equil_steps // 10)):
            h.vmc(10, dv, 50)
            moves += 10 * req.walkers
            c1 = h.counters()
            acc = (c1["accepted"] - c0["accepted"]) / max(c1["proposed"] - c0["proposed"], 1.0)
            c0 = c1
            dv *= min(2.0, max(0.3, acc / 0.5))
        # the pair kernel's walker groups and staging for this population; the
        # inversion layouts and the pair lanes agree only to round-off, and
        # the autotuner's pick depends on timing, which the mix changes: they
        # keep their defaults so a request's result does not depend on what
        # else runs (and are not timed)
        h.set_autotune_scope(1)
        h.autotune()
        # DMC at a tenth of the VMC step (acceptance near 97%)
        tau = req.tau or (dv / 10.0 if req.method == "dmc" else dv)
        if req.method == "dmc":
            # local-energy cutoff of the weights, 0.2 sqrt(N / tau) in total
            # energy (Umrigar, Nightingale and Runge, J. Chem. Phys. 99, 2865
            # (1993)); per electron 0.2 / sqrt(N tau)
            h.set_dmc_ecut(0.2 / np.sqrt(s.N * tau))
        etrial = None

        def median_el():
            # the trial energy from the population's median E_L: one outlier
            # in a block mean can put E_T below every walker's E_L, and then
            # every weight exp(-tau N (E_L - E_T)) underflows to zero
            return float(np.median(h.population_get()["p"][:, 0]))

        if req.method == "dmc":
            h.vmc(req.block_steps, dv, 50)
            moves += req.block_steps * req.walkers
            etrial = median_el()
        st = q.Stats(s)
        status, mean, err, nb = "max_blocks", float("nan"), float("nan"), 0
        for _ in range(req.max_blocks):
            h.block_reset()
            if req.method == "dmc":
                h.dmc(req.block_steps, 1, tau, etrial, 2.0, 50)
            else:
                h.vmc(req.block_steps, tau, 50)
            moves += req.block_steps * req.walkers
            blk, norm = h.block_get()
            if not (norm > 0.0 and np.isfinite(blk[0])):  # weights all underflowed: new E_T
                etrial = median_el()
                continue
            st.add_block(blk, norm)
            means.append(blk[0] / norm)
            m, e, _, nb = st.get()
            mean, err = float(m[0]), float(e[0])
            if req.method == "dmc":
                etrial = mean
            if nb >= req.min_blocks and err <= req.target:
                status = "done"
                break
    return dict(energy=mean, error=err, blocks=nb, moves=moves, status=status, block_means=means)


# Orbitals per spin above which the library keeps a walker's determinant
# matrices in HBM instead of shared memory (45 + 45 is the largest shell in
# shared memory).
HBM_DETS_ABOVE = 45


def hbm_dets(req):
    return max(req.n_up, req.n_down) > HBM_DETS_ABOVE


class Server:
    """Admits requests by HBM footprint and runs the admitted ones together.

    hbm_bytes: the device memory the server may hand out; max_slots: the
    most requests on the device at once; max_hbm_dets: the most of them with
    determinants in HBM (None: no cap; 1 by default: on a stream of 12
    requests from N = 50 to 149 two or more at once lengthened the makespan
    from 102 to 109-119 s and the median latency from 40 to 63-66 s). prepare(req, workdir) -> Prepared
    and run(prepared, device) -> dict are the host preparation and the
    device run (prepare_request and run_request unless replaced)."""

    def __init__(self, hbm_bytes, max_slots=32, device=0, workdir=None, prepare=None, run=None,
                 max_hbm_dets=1):
        self.hbm = int(hbm_bytes)
        self.max_slots = max_slots
        self.max_hbm_dets = max_hbm_dets
        self.active_hbm_dets = 0
        self.device = device
        self.workdir = workdir or tempfile.mkdtemp(prefix="qmc2d_serve_")
        self.prepare = prepare or prepare_request
        self.run_one = run or run_request
        self.cv = threading.Condition()
        self.used = 0
        self.active = 0
        self.peak_used = 0
        self.peak_active = 0

    def serve(self, requests, realtime=True):
        """Run a stream of requests (each with its arrival time, seconds
        after the start) to completion; returns their Results in rid order.
        realtime=False treats every request as arrived at the start."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for i, r in enumerate(reqs):
            if r.rid < 0:
                r.rid = i
        results = {}
        pending = []          # Prepared requests waiting for admission
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        workers, preps = [], []

        def finish(rid, res):
            with self.cv:
                results[rid] = res
                self.cv.notify_all()

        def prep(r):
            t_arr = now() if realtime else 0.0
            try:
                p = self.prepare(r, self.workdir)
            except Exception as e:  # a reader or table failure rejects the request
                finish(r.rid, Result(r.rid, "rejected", t_arrival=t_arr, t_done=now(),
                                     message=str(e)))
                return
            p.t_arrival = t_arr
            with self.cv:
                if p.footprint > self.hbm:
                    results[r.rid] = Result(r.rid, "rejected", t_arrival=t_arr, t_done=now(),
                                            footprint=p.footprint,
                                            message="footprint above the HBM budget")
                else:
                    pending.append(p)
                self.cv.notify_all()

        def arrivals():
            for r in reqs:
                if realtime:
                    dt = r.arrival - now()
                    if dt > 0:
                        time.sleep(dt)
                th = threading.Thread(target=prep, args=(r,), daemon=True)
                th.start()
                preps.append(th)

        def work(p):
            r = p.req
            res = Result(r.rid, "error", t_arrival=p.t_arrival, t_admit=now(),
                         footprint=p.footprint)
            try:
                out = self.run_one(p, self.device)
                res.status = out["status"]
                res.energy, res.error = out["energy"], out["error"]
                res.blocks, res.moves = out["blocks"], out["moves"]
                res.block_means = out.get("block_means", [])
            except Exception as e:  # a library status ends this request only
                # QMC2D_ERR_LIMIT (10): a state point beyond the kernels' limits
                res.status = "rejected" if getattr(e, "code", None) == 10 else "error"
                res.message = str(e)
            res.t_done = now()
            with self.cv:
                self.used -= p.footprint
                self.active -= 1
                self.active_hbm_dets -= int(hbm_dets(r))
                results[r.rid] = res
                self.cv.notify_all()

        arr = threading.Thread(target=arrivals, daemon=True)
        arr.start()
        with self.cv:
            while len(results) < len(reqs):
                admitted = True
                while admitted:
                    admitted = False
                    for p in sorted(pending, key=lambda p: p.t_arrival):  # first fit
                        big = hbm_dets(p.req)
                        if big and self.max_hbm_dets is not None and \
                                self.active_hbm_dets >= self.max_hbm_dets:
                            continue
                        if self.active < self.max_slots and self.used + p.footprint <= self.hbm:
                            pending.remove(p)
                            self.used += p.footprint
                            self.active += 1
                            self.active_hbm_dets += int(big)
                            self.peak_used = max(self.peak_used, self.used)
                            self.peak_active = max(self.peak_active, self.active)
                            th = threading.Thread(target=work, args=(p,), daemon=True)
                            th.start()
                            workers.append(th)
                            admitted = True
                self.cv.wait(timeout=0.5)
        arr.join()
        for th in preps + workers:
            th.join()
        return [results[r.rid] for r in sorted(reqs, key=lambda r: r.rid)]


def poisson_stream(n, rate, seed, shells_unpol, shells_pol, walkers=(512, 4096), rs=(1.0, 40.0),
                   target=1e-4, **kw):
    """n requests with exponential inter-arrival times (mean 1/rate s),
    polarisation 0 or 1, a closed shell of that polarisation, r_s uniform,
    VMC or DMC, and a population uniform in `walkers` (multiples of 64)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        pol = int(rng.integers(0, 2))
        if pol:
            nu, nd = int(rng.choice(shells_pol)), 0
        else:
            h = int(rng.choice(shells_unpol))
            nu, nd = h, h
        w = int(rng.integers(walkers[0] // 64, walkers[1] // 64 + 1)) * 64
        out.append(Request(nu, nd, float(rng.uniform(*rs)), method=("vmc", "dmc")[int(rng.integers(0, 2))],
                           target=target, walkers=w, seed=int(rng.integers(1, 2 ** 62)),
                           arrival=t, rid=i, **kw))
    return out


def summary(results, makespan=None):
    """p50/p99 time to error bar over the requests that finished, the
    aggregate walker-moves/s, and the counts by status."""
    ok = [r for r in results if r.status in ("done", "max_blocks")]
    lat = np.array([r.latency for r in ok]) if ok else np.array([float("nan")])
    moves = sum(r.moves for r in ok)
    if makespan is None:
        t_first = min((r.t_arrival for r in results), default=0.0)
        t_last = max((r.t_done for r in ok), default=t_first)
        makespan = max(t_last - t_first, 1e-9)
    by = {}
    for r in results:
        by[r.status] = by.get(r.status, 0) + 1
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "walker_moves_per_s": moves / makespan, "moves": moves, "makespan_s": makespan,
            "status": by}
