#!/usr/bin/env python
"""Walker-moves/s of the walker-propagation path on B200.

Workload (default): DMC with backflow, N = 58 (29 up + 29 down) at r_s = 5,
4096 walkers, time step tau = 0.05 r_s^2, one move per generation followed
by branch2's fixed-population comb, Jastrow u2 + backflow
eta(r) = 0.2 exp(-((r - r_s)/0.6 r_s)^2) + 2D Ewald (alpha = 5/L, 60
half-space k vectors), FP64. Synthetic: tables written by
2degas_b200/tables.py and walkers drawn uniformly in the cell from a seeded
Philox stream, then equilibrated by VMC.

One step = one DMC generation over the whole population (4096
walker-moves: pairs_kernel, move_kernel, branch, gather). `value` times the device work with CUDA events on the
library's stream (inputs resident in HBM, L2 flushed between steps);
`e2e` times the same steps through the public C-ABI with the walker records
copied from and to pinned host memory every step (qmc2d_population_load_async:
the records other than x and g arrive while the pair kernel runs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Other workloads (not the headline line): --shell NU,ND [--rs R] runs the
same DMC generation on another closed shell (up to 81 + 81 or 161
polarised); --workload batch times 64 uneven populations through
qmc2d_batch_dmc (--batch-lanes sweeps the populations in flight);
--workload serve runs the serving stream; --phases prints the move
kernel's per-phase SM cycles instead of timing.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import importlib  # noqa: E402

import numpy as np  # noqa: E402

CONFIG = "dmc_bf_n58_rs5"
METRIC = "walker-moves/sec (DMC with backflow, N=58 r_s=5, 4096 walkers)"
UNIT = "walker-moves/s"
# DRAM bytes read per walker by one pairs_kernel + orb_inv_kernel +
# move_kernel generation, from the ncu capture summarised in
# profiles/move_kernels_dmc_bf_n58_444w.md (444 walkers, one wave of the
# move kernel; scaled linearly: the walker records and the move scratch,
# read cold in ncu's replays), plus the move scratch block the pair and
# orbital kernels write, which reaches DRAM at 4096 walkers (the blocks
# exceed L2) though not in the 444-walker capture.
MOVE_DRAM_READ_PER_WALKER = (1.114624e6 + 0.526080e6 + 49.427200e6) / 444
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum of pairs_kernel + orb_inv_kernel + move_kernel "
                  "(444 walkers) x walkers/444, + the move scratch written per walker")


def move_scratch_bytes(N, nk, ns=()):
    """Bytes of one walker's move scratch block (MoveScratch, backflow; with
    ns, the spins' orbital counts, the orbitals-and-inversion region when
    every spin has at most 32 orbitals)."""
    pair = (14 * N + 3 + 4 * max(nk, 1) + 3) & ~3
    end = pair + 3 * (N * (N - 1) // 2)
    if ns and max(ns) <= 32:
        end = (end + 1) & ~1
        end += sum((2 * n * n + 2 * n * (n | 1) + 2 * n + 2 + 1) & ~1 for n in ns)
    return 8 * ((end + 31) & ~31)


def flops_per_sweep(N, ns, K):
    """Algorithmic flops of one sweep of single-electron moves (N moves on a
    plain Slater-Jastrow deck, then one measurement; transcendental = 1):
    per move of an electron whose spin has n orbitals, the orbitals, ratio
    and gradient at the old and new positions (2 x 13 n), the two-body
    Jastrow at both (2 x 30 (N - 1)) and the Sherman-Morrison update (16 n^2);
    the measurement's pair sums (60 per pair), rho_k (7 N K) and the
    determinant drift and Laplacian (25 n^2 per spin)."""
    f = 0
    for n in ns:
        f += n * (26 * n + 60 * (N - 1) + 16 * n * n) + 25 * n * n
    return float(f + 60 * N * (N - 1) // 2 + 7 * N * K)


def flops_per_move(N, ns, K, u3, backflow):
    """Algorithmic flops of one all-electron walker-move (proposal + evaluation
    + accept/reject) of the reference's algorithm, counted from its loop
    structure: pairs P = N(N-1)/2 cost 16 (distance) + 32 (u2) + 12
    (potential) + 110 (u3) + 80 (backflow) flops, rho_k costs 7 per
    (particle, k), and per spin determinant of n electrons
    backflow: 53 n^2 + 24 n^3 + 40 N n^2 + 44 N n (orbitals, complex LU and
    inverse, A^-1 dA, drift, Laplacian with the O(N n^2) cross term);
    no backflow: 45 n^2 + 8 n^3."""
    P = N * (N - 1) // 2
    f = P * (16 + 32 + 12 + 110 * u3 + 80 * backflow) + 7 * N * K
    for n in ns:
        if backflow:
            f += 53 * n * n + 24 * n ** 3 + 40 * N * n * n + 44 * N * n
        else:
            f += 45 * n * n + 8 * n ** 3
    return float(f)


def make_config(tmp, nconf, seed, shell=None, rs=None):
    """The headline deck, or with shell = (n_up, n_down) and rs another
    closed shell and density with the same Jastrow and backflow forms.
    Returns (directory, config, workload name)."""
    tables = importlib.import_module("2degas_b200.tables")
    cfg, name = dict(tables.CONFIGS[CONFIG]), CONFIG
    if shell is not None:
        r = rs if rs is not None else cfg["rs"]
        cfg.update(n_up=shell[0], n_down=shell[1], rs=r, backflow=(0.2, r, 0.6 * r))
        name = f"dmc_bf_n{shell[0] + shell[1]}{'p' if shell[1] == 0 else ''}_rs{r:g}"
    d = tables.make_run(os.path.join(tmp, name), "c", nconf=nconf, seed=seed, **cfg)
    return d, cfg, name


# ------------------------------------------------------------ CPU baseline
def _cpu_worker(args):
    """One host process: the oracle's DMC on its own sub-population for
    `seconds` of wall time; returns walker-moves done and seconds."""
    d, nw, seed, seconds, delta, etrial = args
    from oracle_lib import Oracle, OracleSystem

    # the oracle reads the deck itself: this process loads only liboracle.so
    s = OracleSystem.read(d, "c")
    x = s.read_configs(d, ".0", 0, nw)
    o = Oracle(s)
    pop = o.population_init(x)
    o.vmc_philox(pop, 2, delta, 10 ** 9, seed, 0)
    t0 = time.perf_counter()
    moves, gen = 0, 0
    while time.perf_counter() - t0 < seconds:
        o.dmc_philox(pop, 1, 1, delta, etrial, 2.0, 50, seed, gen, 1000 + gen)
        moves += nw
        gen += 1
    return moves, time.perf_counter() - t0


def cpu_rate(d, seconds, walkers_per_proc=8, rs=None):
    """Oracle DMC on every host core (one process per core, spawn)."""
    import multiprocessing as mp

    try:
        ncores = len(os.sched_getaffinity(0))
    except AttributeError:
        ncores = os.cpu_count() or 1
    if rs is None:
        rs = importlib.import_module("2degas_b200.tables").CONFIGS[CONFIG]["rs"]
    delta = 0.05 * rs ** 2
    ctx = mp.get_context("spawn")
    with ctx.Pool(ncores) as pool:
        res = pool.map(_cpu_worker, [(d, walkers_per_proc, 100 + i, seconds, delta, -0.3)
                                     for i in range(ncores)])
    moves = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    sample = (f"{ncores} processes x {walkers_per_proc} walkers, oracle DMC generations "
              f"for {seconds:.0f} s each ({moves} walker-moves)")
    return moves / wall, ncores, sample


# ------------------------------------------------------------------ clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(torch):
    """Measured FP64 throughput of a cuBLAS DGEMM on this GPU (TFLOP/s)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


# ------------------------------------------------------- multi-rank logic
def rank_seeds(rank):
    """(configuration seed, walker-stream seed) of a rank: every rank runs its
    own independent population (weak scaling, no data-path collective)."""
    return 1 + rank, 0x9E3779B97F4A7C15 + rank


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest `value` over all ranks (timings are the slowest rank's)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, walkers_per_rank, steps, seconds):
    """Walker-moves per second of the whole job: every rank's walker-moves
    over the slowest rank's time."""
    return world * walkers_per_rank * steps / seconds


# ------------------------------------------------------------------- arms
def workload_desc(args, world):
    """(metric, config) of the workload `args` selects; the same for the
    device arm and the reference arm, computed without a GPU."""
    tables = importlib.import_module("2degas_b200.tables")
    common = {"l2": "flushed between timed steps (256 MiB write)",
              "parallelism": f"independent populations x{world}"}
    if args.workload == "vmc":
        rs = tables.CONFIGS[VMC_CONFIG]["rs"]
        nw = args.walkers if args.walkers != 4096 else 256
        if args.single:
            metric = (f"walker-moves/sec (VMC, N=26 r_s={rs:g}, {nw} walkers; single-electron "
                      f"moves, one sweep of N moves = one walker-move, {SINGLE_SWEEPS} sweeps "
                      f"per step)")
        else:
            metric = f"walker-moves/sec (VMC, N=26 r_s={rs:g}, {nw} walkers)"
        cfg = {"workload": VMC_CONFIG, "walkers_per_gpu": nw, "N": 26, "rs": rs,
               "tau": 0.045 * rs * rs,
               "moves_per_step": nw * world * (SINGLE_SWEEPS if args.single else 1),
               "moves": "single-electron sweeps, inverse recomputed every 50 moves"
               if args.single else "all-electron"}
    elif args.workload == "rmc":
        name = "rmc_n26_rs10" if args.rmc_n == 26 else RMC_CONFIG
        rs = tables.CONFIGS[name]["rs"]
        nw = args.walkers if args.walkers != 4096 else 512
        metric = (f"walker-moves/sec (reptation, N={args.rmc_n} r_s={rs:g}, {nw} reptiles x "
                  f"200 beads, one bead growth = one walker-move)")
        cfg = {"workload": name, "walkers_per_gpu": nw, "N": args.rmc_n, "rs": rs,
               "tau": 0.01 * rs * rs, "beads": 200, "mdelta": 1, "moves_per_step": nw * world}
    else:
        if args.shell is None:
            metric, name, N, rs = METRIC, CONFIG, 58, 5.0
        else:
            rs = args.rs if args.rs is not None else 5.0
            N = sum(args.shell)
            name = f"dmc_bf_n{N}{'p' if args.shell[1] == 0 else ''}_rs{rs:g}"
            metric = (f"walker-moves/sec (DMC with backflow, N={N}"
                      f"{' polarised' if args.shell[1] == 0 else ''} r_s={rs:g}, "
                      f"{args.walkers} walkers)")
        cfg = {"workload": name, "walkers_per_gpu": args.walkers, "N": N, "rs": rs,
               "precision": args.precision, "tau": 0.05 * rs * rs, "mmstep": 1,
               "moves_per_step": args.walkers * world}
        if args.global_comb:
            common["parallelism"] = f"one population over {world} ranks (global comb)"
    cfg.update(common)
    return metric, cfg


def reference_arm(args, rank, world):
    """The reference's algorithm on the host cores (the oracle, which restates
    it; the Fortran reference cannot be built here) for the same workload,
    metric and config as the device arm."""
    if rank != 0:
        return 0
    metric, config = workload_desc(args, world)
    secs = max(4.0, min(20.0, 0.4 * (args.steps + args.warmup)))
    with tempfile.TemporaryDirectory() as tmp:
        if args.workload in ("vmc", "rmc"):
            tables = importlib.import_module("2degas_b200.tables")
            cfg = tables.CONFIGS[config["workload"]]
            d = tables.make_run(os.path.join(tmp, "c"), "c", nconf=64, seed=1, **cfg)
            rate, cores, sample = config_cpu_baseline(args.workload, d, cfg, secs)
        else:
            d, _, _ = make_config(tmp, 64, 1, args.shell, args.rs)
            rate, cores, sample = cpu_rate(d, secs, rs=config["rs"])
    line = {
        "impl": "reference", "metric": metric, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def b200_arm(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    q = importlib.import_module("2degas_b200")
    capi = q._capi
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    nw = args.walkers
    tmp = tempfile.mkdtemp(prefix="qmc2d_bench_")
    cfg_seed, walker_seed = rank_seeds(rank)
    d, cfg, workload = make_config(tmp, nw, cfg_seed, args.shell, args.rs)
    headline = workload == CONFIG
    sysobj = q.System.read(d, "c")
    N = sysobj.N
    ns = [sysobj.s.np[t] for t in range(sysobj.ntypes)]
    rs = cfg["rs"]
    delta = 0.05 * rs * rs
    x0 = sysobj.read_configs(d, ".0", 0, nw)
    h = q.Handle(sysobj, capacity=nw, seed=walker_seed, device=local_rank)
    h.set_precision(args.precision)
    h.population_set(x0)
    h.vmc(args.equil, delta, 10 ** 9)  # seeded VMC equilibration
    tuned = h.autotune()  # launch choices, timed on this population
    if args.inversion is not None:  # a fixed inversion layout instead of the tuner's
        h.set_inversion(args.inversion)
    if args.pair_lanes is not None:  # fixed lanes per particle instead of the tuner's
        h.set_pair_lanes(args.pair_lanes)
    if args.move_inversion is not None:  # orbitals and inversion in their own kernel or not
        h.set_move_inversion(args.move_inversion)
    h.block_reset()
    h.vmc(10, delta, 10 ** 9)
    blk, norm = h.block_get()
    etrial = blk[0] / norm
    mmult, mage = 2.0, 50
    stream = torch.cuda.ExternalStream(h.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    if args.global_comb:
        # one population over all ranks: branch2's comb and walker exchange
        # every generation (2degas_b200/multirank.py)
        mr = importlib.import_module("2degas_b200.multirank")
        pop = mr.HandleRecords(h, torch.device("cuda", local_rank))
        gen = [0]

        def step():
            mr.dmc_generations(pop, dist, 1, 1, delta, etrial, mmult, mage, 0x5EEDC0B1,
                               gen0=gen[0], device=f"cuda:{local_rank}")
            gen[0] += 1
    else:
        def step():
            h.dmc(1, 1, delta, etrial, mmult, mage)

    if args.phases:
        # SM cycles per walker-move of each phase of the move kernel (clock64
        # deltas of thread 0 of every CTA, summed over CTAs), no timing
        for _ in range(args.warmup):
            step()
        h.phase_timers(True)
        for _ in range(args.steps):
            step()
        ph = h.phase_timers(False)
        moves = nw * args.steps
        tot = sum(ph.values())
        if rank == 0:
            print(json.dumps({"phases_cycles_per_move": {k: v / moves for k, v in ph.items() if v},
                              "share": {k: v / tot for k, v in ph.items() if v},
                              "workload": workload, "walkers": nw, "steps": args.steps}),
                  flush=True)
        h.close()
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    h.profile(True)
    h.block_reset()
    acc0 = h.counters()
    dev_ms = 0.0
    with Clocks(local_rank) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    acc = h.counters()
    move_ms, move_n = h.profile_get(capi.KERNEL_MOVE)
    pair_ms, pair_n = h.profile_get(capi.KERNEL_PAIRS)
    br_ms, br_n = h.profile_get(capi.KERNEL_BRANCH)
    ga_ms, ga_n = h.profile_get(capi.KERNEL_GATHER)
    oi_ms, oi_n = h.profile_get(capi.KERNEL_ORB_INV)
    h.profile(False)
    blk, norm = h.block_get()
    e_mean = blk[0] / norm
    t_max = max_over_ranks(dev_ms, dist, "cuda")
    value = whole_job_rate(world, nw, args.steps, t_max * 1e-3)

    # e2e: walker records from/to pinned host memory every step, public API
    nt, npr = sysobj.ntypes, sysobj.nprops
    pin = {k: torch.empty(n, dtype=torch.float64, pin_memory=True)
           for k, n in (("x", nw * 2 * N), ("g", nw * 2 * N), ("h", nw * nt), ("p", nw * npr),
                        ("s", nw), ("a", nw))}
    ptr = {k: v.data_ptr() for k, v in pin.items()}
    h.population_get_ptr(ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"], ptr["a"])
    h2d = sum(v.numel() * 8 for v in pin.values())
    d2h = h2d + npr * 8 + 8  # records back + block sums
    k2 = max(3, args.steps // 2)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k2):
        # x and g on the library stream, the other records behind the pair kernel
        h.population_load_async_ptr(nw, ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"],
                                    ptr["a"])
        step()
        h.population_get_ptr(ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"], ptr["a"])
        h.block_get()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e = whole_job_rate(world, nw, k2, e2e_s)

    line = None
    if rank == 0:
        K = sysobj.s.nk
        fpm = flops_per_move(N, ns, K, 0, 1)
        # one walker-move of the population = one pairs_kernel, one
        # orb_inv_kernel (where it applies) and one move_kernel launch; the
        # roofline covers them all
        achieved = fpm * nw / ((move_ms + pair_ms + oi_ms) / max(move_n, 1) * 1e-3) / 1e12
        peak = fp64_peak_tflops(torch)
        cpu = None
        if world == 1 and not args.no_cpu:
            rate, cores, sample = cpu_rate(d, args.cpu_seconds, rs=rs)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
        launches = pair_n + oi_n + move_n + br_n + ga_n
        metric, config = workload_desc(args, world)
        line = {
            "metric": metric,
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64 (f32 u2 and v2 pair terms)",
            "data": "synthetic",
            "config": config,
            "pair_launch": {"groups": tuned[0], "stage_rows": tuned[1] == 0,
                            "lanes_per_particle": h.get_pair_lanes(),
                            "inversion_layout": h.get_launch()[2]},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": ((MOVE_DRAM_READ_PER_WALKER + move_scratch_bytes(N, K, ns)) * nw
                                     if headline else None),
                         "traffic_source": TRAFFIC_SOURCE if headline else None,
                         "kernel": ("pairs_kernel + orb_inv_kernel + move_kernel" if oi_n
                                    else "pairs_kernel + move_kernel"),
                         "flops_per_move": fpm,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64)"},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "kernel_ms": {"pairs": pair_ms, "orb_inv": oi_ms, "move": move_ms, "branch": br_ms,
                          "gather": ga_ms},
            "wall_s": wall,
            "e_mixed": e_mean,
            "acceptance": (acc["accepted"] - acc0["accepted"]) /
                          max(acc["proposed"] - acc0["proposed"], 1),  # timed generations
            "clocks": clk.summary(),
        }
    if dist:
        dist.barrier()
    h.close()
    if dist:
        dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------ configs 0 and 2 (VMC, RQMC)
VMC_CONFIG, RMC_CONFIG = "vmc_n26_rs1", "rmc_n58_rs10"
# sweeps per call of the single-electron workload: the inverse stays resident
# within a call, and each call starts from a fresh one
SINGLE_SWEEPS = 10


def _vmc_cpu_worker(args):
    """Oracle VMC steps on `nw` walkers for `seconds` (one host process)."""
    d, nw, seed, seconds, delta = args
    from oracle_lib import Oracle, OracleSystem

    s = OracleSystem.read(d, "c")
    o = Oracle(s)
    pop = o.population_init(s.read_configs(d, ".0", 0, nw))
    t0 = time.perf_counter()
    moves, stp = 0, 0
    while time.perf_counter() - t0 < seconds:
        o.vmc_philox(pop, 1, delta, 10 ** 9, seed, stp)
        moves += nw
        stp += 1
    return moves, time.perf_counter() - t0


def _rmc_cpu_worker(args):
    """Oracle reptation moves of one reptile for `seconds` (one host
    process); the path set-up (ntau evaluations) is not timed."""
    d, ntau, seed, seconds, delta, etrial, mage_r, rs = args
    from oracle_lib import Oracle, OracleSystem, Reptile

    capi = importlib.import_module("2degas_b200._capi")
    s = OracleSystem.read(d, "c")
    o = Oracle(s)
    x = rmc_start_paths(s.read_configs(d, ".0", 0, 1), ntau, delta, rs, seed)
    rep = Reptile(o, capi.RmcParams(ntau, 1, 1, delta, etrial, 10 ** 9, mage_r))
    rep.init(x)
    t0 = time.perf_counter()
    moves = 0
    while time.perf_counter() - t0 < seconds:
        rep.run(seed, seed, moves, 1)
        moves += 1
    return moves, time.perf_counter() - t0


def cpu_pool_rate(worker, argsets):
    """Run `worker` on every host core (spawned processes); returns
    (walker-moves/s, cores, total moves)."""
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(len(argsets)) as pool:
        res = pool.map(worker, argsets)
    moves = sum(r[0] for r in res)
    return moves / max(r[1] for r in res), len(argsets), moves


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def rmc_start_paths(x0, ntau, delta, rs, seed):
    """Reptiles as random walks of ntau beads from the configurations x0,
    with the propagator's link variance 2 hbs2m delta = 2 delta / r_s^2."""
    rng = np.random.default_rng(seed)
    var = 2.0 * delta / rs ** 2
    st = rng.normal(0.0, math.sqrt(var), size=(x0.shape[0], ntau, x0.shape[1]))
    st[:, 0] = 0.0
    return (x0[:, None, :] + np.cumsum(st, axis=1)).reshape(x0.shape[0] * ntau, -1)


def config_cpu_baseline(kind, d, cfg, seconds):
    """The oracle on every host core for a bounded sample of the workload."""
    rs = cfg["rs"]
    n = host_cores()
    if kind == "vmc":
        delta = 0.045 * rs * rs
        rate, cores, moves = cpu_pool_rate(
            _vmc_cpu_worker, [(d, 8, 300 + i, seconds, delta) for i in range(n)])
        sample = (f"{cores} processes x 8 walkers, oracle VMC steps for {seconds:.0f} s each "
                  f"({moves} walker-moves)")
    else:
        delta = 0.01 * rs * rs
        rate, cores, moves = cpu_pool_rate(
            _rmc_cpu_worker, [(d, 200, 500 + i, seconds, delta, -0.27, 50, rs)
                              for i in range(n)])
        sample = (f"{cores} processes x 1 reptile of 200 beads, oracle reptation moves "
                  f"(mdelta 1) for {seconds:.0f} s each ({moves} bead growths)")
    return rate, cores, sample


def config_arm(args, rank, world, local_rank):
    """The plain-VMC workload (--workload vmc: N = 26 r_s = 1,
    256 walkers, Gaussian step 0.3 r_s) or the reptation one (--workload rmc: reptation,
    N = 58 r_s = 10 with u2 + u3 + backflow, 512 reptiles of 200 beads,
    one-bead head moves, tau = 0.01 r_s^2; --rmc-n 26 for the N = 26 deck).
    One step = one VMC step of every walker, or one reptation move of every
    reptile (one bead growth each = one walker-move)."""
    import torch

    torch.cuda.set_device(local_rank)
    q = importlib.import_module("2degas_b200")
    tables = importlib.import_module("2degas_b200.tables")
    capi = q._capi
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    vmc = args.workload == "vmc"
    name = VMC_CONFIG if vmc else ("rmc_n26_rs10" if args.rmc_n == 26 else RMC_CONFIG)
    cfg = tables.CONFIGS[name]
    rs = cfg["rs"]
    nw = args.walkers if args.walkers != 4096 else (256 if vmc else 512)
    ntau = 200
    cfg_seed, walker_seed = rank_seeds(rank)
    tmp = tempfile.mkdtemp(prefix="qmc2d_bench_")
    d = tables.make_run(os.path.join(tmp, name), "c", nconf=nw, seed=cfg_seed, **cfg)
    sysobj = q.System.read(d, "c")
    N, nt, npr = sysobj.N, sysobj.ntypes, sysobj.nprops
    ns = [sysobj.s.np[t] for t in range(nt)]
    x0 = sysobj.read_configs(d, ".0", 0, nw)
    nw_moves = 1  # walker-moves per walker in one step
    if vmc and args.single:
        delta = 0.045 * rs * rs
        h = q.Handle(sysobj, capacity=nw, seed=walker_seed, device=local_rank)
        h.population_set(x0)
        h.vmc_single(args.equil, delta, 50)
        tuned = None

        def step():
            h.vmc_single(SINGLE_SWEEPS, delta, 50)
        kernels = (capi.KERNEL_SINGLE,)
        nw_moves = SINGLE_SWEEPS
    elif vmc:
        delta = 0.045 * rs * rs
        h = q.Handle(sysobj, capacity=nw, seed=walker_seed, device=local_rank)
        h.population_set(x0)
        h.vmc(args.equil, delta, 10 ** 9)
        tuned = h.autotune()
        if args.move_inversion is not None:
            h.set_move_inversion(args.move_inversion)

        def step():
            h.vmc(1, delta, 10 ** 9)
        kernels = (capi.KERNEL_PAIRS, capi.KERNEL_ORB_INV, capi.KERNEL_MOVE)
    else:
        delta, etrial, mage_r = 0.01 * rs * rs, -0.27, 50
        h = q.Handle(sysobj, capacity=nw, seed=walker_seed, device=local_rank)
        h.population_set(x0)
        h.vmc(args.equil, 0.045 * rs * rs, 10 ** 9)  # seeded VMC start configurations
        x1 = h.population_get()["x"]
        # the pair kernel's launch choices (groups, staging, lanes), timed on
        # the start configurations; the reptation pair kernel uses them too
        h.autotune()
        if args.pair_lanes is not None:
            h.set_pair_lanes(args.pair_lanes)
        if args.rmc_split is not None:
            h.rmc_set_launch(args.rmc_split)
        h.rmc_init(nw, rmc_start_paths(x1, ntau, delta, rs, walker_seed & 0xFFFF), ntau, 1, 1,
                   delta, etrial, 10 ** 9, mage_r)
        tuned = h.get_launch()

        def step():
            h.rmc(1)
        kernels = (capi.KERNEL_PAIRS, capi.KERNEL_RMC)
    stream = torch.cuda.ExternalStream(h.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if args.phases:
        # SM cycles per walker-move of each phase (thread 0 of every CTA)
        h.phase_timers(True)
        for _ in range(args.steps):
            step()
        ph = h.phase_timers(False)
        tot = sum(ph.values())
        print(json.dumps({"phases_cycles_per_move": {k: v / (nw * args.steps)
                                                     for k, v in ph.items() if v},
                          "share": {k: v / tot for k, v in ph.items() if v},
                          "workload": name, "walkers": nw, "steps": args.steps}), flush=True)
        h.close()
        return 0
    if dist:
        dist.barrier()
    h.profile(True)
    h.block_reset()
    dev_ms = 0.0
    with Clocks(local_rank) as clk:
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
        torch.cuda.synchronize()
    kms = {k: h.profile_get(k) for k in kernels}
    h.profile(False)
    blk, norm = h.block_get()
    acc = h.counters()
    t_max = max_over_ranks(dev_ms, dist, "cuda")
    value = whole_job_rate(world, nw * nw_moves, args.steps, t_max * 1e-3)

    # e2e through the public C-ABI with pinned host buffers every step
    k2 = max(3, args.steps // 2)
    if vmc:
        pin = {k: torch.empty(n, dtype=torch.float64, pin_memory=True)
               for k, n in (("x", nw * 2 * N), ("g", nw * 2 * N), ("h", nw * nt),
                            ("p", nw * npr), ("s", nw), ("a", nw))}
        ptr = {k: v.data_ptr() for k, v in pin.items()}
        h.population_get_ptr(ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"], ptr["a"])
        h2d = sum(v.numel() * 8 for v in pin.values())
        d2h = h2d + npr * 8 + 8

        def e2e_step():
            h.population_load_async_ptr(nw, ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"],
                                        ptr["a"])
            step()
            h.population_get_ptr(ptr["x"], ptr["g"], ptr["h"], ptr["p"], ptr["s"], ptr["a"])
            h.block_get()
    else:
        # reptiles stay resident (the reference keeps its path in COMMON);
        # each step the host reads the block sums back
        h2d, d2h = 0, npr * 8 + 8

        def e2e_step():
            step()
            h.block_get()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k2):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e = whole_job_rate(world, nw * nw_moves, k2, e2e_s)

    line = None
    if rank == 0:
        K = sysobj.s.nk
        # config 0's deck carries an eta = 0 backflow table (the reference
        # builds its determinant only in the backflow routine): counted as
        # the plain Slater-Jastrow algorithm it is
        fpm = (flops_per_sweep(N, ns, K) if vmc and args.single else
               flops_per_move(N, ns, K, 0 if vmc else 1, 0 if vmc else 1))
        kern_ms = sum(kms[k][0] for k in kernels)
        n_launch = max(kms[kernels[-1]][1], 1)
        achieved = fpm * nw * nw_moves / (kern_ms / n_launch * 1e-3) / 1e12
        peak = fp64_peak_tflops(torch)
        cpu = None
        if world == 1 and not args.no_cpu:
            rate, cores, sample = config_cpu_baseline(args.workload, d, cfg, args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
        metric, config = workload_desc(args, world)
        line = {
            "metric": metric,
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config,
            "pair_launch": ({"groups": tuned[0], "stage_rows": tuned[1] == 0,
                             "lanes_per_particle": h.get_pair_lanes()} if tuned else None),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "kernel": ("single_kernel" if vmc and args.single else
                                    "pairs_kernel + move_kernel" if vmc else
                                    "rmc_pairs_kernel + rmc_det_kernel"),
                         "flops_per_move": fpm,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64)"},
            "cpu_baseline": cpu,
            "gpu_launches": sum(kms[k][1] for k in kernels),
            "kernel_ms": {str(k): kms[k][0] for k in kernels},
            "acceptance": acc["accepted"] / max(acc["proposed"], 1),
            "e_mean": blk[0] / norm,
            "clocks": clk.summary(),
        }
    if dist:
        dist.barrier()
    h.close()
    if dist:
        dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)
    return 0


def _serve_cpu_worker(args):
    """Oracle moves of one request's state point (VMC steps or DMC
    generations of `nw` walkers) for `seconds`; returns (moves, seconds)."""
    d, method, nw, seed, seconds, delta = args
    from oracle_lib import Oracle, OracleSystem

    s = OracleSystem.read(d, "s")
    o = Oracle(s)
    rng = np.random.default_rng(seed)
    el = math.sqrt(s.N * math.pi)
    pop = o.population_init(rng.uniform(-0.5 * el, 0.5 * el, size=(nw, 2 * s.N)))
    t0 = time.perf_counter()
    moves, k = 0, 0
    while time.perf_counter() - t0 < seconds:
        if method == "dmc":
            o.dmc_philox(pop, 1, 1, delta, -0.3, 2.0, 50, seed, k, k)
        else:
            o.vmc_philox(pop, 1, delta, 50, seed, k)
        moves += nw
        k += 1
    return moves, time.perf_counter() - t0


def serve_cpu_baseline(reqs, results, seconds, max_requests=6):
    """The reference's algorithm (the oracle) on every host core for the first
    requests of the stream: each request's deck, its method, a bounded time.
    The rate is the CPU time those requests' served walker-moves would take:
    sum of moves / sum of (moves / per-request CPU rate)."""
    import multiprocessing as mp

    tables = importlib.import_module("2degas_b200.tables")
    n = host_cores()
    sample = [(r, res) for r, res in zip(reqs, results) if res.status != "rejected"]
    sample = sample[:max_requests]
    if not sample:
        return None
    per = max(2.0, seconds / len(sample))
    tot_moves, tot_time, rows = 0.0, 0.0, []
    with tempfile.TemporaryDirectory() as tmp, mp.get_context("spawn").Pool(n) as pool:
        for r, res in sample:
            d = os.path.join(tmp, f"req{r.rid}")
            bf = (0.2, 1.0 * r.rs, 0.6 * r.rs) if r.backflow else None
            tables.make_run(d, "s", r.n_up, r.n_down, r.rs, backflow=bf, ewald="fitpn")
            out = pool.map(_serve_cpu_worker, [(d, r.method, 2, 900 + i, per, 0.05 * r.rs ** 2)
                                               for i in range(n)])
            rate = sum(o[0] for o in out) / max(o[1] for o in out)
            m = max(res.moves, 1)
            tot_moves += m
            tot_time += m / rate
            rows.append({"rid": r.rid, "N": r.N, "method": r.method, "cpu_moves_per_s": rate})
    return {"value": tot_moves / tot_time, "unit": UNIT, "cores": n, "kind": "port",
            "sample": (f"first {len(sample)} requests of the stream, oracle "
                       f"VMC/DMC on {n} processes x 2 walkers for {per:.0f} s each, weighted by "
                       f"each request's served walker-moves"),
            "per_request": rows}


def precision_arm(args, rank, world, local_rank):
    """The plain FP64 path and the mixed-precision form on the headline DMC
    state point (N = 58, r_s = 5, 4096 walkers), same box, same start:
    walker-moves/s of each and their ratio (at fixed E_L error the ratio of
    walker-moves/s is the ratio of cost, as long as the mixed form samples
    the same distribution), the per-configuration |Delta E_L| against the
    FP64 path on 512 configurations, each run's mean energy with its error
    bar, and the acceptance ratio."""
    import torch

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    q = importlib.import_module("2degas_b200")
    tmp = tempfile.mkdtemp(prefix="qmc2d_prec_")
    nw = args.walkers
    d, cfg, workload = make_config(tmp, nw, 1)
    sysobj = q.System.read(d, "c")
    rs = cfg["rs"]
    delta, mmult, mage = 0.05 * rs * rs, 2.0, 50
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    with q.Handle(sysobj, capacity=nw, seed=7) as h0:
        h0.population_set(sysobj.read_configs(d, ".0", 0, nw))
        h0.vmc(args.equil, delta, 10 ** 9)
        h0.block_reset()
        h0.vmc(10, delta, 10 ** 9)
        blk, norm = h0.block_get()
        etrial = blk[0] / norm
        start = h0.population_get()
    out = {}
    for prec in ("fp64", "mixed"):
        with q.Handle(sysobj, capacity=nw, seed=11) as h:
            h.set_precision(prec)
            h.population_set(start["x"])
            h.autotune()
            stream = torch.cuda.ExternalStream(h.stream())
            for _ in range(args.warmup):
                h.dmc(1, 1, delta, etrial, mmult, mage)
            c0 = h.counters()
            dev_ms, means = 0.0, []
            nb = max(10, args.steps // 10)
            per = max(1, args.steps // nb)
            for b in range(nb):
                h.block_reset()
                for _ in range(per):
                    flush.zero_()
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    h.dmc(1, 1, delta, etrial, mmult, mage)
                    e1.record(stream)
                    e1.synchronize()
                    dev_ms += e0.elapsed_time(e1)
                blk, norm = h.block_get()
                means.append(blk[0] / norm)
            c1 = h.counters()
            means = np.array(means)
            out[prec] = {"walker_moves_per_s": nw * nb * per / (dev_ms * 1e-3),
                         "ms_per_step": dev_ms / (nb * per),
                         "e_mean": float(means.mean()),
                         "e_err": float(means.std(ddof=1) / math.sqrt(len(means))),
                         "acceptance": (c1["accepted"] - c0["accepted"]) /
                                       max(c1["proposed"] - c0["proposed"], 1)}
    # per-configuration error of the mixed form against the FP64 path
    x = start["x"][:512]
    res = {}
    for prec in ("fp64", "mixed"):
        with q.Handle(sysobj, capacity=len(x), seed=1) as h:
            h.set_precision(prec)
            res[prec] = h.compute_properties(x)
    de = np.abs(res["mixed"][2][:, 0] - res["fp64"][2][:, 0])
    dl = np.abs(res["mixed"][2][:, 1] - res["fp64"][2][:, 1])
    ratio = out["mixed"]["walker_moves_per_s"] / out["fp64"]["walker_moves_per_s"]
    comb = math.hypot(out["mixed"]["e_err"], out["fp64"]["e_err"])
    line = {
        "metric": ("walker-moves/sec ratio, mixed precision over plain FP64 (DMC with "
                   f"backflow, N=58 r_s={rs:g}, {nw} walkers, same E_L error)"),
        "value": ratio, "unit": "x", "n_gpus": 1, "steps": nb * per, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 / f64 with f32 u2 and v2 pair terms", "data": "synthetic",
        "config": {"workload": workload, "walkers_per_gpu": nw, "N": 58, "rs": rs,
                   "tau": delta, "l2": "flushed between timed steps (256 MiB write)"},
        "fp64": out["fp64"], "mixed": out["mixed"],
        "per_configuration_vs_fp64": {"configs": len(x), "max_abs_dE_L_ry_per_el": float(de.max()),
                                      "rms_dE_L_ry_per_el": float(np.sqrt((de ** 2).mean())),
                                      "max_abs_d_minus_ln_psi": float(dl.max())},
        "mean_energy_difference_in_combined_errors":
            (out["mixed"]["e_mean"] - out["fp64"]["e_mean"]) / max(comb, 1e-300),
    }
    print(json.dumps(line), flush=True)
    return 0


def serve_arm(args, rank, world):
    """The serving stream: Poisson arrivals (20 requests/s, seeded) of
    state points on the closed shells 26..162 that the kernels hold, r_s
    uniform in [1, 40], polarisation 0 or 1, VMC or DMC, 512..4096 walkers,
    target error bar 1e-4 Ry/electron; admitted by HBM footprint and run
    together. Then the same requests one at a time on the FP64 path."""
    import torch

    if rank != 0:  # one GPU serves; further ranks would be further servers
        return 0
    serve = importlib.import_module("2degas_b200.serve")
    unpol = [n for n in serve.closed_shells(81) if 26 <= 2 * n <= 162]
    pol = [n for n in serve.closed_shells(162) if 26 <= n <= 162]
    kw = dict(block_steps=20, min_blocks=5, max_blocks=args.serve_blocks,
              precision=args.precision)
    stream = lambda: serve.poisson_stream(args.serve_requests, 20.0, 2026, unpol, pol,  # noqa: E731
                                          **kw)
    free, total = torch.cuda.mem_get_info()
    budget = int(0.8 * free)
    srv = serve.Server(budget, max_slots=args.serve_slots,
                       max_hbm_dets=args.serve_hbm_dets if args.serve_hbm_dets > 0 else None)
    with Clocks(0) as clk:
        res = srv.serve(stream())
    sm = serve.summary(res)
    seq = None
    if not args.no_cpu:  # the same requests one at a time, FP64, as they arrive
        reqs = stream()
        for r in reqs:
            r.precision = "fp64"
        srv1 = serve.Server(budget, max_slots=1)
        t0 = time.perf_counter()
        res1 = srv1.serve(reqs, realtime=False)
        wall1 = time.perf_counter() - t0
        seq = serve.summary(res1, makespan=wall1)
        seq["energy_agreement"] = [
            (a.energy - b.energy) / max(math.hypot(a.error, b.error), 1e-300)
            for a, b in zip(res, res1) if a.status != "rejected" and b.status != "rejected"]
    line = {
        "metric": "walker-moves/sec (serving stream)", "value": sm["walker_moves_per_s"],
        "unit": UNIT, "n_gpus": 1, "steps": args.serve_requests, "warmup": 0,
        "ms_per_step": 1e3 * sm["makespan_s"] / max(args.serve_requests, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64 (f32 u2 and v2 pair terms)",
        "data": "synthetic",
        "config": {"workload": "serving_stream", "requests": args.serve_requests,
                   "arrivals_per_s": 20.0, "unpolarised_per_spin": unpol, "polarised": pol,
                   "rs": [1.0, 40.0], "walkers": [512, 4096], "target_ry_per_el": 1e-4,
                   "block_steps": 20, "max_blocks": args.serve_blocks,
                   "hbm_budget_bytes": budget, "slots": args.serve_slots,
                   "hbm_dets_at_once": args.serve_hbm_dets if args.serve_hbm_dets > 0 else None,
                   "precision": args.precision},
        "serving": {**sm, "peak_active": srv.peak_active, "peak_hbm_bytes": srv.peak_used,
                    "per_request": [dict(rid=r.rid, N=0, status=r.status, latency_s=r.latency,
                                         energy=r.energy, error=r.error, blocks=r.blocks,
                                         moves=r.moves, message=r.message[:80]) for r in res]},
        "one_at_a_time_fp64": seq,
        "cpu_baseline": (serve_cpu_baseline(stream(), res, args.cpu_seconds)
                         if not args.no_cpu else None),
        "clocks": clk.summary(),
    }
    for d, r in zip(line["serving"]["per_request"], stream()):
        d["N"], d["rs"], d["method"], d["walkers"] = r.N, r.rs, r.method, r.walkers
    print(json.dumps(line), flush=True)
    return 0


def batch_arm(args, rank, world):
    """Batched uneven populations: 64 DMC populations spanning N in {26, 42,
    58, 90, 122} and r_s in {1, 2, 5, 10, 20}, half unpolarised (N/2 per
    spin) and half fully polarised (the nearest closed shell: 25, 45, 57, 89,
    121), backflow on, 1024 walkers each, advanced together through
    qmc2d_batch_dmc (one CUDA graph per call), against the same generations
    issued handle by handle."""
    import torch

    if rank != 0:
        return 0
    q = importlib.import_module("2degas_b200")
    tables = importlib.import_module("2degas_b200.tables")
    tmp = tempfile.mkdtemp(prefix="qmc2d_batch_")
    Ns, rss = [26, 42, 58, 90, 122], [1.0, 2.0, 5.0, 10.0, 20.0]
    pol_of = {26: 25, 42: 45, 58: 57, 90: 89, 122: 121}
    nw = args.batch_walkers
    specs = []
    for i in range(args.batch_pops):
        N, pol, rs = Ns[i % 5], (i // 5) % 2, rss[(i // 10) % 5]
        specs.append((pol_of[N], 0, rs) if pol else (N // 2, N // 2, rs))
    systems, handles = {}, []
    for k, (nu, nd, rs) in enumerate(specs):
        key = (nu, nd, rs)
        if key not in systems:
            d = tables.make_run(os.path.join(tmp, f"s{len(systems)}"), "c", nu, nd, rs,
                                backflow=(0.2, rs, 0.6 * rs))
            systems[key] = q.System.read(d, "c")
        s = systems[key]
        h = q.Handle(s, capacity=nw, seed=1000 + k)
        h.set_precision(args.precision)
        L = s.s.el[0]
        h.population_set(np.random.default_rng(k).uniform(-L / 2, L / 2, size=(nw, 2 * s.N)))
        handles.append(h)
    taus = [0.01 * rs * rs for (_, _, rs) in specs]
    for h, (_, _, rs) in zip(handles, specs):
        h.vmc(args.equil, 0.05 * rs * rs, 10 ** 9)
        h.autotune()
        if args.move_inversion is not None:
            h.set_move_inversion(args.move_inversion)
    et = []
    for h, t in zip(handles, taus):
        h.block_reset()
        h.vmc(4, t, 10 ** 9)
        blk, norm = h.block_get()
        et.append(blk[0] / norm)
    K = args.steps
    moves = K * nw * len(handles)
    b = q.Batch(handles)
    sweep = {}
    with Clocks(0) as clk:
        for lanes in args.batch_lanes:  # concurrent chains of populations (0: all)
            b.set_lanes(lanes)
            b.dmc(max(2, min(K - K % 2, 16)), taus, et)  # warm-up and capture (the graph of K)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.dmc(K, taus, et)
            torch.cuda.synchronize()
            sweep[lanes] = time.perf_counter() - t0
        best = min(sweep, key=sweep.get)
        t_batch = sweep[best]
        t0 = time.perf_counter()
        for h, t, e in zip(handles, taus, et):  # the same work, one population at a time
            h.dmc(K, 1, t, e, 2.0, 50)
        torch.cuda.synchronize()
        t_seq = time.perf_counter() - t0
    line = {
        "metric": "walker-moves/sec (64 uneven DMC populations, one graph per call)",
        "value": moves / t_batch, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": 2,
        "ms_per_step": 1e3 * t_batch / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64 (f32 u2 and v2 pair terms)",
        "data": "synthetic",
        "config": {"workload": "batched_populations", "populations": len(handles),
                   "walkers_each": nw, "N": Ns, "rs": rss, "polarised_shells": pol_of,
                   "tau": "0.01 r_s^2", "precision": args.precision, "lanes": best,
                   "lanes_sweep_s": sweep,
                   "timing": "host wall clock around one qmc2d_batch_dmc call (synchronised)"},
        "handle_by_handle": {"value": moves / t_seq, "seconds": t_seq},
        "speedup_vs_handle_by_handle": t_seq / t_batch,
        # each population's autotuned launch: (pair-kernel walker groups,
        # rows not staged, inversion layout, lanes per particle) -> populations
        "launch_choices": {str(k): v for k, v in sorted(
            __import__("collections").Counter(tuple(h.get_launch()) + (h.get_pair_lanes(),)
                                              for h in handles).items())},
        "clocks": clk.summary(),
    }
    b.close()
    for h in handles:
        h.close()
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--walkers", type=int, default=4096)
    ap.add_argument("--equil", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="pair passes in FP64 (default), or u2 and real-space Ewald pair terms "
                         "in FP32 with compensated sums")
    ap.add_argument("--workload", default="dmc",
                    choices=["dmc", "vmc", "rmc", "serve", "batch", "precision"],
                    help="dmc: the N=58 DMC generation (default); vmc: plain VMC N=26 r_s=1, "
                         "256 walkers; rmc: reptation N=58 r_s=10, 512 reptiles x 200 beads; "
                         "serve: the serving stream; batch: 64 uneven populations through "
                         "one graph")
    ap.add_argument("--global-comb", action="store_true",
                    help="dmc workload over N ranks as one population: branch2's comb over "
                         "all ranks' walkers and the walker exchange every generation "
                         "(default: independent populations per rank)")
    ap.add_argument("--inversion", type=int, default=None, choices=[0, 1, 2],
                    help="determinant inversion layout (qmc2d_set_inversion)")
    ap.add_argument("--pair-lanes", type=int, default=None, choices=[4, 8, 16],
                    help="lanes per particle of the pair passes (qmc2d_set_pair_lanes)")
    ap.add_argument("--move-inversion", type=int, default=None, choices=[0, 1, 2],
                    help="orbitals and inversion of a move in their own kernel "
                         "(qmc2d_set_move_inversion)")
    ap.add_argument("--single", action="store_true",
                    help="vmc workload with single-electron moves and Sherman-Morrison updates")
    ap.add_argument("--rmc-split", type=int, default=None, choices=[0, 1],
                    help="reptation launch shape (qmc2d_rmc_set_launch)")
    ap.add_argument("--rmc-n", type=int, default=58, choices=[26, 58],
                    help="electrons of the reptation workload's deck")
    ap.add_argument("--shell", type=lambda v: tuple(int(t) for t in v.split(",")),
                    default=None, metavar="NU,ND",
                    help="dmc workload on another closed shell (electrons up, down)")
    ap.add_argument("--rs", type=float, default=None, help="r_s with --shell")
    ap.add_argument("--batch-pops", type=int, default=64)
    ap.add_argument("--batch-walkers", type=int, default=1024)
    ap.add_argument("--batch-lanes", type=lambda v: [int(t) for t in v.split(",")],
                    default=[0, 4, 8, 16], metavar="S,S,...",
                    help="populations in flight at a time to try (0: all); the best is kept")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-blocks", type=int, default=100)
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-hbm-dets", type=int, default=1,
                    help="requests with determinants in HBM at once (0: no cap)")
    ap.add_argument("--phases", action="store_true",
                    help="print SM cycles per walker-move of each move-kernel phase instead")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.workload == "serve":
        return serve_arm(args, rank, world)
    if args.workload == "batch":
        return batch_arm(args, rank, world)
    if args.workload in ("vmc", "rmc"):
        return config_arm(args, rank, world, local_rank)
    if args.workload == "precision":
        return precision_arm(args, rank, world, local_rank)
    return b200_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
