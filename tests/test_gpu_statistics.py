"""Independent runs, GPU against the oracle (the reference's algorithm
restated on the CPU): VMC, DMC and reptation energies of the n26 golden
deck from different random streams agree within their combined
statistical error.

Both sides start from one population equilibrated on the GPU (2000 VMC
steps from the stored configurations, whose energy is still drifting
then), run their own equilibration with their own streams, then blocks of
100 steps. A side's mean and error are the mean of its block energies and
their spread over sqrt(blocks); blocks of 100 steps are several
autocorrelation times of E_L. The GPU runs 8x the oracle's population; the
bar is 4 combined standard errors."""
import numpy as np
import pytest

from oracle_lib import Reptile

pytestmark = pytest.mark.gpu

NB, BS = 10, 100


def _ms(e):
    e = np.asarray(e)
    return e.mean(), e.std(ddof=1) / np.sqrt(len(e))


def _agree(gpu, cpu, what):
    (m1, s1), (m2, s2) = _ms(gpu), _ms(cpu)
    assert abs(m1 - m2) < 4.0 * np.hypot(s1, s2), (what, m1, s1, m2, s2)


@pytest.fixture(scope="module")
def equilibrated(q, n26_dir):
    s = q.System.read(n26_dir, "n26")
    x = s.read_configs(n26_dir, ".0", 0, 64)
    with q.Handle(s, capacity=len(x), seed=0x0E0E) as h:
        h.population_set(x)
        h.vmc(2000, 0.05, 10 ** 9)
        return h.population_get()["x"]


def test_vmc_energy(q, oracle_cls, n26, equilibrated):
    """With mage = 50 (a move forced after 50 rejections, as the reference's
    persistent-walker rule): without it a walker stuck at a high E_L stays
    in the average for good, and the larger GPU population meets one more
    often."""
    x = equilibrated
    mage = 50
    o = oracle_cls(n26)
    pop = o.population_init(x)
    o.vmc_philox(pop, 100, 0.05, mage, 0x1111, 0)
    cpu = []
    for b in range(NB):
        blk, _ = o.vmc_philox(pop, BS, 0.05, mage, 0x1111, 100 + BS * b)
        cpu.append(blk[0] / (len(x) * BS))
    gpu = []
    with q.Handle(n26, capacity=8 * len(x), seed=0x2222) as h:
        h.population_set(np.tile(x, (8, 1)))
        h.vmc(100, 0.05, mage)
        for _ in range(NB):
            h.block_reset()
            h.vmc(BS, 0.05, mage)
            blk, norm = h.block_get()
            gpu.append(blk[0] / norm)
    _agree(gpu, cpu, "vmc")


def test_dmc_energy(q, oracle_cls, n26, equilibrated):
    x = equilibrated
    tau, et = 0.01, -0.445
    o = oracle_cls(n26)
    pop = o.population_init(x)
    o.dmc_philox(pop, 100, 1, tau, et, 2.0, 50, 0x3333, 0, 0)
    cpu = []
    for b in range(NB):
        blk, norm, _ = o.dmc_philox(pop, BS, 1, tau, et, 2.0, 50, 0x3333, 100 + BS * b,
                                    100 + BS * b)
        cpu.append(blk[0] / np.asarray(norm).ravel()[0])
    gpu = []
    with q.Handle(n26, capacity=8 * len(x), seed=0x4444) as h:
        h.population_set(np.tile(x, (8, 1)))
        h.dmc(100, 1, tau, et, 2.0, 50)
        for _ in range(NB):
            h.block_reset()
            h.dmc(BS, 1, tau, et, 2.0, 50)
            blk, norm = h.block_get()
            gpu.append(blk[0] / norm)
    _agree(gpu, cpu, "dmc")


def test_reptation_energy(q, oracle_cls, n26, equilibrated):
    import importlib

    capi = importlib.import_module("2degas_b200._capi")
    ntau, nrep_cpu = 16, 8
    prm = capi.RmcParams(ntau, 2, 2, 0.01, -0.445, 1000, 1000)
    o = oracle_cls(n26)
    paths = [equilibrated[(r * ntau) % 64:(r * ntau) % 64 + ntau] for r in range(4)]
    reps = []
    for r in range(nrep_cpu):
        rep = Reptile(o, prm)
        rep.init(paths[r % 4])
        rep.run(r, 0x5555, 0, 200)
        reps.append(rep)
    cpu = []
    for b in range(NB):
        tot = np.zeros(n26.nprops)
        for r, rep in enumerate(reps):
            blk, _ = rep.run(r, 0x5555, 200 + BS * b, BS)
            tot += blk
        cpu.append(tot[0] / (nrep_cpu * BS))
    nrep = 8 * nrep_cpu
    gpu = []
    with q.Handle(n26, capacity=nrep, seed=0x6666) as h:
        h.rmc_init(nrep, np.concatenate([paths[r % 4] for r in range(nrep)]), ntau, 2, 2, 0.01,
                   -0.445, 1000, 1000)
        h.rmc(200)
        for _ in range(NB):
            h.block_reset()
            h.rmc(BS)
            blk, norm = h.block_get()
            gpu.append(blk[0] / norm)
    _agree(gpu, cpu, "rmc")
