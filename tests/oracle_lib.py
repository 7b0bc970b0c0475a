"""ctypes binding of the CPU oracle (oracle/build/liboracle.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg load the oracle, and only as the checker.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_long, c_uint32, c_uint64, c_void_p

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "build", "liboracle.so")

PD = POINTER(c_double)
PI = POINTER(c_int)


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def _ptr(a):
    return a.ctypes.data_as(PD)


def _load():
    if not os.path.exists(ORACLE_SO):
        build()
    lib = ctypes.CDLL(ORACLE_SO)
    lib.oracle_system_read.restype = c_int
    lib.oracle_system_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p, POINTER(c_void_p)]
    lib.oracle_system_free.argtypes = [c_void_p]
    lib.oracle_system_set_twist.restype = c_int
    lib.oracle_system_set_twist.argtypes = [c_void_p, c_int, c_int]
    lib.oracle_read_configs.restype = c_int
    lib.oracle_read_configs.argtypes = [c_void_p, ctypes.c_char_p, ctypes.c_char_p, c_int, c_int,
                                        PD, PI]
    lib.oracle_system_sizes.argtypes = [c_void_p, PI, PI, PI]
    return lib


class OracleSystem:
    """A run directory read by the oracle's own reader (oracle_input.c),
    independently of the product library's qmc2d_system_read."""

    def __init__(self, directory, runid, twist=None):
        self.lib = _load()
        self.ptr = c_void_p()
        self.directory, self.runid = str(directory), runid
        st = self.lib.oracle_system_read(self.directory.encode(), runid.encode(),
                                         ctypes.byref(self.ptr))
        if st:
            raise RuntimeError(f"oracle reader: status {st} on {directory}/{runid}.sy")
        if twist is not None:
            self.set_twist(*twist)
        n, t, p = c_int(), c_int(), c_int()
        self.lib.oracle_system_sizes(self.ptr, ctypes.byref(n), ctypes.byref(t), ctypes.byref(p))
        self.N, self.ntypes, self.nprops = n.value, t.value, p.value

    @classmethod
    def read(cls, directory, runid):
        return cls(directory, runid)

    def __del__(self):
        try:
            if self.ptr:
                self.lib.oracle_system_free(self.ptr)
                self.ptr = c_void_p()
        except Exception:
            pass

    def set_twist(self, ith, jth):
        st = self.lib.oracle_system_set_twist(self.ptr, ith, jth)
        if st:
            raise RuntimeError(f"oracle set_twist: status {st}")

    def read_configs(self, directory, suffix, first, count):
        x = np.zeros((count, 2 * self.N))
        n = c_int(0)
        st = self.lib.oracle_read_configs(self.ptr, str(directory).encode(), suffix.encode(),
                                          first, count, _ptr(x), ctypes.byref(n))
        if st:
            raise RuntimeError(f"oracle read_configs: status {st}")
        return x[: n.value]


class Oracle:
    def __init__(self, system):
        """system: an OracleSystem, or any object with `directory`, `runid`
        and `twist` (the product's System): the oracle then reads the same run
        directory itself and sets the same twist."""
        if not isinstance(system, OracleSystem):
            system = OracleSystem(system.directory, system.runid,
                                  getattr(system, "twist", None))
        self.system = system
        self.lib = lib = _load()
        lib.oracle_work_new.restype = c_void_p
        lib.oracle_work_new.argtypes = [c_void_p]
        lib.oracle_work_free.argtypes = [c_void_p]
        lib.oracle_compute_properties.restype = c_int
        lib.oracle_compute_properties.argtypes = [c_void_p, c_void_p, PD, PD, PD, PD, PD, PI]
        lib.oracle_vmc_rannyu.restype = c_int
        lib.oracle_vmc_rannyu.argtypes = [c_void_p, PD, c_int, c_double, c_int, PI, c_int, PD,
                                          PD, PI, POINTER(c_long)]
        lib.oracle_vmc_philox.restype = c_int
        lib.oracle_vmc_philox.argtypes = [c_void_p, c_int, c_int, c_double, c_int, c_uint64,
                                          c_long, PD, PD, PD, PD, PD, PD, PD, POINTER(c_long)]
        lib.oracle_population_init.restype = c_int
        lib.oracle_population_init.argtypes = [c_void_p, c_int, PD, PD, PD, PD, PD, PD]
        lib.oracle_branch2.restype = c_int
        lib.oracle_branch2.argtypes = [c_int, PD, PD, PI, PI, PI]
        lib.oracle_dmc_philox.restype = c_int
        lib.oracle_dmc_philox.argtypes = [c_void_p, c_int, c_int, c_int, c_double, c_double,
                                          c_double, c_int, c_uint64, c_long, c_long, PD, PD, PD,
                                          PD, PD, PD, PD, PD, POINTER(c_long)]
        lib.oracle_philox_uniform2.argtypes = [c_uint64, c_uint32, c_uint32, c_uint32, c_uint32,
                                               PD]
        lib.oracle_vmc_single.restype = c_int
        lib.oracle_vmc_single.argtypes = [c_void_p, c_int, c_int, c_double, c_uint64, c_long,
                                          PD, PD, PD, PD, PD, PD, PD, POINTER(c_long)]
        lib.oracle_reptile_new.restype = c_void_p
        lib.oracle_reptile_new.argtypes = [c_void_p, c_void_p]
        lib.oracle_reptile_free.argtypes = [c_void_p]
        lib.oracle_reptile_init.restype = c_int
        lib.oracle_reptile_init.argtypes = [c_void_p, c_void_p, PD]
        lib.oracle_reptile_run.restype = c_int
        lib.oracle_reptile_run.argtypes = [c_void_p, c_void_p, c_int, c_uint64, c_long, c_int, PD,
                                           POINTER(c_long)]
        lib.oracle_reptile_path.argtypes = [c_void_p, PD, PD]
        lib.oracle_setrn.argtypes = [c_void_p, PI]
        lib.oracle_savern.argtypes = [c_void_p, PI]
        lib.oracle_rannyu.restype = c_double
        lib.oracle_rannyu.argtypes = [c_void_p]
        self.N = system.N
        self.nt = system.ntypes
        self.nprops = system.nprops
        self.work = lib.oracle_work_new(system.ptr)

    def __del__(self):
        try:
            self.lib.oracle_work_free(self.work)
        except Exception:
            pass

    @property
    def _s(self):
        return self.system.ptr

    def compute_properties(self, x):
        """x: (2N,) float64 -> (g, h, p, s, underflow)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        g = np.zeros(2 * self.N)
        h = np.zeros(self.nt)
        p = np.zeros(self.nprops)
        s = np.zeros(1)
        uf = c_int(0)
        st = self.lib.oracle_compute_properties(self._s, self.work, _ptr(x), _ptr(g), _ptr(h),
                                                _ptr(p), _ptr(s), ctypes.byref(uf))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return g, h, p, s[0], uf.value

    def vmc_rannyu(self, x0, nstp, delta, mage, seed, rng_order=0):
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        blk = np.zeros(self.nprops)
        xf = np.zeros(2 * self.N)
        sd = (c_int * 4)(*seed)
        so = (c_int * 4)()
        nacc = c_long(0)
        st = self.lib.oracle_vmc_rannyu(self._s, _ptr(x0), nstp, delta, mage, sd, rng_order,
                                        _ptr(blk), _ptr(xf), so, ctypes.byref(nacc))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return blk, xf, list(so), nacc.value

    def population_init(self, x):
        nw = x.shape[0]
        x = np.ascontiguousarray(x, dtype=np.float64)
        pop = dict(x=x.copy(), g=np.zeros((nw, 2 * self.N)), h=np.zeros((nw, self.nt)),
                   p=np.zeros((nw, self.nprops)), s=np.zeros(nw), age=np.zeros(nw))
        st = self.lib.oracle_population_init(self._s, nw, _ptr(pop["x"]), _ptr(pop["g"]),
                                             _ptr(pop["h"]), _ptr(pop["p"]), _ptr(pop["s"]),
                                             _ptr(pop["age"]))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return pop

    def vmc_philox(self, pop, nstp, delta, mage, seed, step0=0):
        nw = pop["x"].shape[0]
        blk = np.zeros(self.nprops)
        nacc = c_long(0)
        st = self.lib.oracle_vmc_philox(self._s, nw, nstp, delta, mage, seed, step0,
                                        _ptr(pop["x"]), _ptr(pop["g"]), _ptr(pop["h"]),
                                        _ptr(pop["p"]), _ptr(pop["s"]), _ptr(pop["age"]),
                                        _ptr(blk), ctypes.byref(nacc))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return blk, nacc.value

    def vmc_single(self, pop, nsweep, delta, seed, sweep0=0):
        """Single-electron sweeps (qmc2d_vmc_single's streams); pop["x"] in,
        every record out; returns (block sums, accepted moves)."""
        nw = pop["x"].shape[0]
        blk = np.zeros(self.nprops)
        nacc = c_long(0)
        st = self.lib.oracle_vmc_single(self._s, nw, nsweep, delta, seed, sweep0,
                                        _ptr(pop["x"]), _ptr(pop["g"]), _ptr(pop["h"]),
                                        _ptr(pop["p"]), _ptr(pop["s"]), _ptr(pop["age"]),
                                        _ptr(blk), ctypes.byref(nacc))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return blk, nacc.value

    def dmc_philox(self, pop, ngen, mmstep, delta, etrial, mmult, mage, seed, gen0=0,
                   move0=0):
        nw = pop["x"].shape[0]
        blk = np.zeros(self.nprops)
        norm = np.zeros(1)
        nacc = c_long(0)
        st = self.lib.oracle_dmc_philox(self._s, nw, ngen, mmstep, delta, etrial, mmult, mage,
                                        seed, gen0, move0, _ptr(pop["x"]), _ptr(pop["g"]),
                                        _ptr(pop["h"]), _ptr(pop["p"]), _ptr(pop["s"]),
                                        _ptr(pop["age"]), _ptr(blk), _ptr(norm),
                                        ctypes.byref(nacc))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return blk, norm[0], nacc.value

    def branch2(self, wate, r):
        wate = np.ascontiguousarray(wate, dtype=np.float64).copy()
        r = np.ascontiguousarray(r, dtype=np.float64)
        nw = wate.shape[0]
        mult = np.zeros(nw, dtype=np.int32)
        src = np.zeros(nw, dtype=np.int32)
        ncap = c_int(0)
        used = self.lib.oracle_branch2(nw, _ptr(wate), _ptr(r), mult.ctypes.data_as(PI),
                                       src.ctypes.data_as(PI), ctypes.byref(ncap))
        return mult, src, used, ncap.value

    def rannyu_stream(self, seed, count):
        """count draws of the reference's rannyu after setrn(seed); returns
        (draws, savern state)."""
        st = (c_int * 8)()
        sd = (c_int * 4)(*seed)
        self.lib.oracle_setrn(ctypes.byref(st), sd)
        out = np.array([self.lib.oracle_rannyu(ctypes.byref(st)) for _ in range(count)])
        so = (c_int * 4)()
        self.lib.oracle_savern(ctypes.byref(st), so)
        return out, list(so)

    def philox_uniform2(self, seed, c0, c1, c2, c3):
        u = np.zeros(2)
        self.lib.oracle_philox_uniform2(seed, c0, c1, c2, c3, _ptr(u))
        return u

    def reptile(self, prm):
        return Reptile(self, prm)


class Reptile:
    def __init__(self, oracle, prm):
        self.o = oracle
        self.prm = prm
        self.ptr = oracle.lib.oracle_reptile_new(oracle._s, ctypes.cast(ctypes.pointer(prm),
                                                                        c_void_p))

    def __del__(self):
        try:
            self.o.lib.oracle_reptile_free(self.ptr)
        except Exception:
            pass

    def init(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        st = self.o.lib.oracle_reptile_init(self.o._s, self.ptr, _ptr(x))
        if st:
            raise RuntimeError(f"oracle status {st}")

    def run(self, rid, seed, step0, nstp):
        blk = np.zeros(self.o.nprops)
        nacc = c_long(0)
        st = self.o.lib.oracle_reptile_run(self.o._s, self.ptr, rid, seed, step0, nstp,
                                           _ptr(blk), ctypes.byref(nacc))
        if st:
            raise RuntimeError(f"oracle status {st}")
        return blk, nacc.value

    def path(self):
        x = np.zeros((self.prm.ntau, 2 * self.o.N))
        p = np.zeros((self.prm.ntau, self.o.nprops))
        self.o.lib.oracle_reptile_path(self.ptr, _ptr(x), _ptr(p))
        return x, p
