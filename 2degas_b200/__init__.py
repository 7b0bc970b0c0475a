"""qmc2d-b200: the walker-propagation path of 2degas on B200 (sm_100a).

Python view of the C-ABI in include/qmc2d.h. The heavy lifting is in
lib/libqmc2d.so (CUDA kernels + C++ host); this module only marshals
arrays. There is no CPU fallback: if the library or a GPU is missing, the
calls raise.

    import importlib
    q = importlib.import_module("2degas_b200")
    sys_ = q.System.read("tests/golden/n26", "n26")
    with q.Handle(sys_, capacity=256, seed=1) as h:
        g, hl, props, s = h.compute_properties(x)
"""
import ctypes

import numpy as np

from . import _capi

__all__ = ["System", "Handle", "Batch", "Stats", "tabc", "QMCError", "load_library", "_capi"]

QMCError = _capi.QMCError


def load_library():
    return _capi.load()


def _pd(a):
    return a.ctypes.data_as(_capi.PD)


class System:
    """A qmc2d_system read from a reference run directory (input, t_read, kread)."""

    def __init__(self, ptr, lib, directory=None, runid=None):
        self.ptr = ptr
        self.lib = lib
        self.directory, self.runid = directory, runid
        self.twist = None  # (ith, jth) after set_twist; None: as read

    @classmethod
    def read(cls, directory, runid):
        lib = _capi.load()
        sp = _capi.SYSP()
        _capi.check(lib, lib.qmc2d_system_read(str(directory).encode(), runid.encode(),
                                               ctypes.byref(sp)))
        return cls(sp, lib, str(directory), runid)

    def __del__(self):
        try:
            if self.ptr:
                self.lib.qmc2d_system_free(self.ptr)
                self.ptr = None
        except Exception:
            pass

    @property
    def s(self):
        return self.ptr.contents

    @property
    def N(self):
        return self.s.nptot

    @property
    def ntypes(self):
        return self.s.ntypes

    @property
    def nprops(self):
        return self.s.n_props

    def set_twist(self, ith, jth):
        _capi.check(self.lib, self.lib.qmc2d_system_set_twist(self.ptr, ith, jth))
        self.twist = (ith, jth)

    def rmc_estimators_setup(self, ntau, ntauskip):
        """mstar/cmass/itc setup of the deck's records for ntau-bead paths."""
        est = _capi.RmcEstimators()
        _capi.check(self.lib, self.lib.qmc2d_rmc_estimators_setup(self.ptr, ntau, ntauskip,
                                                                  ctypes.byref(est)))
        return est

    def footprint(self, capacity):
        """Device bytes a Handle of this capacity allocates (no GPU needed)."""
        b = ctypes.c_uint64(0)
        _capi.check(self.lib, self.lib.qmc2d_footprint(self.ptr, capacity, ctypes.byref(b)))
        return b.value

    def gvec(self):
        s = self.s
        return np.ctypeslib.as_array(s.gvec, shape=(2 * s.ngvec,)).reshape(-1, 2).copy()

    def read_configs(self, directory, suffix, first, count):
        x = np.zeros((count, 2 * self.N))
        n = ctypes.c_int(0)
        _capi.check(self.lib, self.lib.qmc2d_read_configs(self.ptr, str(directory).encode(),
                                                          suffix.encode(), first, count, _pd(x),
                                                          ctypes.byref(n)))
        return x[: n.value]


class Handle:
    """Device-resident state for one system (qmc2d_create .. qmc2d_destroy)."""

    def __init__(self, system, capacity, seed=1, device=0):
        self.system = system
        self.lib = system.lib
        self.cap = capacity
        self.h = ctypes.c_void_p()
        opt = _capi.Options(capacity, device, seed)
        _capi.check(self.lib, self.lib.qmc2d_create(system.ptr, ctypes.byref(opt),
                                                    ctypes.byref(self.h)))

    def close(self):
        if self.h:
            self.lib.qmc2d_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code):
        return _capi.check(self.lib, code)

    # compute_properties (reptation.f:2661)
    def compute_properties(self, x):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        nw, N, nt, np_ = x.shape[0], self.system.N, self.system.ntypes, self.system.nprops
        g = np.zeros((nw, 2 * N))
        hl = np.zeros((nw, nt))
        p = np.zeros((nw, np_))
        s = np.zeros(nw)
        self._chk(self.lib.qmc2d_compute_properties(self.h, nw, _pd(x), _pd(g), _pd(hl), _pd(p),
                                                    _pd(s)))
        return g, hl, p, s

    def compute_properties_dev(self, nw, x_ptr, g_ptr, h_ptr, p_ptr, s_ptr, stream=None):
        self._chk(self.lib.qmc2d_compute_properties_dev(self.h, nw, x_ptr, g_ptr, h_ptr, p_ptr,
                                                        s_ptr, stream))

    def compute_properties_dev_status(self, nw, stream=None):
        """Wait for the last compute_properties_dev and raise on a failed walker."""
        self._chk(self.lib.qmc2d_compute_properties_dev_status(self.h, nw, stream))

    def population_set(self, x):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        self._chk(self.lib.qmc2d_population_set(self.h, x.shape[0], _pd(x)))

    def population_size(self):
        n = ctypes.c_int()
        self._chk(self.lib.qmc2d_population_size(self.h, ctypes.byref(n)))
        return n.value

    def population_get(self):
        nw, N, np_ = self.population_size(), self.system.N, self.system.nprops
        x = np.zeros((nw, 2 * N))
        g = np.zeros((nw, 2 * N))
        hl = np.zeros((nw, self.system.ntypes))
        p = np.zeros((nw, np_))
        s = np.zeros(nw)
        age = np.zeros(nw)
        self._chk(self.lib.qmc2d_population_get(self.h, _pd(x), _pd(g), _pd(hl), _pd(p), _pd(s),
                                                _pd(age)))
        return dict(x=x, g=g, h=hl, p=p, s=s, age=age)

    def population_get_ptr(self, x, g, hl, p, s, age):
        """Copy out into caller buffers given as raw addresses (e.g. pinned memory)."""
        c = ctypes.cast
        self._chk(self.lib.qmc2d_population_get(self.h, c(x, _capi.PD), c(g, _capi.PD),
                                                c(hl, _capi.PD), c(p, _capi.PD),
                                                c(s, _capi.PD), c(age, _capi.PD)))

    def population_load_ptr(self, nw, x, g, hl, p, s, age):
        """Load walker records from raw host addresses (putconf for a population)."""
        self._chk(self.lib.qmc2d_population_load(self.h, nw, x, g, hl, p, s, age))

    def population_load_async_ptr(self, nw, x, g, hl, p, s, age):
        """qmc2d_population_load_async: returns at once; the buffers stay in use
        until the next call that synchronises the handle (a move, a get)."""
        self._chk(self.lib.qmc2d_population_load_async(self.h, nw, x, g, hl, p, s, age))

    def stream(self):
        st = ctypes.c_void_p()
        self._chk(self.lib.qmc2d_stream(self.h, ctypes.byref(st)))
        return st.value

    def profile(self, enable=True):
        self._chk(self.lib.qmc2d_profile(self.h, 1 if enable else 0))

    PHASES = ("propose", "pairs", "rhok", "u3", "orbitals", "invert", "fmat", "drift",
              "mbuild", "cross", "assemble", "accept", "path")

    def phase_timers(self, enable=True):
        """Start (enable) or stop and return {phase: SM cycles summed over CTAs}."""
        buf = (ctypes.c_ulonglong * 16)()
        self._chk(self.lib.qmc2d_phase_timers(self.h, 1 if enable else 0, buf))
        if enable:
            return None
        return {name: int(buf[i]) for i, name in enumerate(self.PHASES)}

    def profile_get(self, kernel):
        ms = ctypes.c_double()
        n = ctypes.c_long()
        self._chk(self.lib.qmc2d_profile_get(self.h, kernel, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def block_reset(self):
        self._chk(self.lib.qmc2d_block_reset(self.h))

    def block_get(self):
        b = np.zeros(self.system.nprops)
        n = ctypes.c_double()
        self._chk(self.lib.qmc2d_block_get(self.h, _pd(b), ctypes.byref(n)))
        return b, n.value

    def counters(self):
        c = _capi.Counters()
        self._chk(self.lib.qmc2d_counters_get(self.h, ctypes.byref(c)))
        return dict(accepted=c.accepted, proposed=c.proposed, forced=c.forced,
                    capped=c.max_weight_capped)

    def vmc(self, nstp, delta, mage):
        self._chk(self.lib.qmc2d_vmc(self.h, nstp, delta, mage))

    def dmc_weights(self, mmstep, delta, etrial, mmult, mage):
        """One DMC generation's moves and weights, without the comb."""
        w = np.zeros(self.population_size())
        self._chk(self.lib.qmc2d_dmc_weights(self.h, mmstep, delta, etrial, mmult, mage, _pd(w)))
        return w

    def record_len(self):
        n = ctypes.c_int()
        self._chk(self.lib.qmc2d_record_len(self.h, ctypes.byref(n)))
        return n.value

    def records_pack(self, slots, buf_ptr, stream=None):
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        self._chk(self.lib.qmc2d_records_pack(self.h, len(sl), sl.ctypes.data_as(_capi.PI),
                                              buf_ptr, stream))

    def records_unpack(self, slots, buf_ptr, stream=None):
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        self._chk(self.lib.qmc2d_records_unpack(self.h, len(sl), sl.ctypes.data_as(_capi.PI),
                                                buf_ptr, stream))

    def population_resample(self, src):
        s = np.ascontiguousarray(src, dtype=np.int32)
        self._chk(self.lib.qmc2d_population_resample(self.h, s.ctypes.data_as(_capi.PI)))

    def vmc_single(self, nsweep, delta, refresh=50):
        """nsweep sweeps of single-electron moves (plain Slater-Jastrow decks);
        the inverse is recomputed every `refresh` moves (0: at the start only)."""
        self._chk(self.lib.qmc2d_vmc_single(self.h, nsweep, delta, refresh))

    def single_drift(self):
        """Largest |W D - I| before a recompute in the last vmc_single call."""
        d = ctypes.c_double()
        self._chk(self.lib.qmc2d_single_drift(self.h, ctypes.byref(d)))
        return d.value

    def dmc(self, nstp, mmstep, delta, etrial, mmult, mage):
        self._chk(self.lib.qmc2d_dmc(self.h, nstp, mmstep, delta, etrial, mmult, mage))

    def rmc_init(self, nrep, x, ntau, ntauskip, mdelta, delta, etrial, mage, mage_r):
        x = np.ascontiguousarray(x, dtype=np.float64)
        prm = _capi.RmcParams(ntau, ntauskip, mdelta, delta, etrial, mage, mage_r)
        self._chk(self.lib.qmc2d_rmc_init(self.h, nrep, ctypes.byref(prm), _pd(x)))

    def rmc_set_launch(self, split):
        """1: pair kernel + determinant kernel per bead growth (default); 0: one
        kernel per launch for whole moves."""
        self._chk(self.lib.qmc2d_rmc_set_launch(self.h, split))

    def rmc(self, nstp):
        self._chk(self.lib.qmc2d_rmc(self.h, nstp))

    def rmc_estimators(self, est):
        """The path estimators of the current reptiles, averaged over them."""
        out = np.zeros(max(est.nvalues, 1))
        self._chk(self.lib.qmc2d_rmc_path_estimators(self.h, ctypes.byref(est), _pd(out)))
        return out[: est.nvalues]

    def rmc_get_path(self, rep, ntau):
        N, np_ = self.system.N, self.system.nprops
        x = np.zeros((ntau, 2 * N))
        p = np.zeros((ntau, np_))
        self._chk(self.lib.qmc2d_rmc_get_path(self.h, rep, _pd(x), _pd(p)))
        return x, p

    def set_precision(self, precision):
        """Precision of the pair passes: "fp64" (the default) or "mixed" (u2
        and real-space Ewald pair terms in FP32 with compensated sums, all
        else FP64)."""
        code = {"fp64": _capi.PRECISION_FP64, "mixed": _capi.PRECISION_MIXED}[precision]
        self._chk(self.lib.qmc2d_set_precision(self.h, code))

    def set_dmc_ecut(self, ecut):
        """Clamp E_L in the DMC weight to etrial +- ecut (Ry/electron; 0: off,
        the reference's weights)."""
        self._chk(self.lib.qmc2d_set_dmc_ecut(self.h, ecut))

    def set_launch(self, groups=0, stage=0):
        """Pair-kernel launch choice: walker groups per CTA (1, 2; 0 default)
        and pair-row staging (0 when it fits, 1 never)."""
        self._chk(self.lib.qmc2d_set_launch(self.h, groups, stage))

    def set_inversion(self, layout):
        """0: register-resident Gauss-Jordan over every warp (default); 1: one
        warp per spin in shared memory; 2: panel-blocked."""
        self._chk(self.lib.qmc2d_set_inversion(self.h, layout))

    def set_pair_lanes(self, lanes):
        """Lanes per particle of the pair passes: 4, 8 or 16 (0: the default, 8)."""
        self._chk(self.lib.qmc2d_set_pair_lanes(self.h, lanes))

    def set_move_inversion(self, mode):
        """Orbitals and inversion of a move in their own kernel before the move
        kernel: 1 when the population is large enough (default), 2 whenever it
        fits, 0 never (inside the move kernel)."""
        self._chk(self.lib.qmc2d_set_move_inversion(self.h, mode))

    def set_autotune_scope(self, mask):
        """What autotune() times: 1 groups/staging, 2 lanes, 4 inversion layout."""
        self._chk(self.lib.qmc2d_set_autotune_scope(self.h, mask))

    def get_move_inversion(self):
        v = ctypes.c_int()
        self._chk(self.lib.qmc2d_get_move_inversion(self.h, ctypes.byref(v)))
        return v.value

    def get_pair_lanes(self):
        v = ctypes.c_int()
        self._chk(self.lib.qmc2d_get_pair_lanes(self.h, ctypes.byref(v)))
        return v.value

    def get_launch(self):
        """(pair-kernel walker groups, staging, inversion layout) in force."""
        g, st, inv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._chk(self.lib.qmc2d_get_launch(self.h, ctypes.byref(g), ctypes.byref(st),
                                            ctypes.byref(inv)))
        return g.value, st.value, inv.value

    def autotune(self):
        """Time the pair kernel's launch choices on the current population,
        keep the fastest; returns (groups, stage, ms per launch)."""
        g, st, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._chk(self.lib.qmc2d_autotune(self.h, ctypes.byref(g), ctypes.byref(st),
                                          ctypes.byref(ms)))
        return g.value, st.value, ms.value

    def update_twist(self):
        """After system.set_twist(ith, jth): the orbitals use the new wave vectors."""
        self._chk(self.lib.qmc2d_update_twist(self.h, self.system.ptr))

    def write_conf(self, directory, rank=0):
        """write_conf: the population's coordinates to <dir>/<x_file>.<rank>."""
        self._chk(self.lib.qmc2d_write_conf(self.h, self.system.ptr, str(directory).encode(),
                                            rank))

    def restart_write(self, stats, iblk, who, directory, runid, rank=0):
        """restart(1): <dir>/<runid>.res and <dir>/<x_file>.res.<rank>."""
        self._chk(self.lib.qmc2d_restart_write(self.h, self.system.ptr, stats.p, iblk,
                                               who.encode(), str(directory).encode(),
                                               runid.encode(), rank))

    def restart_read(self, stats, who, directory, runid, rank=0):
        """restart(0): returns (stored block, etrial); the configurations
        become the population."""
        ib = ctypes.c_int()
        et = ctypes.c_double()
        self._chk(self.lib.qmc2d_restart_read(self.h, self.system.ptr, stats.p, who.encode(),
                                              str(directory).encode(), runid.encode(), rank,
                                              ctypes.byref(ib), ctypes.byref(et)))
        return ib.value, et.value

    def restart_read_rmc(self, stats, directory, runid, ntau, ntauskip, mdelta, delta, etrial,
                         mage, mage_r, rank=0):
        """restart(0) + read_path for reptation: the stored paths become
        ntau-bead reptiles; returns the stored block."""
        ib = ctypes.c_int()
        prm = _capi.RmcParams(ntau, ntauskip, mdelta, delta, etrial, mage, mage_r)
        self._chk(self.lib.qmc2d_restart_read_rmc(self.h, self.system.ptr, stats.p,
                                                  ctypes.byref(prm), str(directory).encode(),
                                                  runid.encode(), rank, ctypes.byref(ib)))
        return ib.value


class Stats:
    """Cumulative block statistics of averages(3) (qmc2d_stats_*)."""

    def __init__(self, system, n=None):
        """Statistics of the system's n_props properties, or of n values
        (e.g. the reptation path estimators, n = est.nvalues)."""
        self.system = system
        self.lib = system.lib
        self.n = system.nprops if n is None else n
        self.p = ctypes.c_void_p()
        _capi.check(self.lib, self.lib.qmc2d_stats_create(self.n, ctypes.byref(self.p)))

    def __del__(self):
        try:
            if self.p:
                self.lib.qmc2d_stats_destroy(self.p)
                self.p = None
        except Exception:
            pass

    def add_block(self, blk, norm):
        blk = np.ascontiguousarray(blk, dtype=np.float64)
        _capi.check(self.lib, self.lib.qmc2d_stats_add_block(self.p, _pd(blk), norm))

    def get(self):
        """(cumulative means, errors, cml_norm, blocks)."""
        n = self.n
        mean, err = np.zeros(n), np.zeros(n)
        norm, ib = ctypes.c_double(), ctypes.c_int()
        _capi.check(self.lib, self.lib.qmc2d_stats_get(self.p, _pd(mean), _pd(err),
                                                       ctypes.byref(norm), ctypes.byref(ib)))
        return mean, err, norm.value, ib.value

    def write_estimators(self, est, blk, norm, directory, runid):
        """The reptation estimator files of averages(3) for this block."""
        blk = np.ascontiguousarray(blk, dtype=np.float64)
        _capi.check(self.lib, self.lib.qmc2d_stats_write_estimators(
            self.p, self.system.ptr, ctypes.byref(est), _pd(blk), norm,
            str(directory).encode(), runid.encode()))

    def report(self, blk, norm, who):
        """The averages(3) block report text."""
        blk = np.ascontiguousarray(blk, dtype=np.float64)
        need = ctypes.c_size_t()
        _capi.check(self.lib, self.lib.qmc2d_stats_report(self.p, self.system.ptr, _pd(blk), norm,
                                                          who.encode(), None, 0,
                                                          ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        _capi.check(self.lib, self.lib.qmc2d_stats_report(self.p, self.system.ptr, _pd(blk), norm,
                                                          who.encode(), buf, need.value, None))
        return buf.value.decode()

    def write_rhok(self, blk, norm, directory, runid):
        blk = np.ascontiguousarray(blk, dtype=np.float64)
        _capi.check(self.lib, self.lib.qmc2d_stats_write_rhok(self.p, self.system.ptr, _pd(blk),
                                                              norm, str(directory).encode(),
                                                              runid.encode()))


class Batch:
    """Populations (Handles on one device) advanced together through one
    CUDA graph per call (qmc2d_batch_*). Results equal the same vmc/dmc
    calls made handle by handle."""

    def __init__(self, handles):
        self.handles = list(handles)
        self.lib = self.handles[0].lib
        arr = (ctypes.c_void_p * len(self.handles))(*[h.h.value for h in self.handles])
        self.b = ctypes.c_void_p()
        _capi.check(self.lib, self.lib.qmc2d_batch_create(arr, len(self.handles),
                                                          ctypes.byref(self.b)))

    def close(self):
        if self.b:
            self.lib.qmc2d_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_lanes(self, lanes):
        """At most `lanes` populations in flight at a time (0: all)."""
        _capi.check(self.lib, self.lib.qmc2d_batch_set_lanes(self.b, lanes))

    def vmc(self, nstp, delta, mage=10 ** 9):
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(delta, float), (len(self.handles),)))
        _capi.check(self.lib, self.lib.qmc2d_batch_vmc(self.b, nstp, _pd(d), mage))

    def dmc(self, ngen, delta, etrial, mmult=2.0, mage=50):
        n = len(self.handles)
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(delta, float), (n,)))
        e = np.ascontiguousarray(np.broadcast_to(np.asarray(etrial, float), (n,)))
        _capi.check(self.lib, self.lib.qmc2d_batch_dmc(self.b, ngen, _pd(d), _pd(e), mmult, mage))


def tabc(handle, run, ntheta=None, resume=None, dmc_preequilibrate=None):
    """The twist loop of tabc (reptation.f:9559-9636): for ith, jth =
    1..ntheta (jth fastest) set the twist's wave vectors, then call
    run(handle, ith, jth); the walkers carry over from one twist to the next.

    resume = (ith, jth, iblk0) continues a restarted run the reference's way
    (:9567-9576): at the stored twist if iblk0 != 1, else at the next one.
    dmc_preequilibrate(handle), when given, runs before run() at every twist
    that is not resumed mid-way, like the reference's short DMC (one block of
    min(100, nstp) steps at delta/4, :9621-9632).
    Returns the list of twists visited."""
    system = handle.system
    nth = ntheta if ntheta is not None else system.s.ntheta
    if nth <= 0:
        raise ValueError("tabc: ntheta must be positive")
    i0, j0, mid = 1, 1, False
    if resume is not None:
        ith, jth, iblk0 = resume
        if iblk0 != 1:
            i0, j0, mid = ith, jth, True
        else:
            i0, j0 = ith + jth // nth, jth % nth + 1
    done = []
    for ith in range(i0, nth + 1):
        for jth in range(j0, nth + 1):
            system.set_twist(ith, jth)
            handle.update_twist()
            if dmc_preequilibrate is not None and not mid:
                dmc_preequilibrate(handle)
            mid = False
            run(handle, ith, jth)
            done.append((ith, jth))
        j0 = 1
    return done
