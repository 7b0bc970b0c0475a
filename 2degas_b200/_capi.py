"""ctypes view of the C-ABI in include/qmc2d.h (libqmc2d.so).

The library is built in-tree by ``2degas_b200/build.py`` (nvcc, sm_100a).
Loading fails loudly if it is missing: there is no CPU fallback.
"""
import ctypes
import os
from ctypes import POINTER, c_char, c_double, c_int, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libqmc2d.so")

MAX_TYPES = 2
MAX_TABLES = 16
NAME_LEN = 64
MAX_EST = 4
RECORD_LEN = 256
MAX_ADD = 4
MAX_CMSKIP = 8

# status codes (enum qmc2d_status)
OK = 0
ERR_ARG = 1
ERR_IO = 2
ERR_PARSE = 3
ERR_UNSUPPORTED = 4
ERR_CUDA = 5
ERR_NOMEM = 6
ERR_SINGULAR = 7
ERR_NONFINITE = 8
ERR_POPULATION = 9
ERR_LIMIT = 10
ERR_STACK = 11

# kernels for qmc2d_profile_get
(KERNEL_MOVE, KERNEL_BRANCH, KERNEL_GATHER, KERNEL_EVAL, KERNEL_RMC, KERNEL_PAIRS,
 KERNEL_SINGLE, KERNEL_ORB_INV) = range(8)
PRECISION_FP64, PRECISION_MIXED = 0, 1

# property indices (0-based; reptation.f:577-637)
JETOT, JLTF, JACC, JPOT0, JKIN0, JE2, JGG = range(7)


def jpot(nt, it):
    return 7 + it


def jkin(nt, it):
    return 7 + nt + it


def jun(nt, it):
    return 7 + 2 * nt + it


def jefp(nt):
    return 7 + 3 * nt


class Table(ctypes.Structure):
    _fields_ = [
        ("name", c_char * NAME_LEN),
        ("ngrid", c_int),
        ("ut", POINTER(c_double)),
        ("tail", c_double),
        ("iexp", c_int),
        ("nk_ewald", c_int),
        ("vk", POINTER(c_double)),
    ]


_I2x2 = (c_int * MAX_TYPES) * MAX_TYPES


class System(ctypes.Structure):
    _fields_ = [
        ("ndim", c_int),
        ("ntypes", c_int),
        ("type_name", (c_char * NAME_LEN) * MAX_TYPES),
        ("x_file", (c_char * NAME_LEN) * MAX_TYPES),
        ("np", c_int * MAX_TYPES),
        ("ipfrst", c_int * MAX_TYPES),
        ("nptot", c_int),
        ("npnorm", c_int),
        ("hbs2m", c_double * MAX_TYPES),
        ("el", c_double * 2),
        ("eli", c_double * 2),
        ("nk", c_int),
        ("kvec", POINTER(c_double)),
        ("ngvec", c_int),
        ("gvec", POINTER(c_double)),
        ("drt", c_double),
        ("drti", c_double),
        ("drti2", c_double),
        ("ntables", c_int),
        ("tables", Table * MAX_TABLES),
        ("iu2", _I2x2),
        ("iu3", _I2x2),
        ("iub", _I2x2),
        ("iv2", _I2x2),
        ("irhok", c_int * MAX_TYPES),
        ("nrhok", c_int),
        ("v0", c_double),
        ("adrift", c_double),
        ("delta", c_double),
        ("ecut", c_int),
        ("value_ecut", c_double),
        ("ntheta", c_int),
        ("ith", c_int),
        ("jth", c_int),
        ("ibckf", c_int),
        ("gstorto", c_int),
        ("wpiu", c_int),
        ("nodalaction", c_int),
        ("rejection", c_int),
        ("seed", c_int * 4),
        ("n_scalar_props", c_int),
        ("n_props", c_int),
        ("jrhok", c_int),
        ("ref_underflow_return", c_int),
        ("nmstar", c_int),
        ("ncmass", c_int),
        ("nitc", c_int),
        ("mstar_record", (c_char * RECORD_LEN) * MAX_EST),
        ("cmass_record", (c_char * RECORD_LEN) * MAX_EST),
        ("itc_record", (c_char * RECORD_LEN) * MAX_EST),
    ]


class RmcEstimators(ctypes.Structure):
    _fields_ = [
        ("ntau", c_int), ("ntauskip", c_int),
        ("nmstar", c_int), ("mstar_type", c_int * MAX_EST), ("mstar_tau_skip", c_int * MAX_EST),
        ("ncmass", c_int), ("cmass_type", c_int * MAX_EST), ("cmass_tau_skip", c_int * MAX_EST),
        ("cmass_nskip", c_int), ("cmass_ntauskip", (c_int * MAX_CMSKIP) * MAX_EST),
        ("nitc", c_int), ("itc_add", c_int * MAX_EST), ("itc_start", (c_int * MAX_ADD) * MAX_EST),
        ("itc_count", c_int * MAX_EST), ("itc_complex", c_int * MAX_EST),
        ("jtc_add", c_int * MAX_EST), ("jtc_start", (c_int * MAX_ADD) * MAX_EST),
        ("jtc_complex", c_int * MAX_EST), ("itc_tau_skip", c_int * MAX_EST),
        ("jcmass_z", c_int), ("jcmass_d", c_int), ("jmstar", c_int), ("jitc", c_int),
        ("nvalues", c_int),
    ]


class Options(ctypes.Structure):
    _fields_ = [("capacity", c_int), ("device", c_int), ("seed", c_uint64)]


class Counters(ctypes.Structure):
    _fields_ = [
        ("accepted", c_double),
        ("proposed", c_double),
        ("forced", c_double),
        ("sign_changes", c_double),
        ("max_weight_capped", c_double),
    ]


class RmcParams(ctypes.Structure):
    _fields_ = [
        ("ntau", c_int),
        ("ntauskip", c_int),
        ("mdelta", c_int),
        ("delta", c_double),
        ("etrial", c_double),
        ("mage", c_int),
        ("mage_r", c_int),
    ]


PD = POINTER(c_double)
PI = POINTER(c_int)
SYSP = POINTER(System)

# name -> (restype, argtypes); every symbol include/qmc2d.h declares.
SIGNATURES = {
    "qmc2d_system_read": (c_int, [ctypes.c_char_p, ctypes.c_char_p, POINTER(SYSP)]),
    "qmc2d_system_free": (None, [SYSP]),
    "qmc2d_system_set_twist": (c_int, [SYSP, c_int, c_int]),
    "qmc2d_read_configs": (c_int, [SYSP, ctypes.c_char_p, ctypes.c_char_p, c_int, c_int, PD,
                                   POINTER(c_int)]),
    "qmc2d_last_error": (ctypes.c_char_p, []),
    "qmc2d_version": (ctypes.c_char_p, []),
    "qmc2d_create": (c_int, [SYSP, POINTER(Options), POINTER(c_void_p)]),
    "qmc2d_destroy": (c_int, [c_void_p]),
    "qmc2d_compute_properties": (c_int, [c_void_p, c_int, PD, PD, PD, PD, PD]),
    "qmc2d_compute_properties_dev": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p]),
    "qmc2d_compute_properties_noalloc": (c_int, [SYSP, c_int, c_void_p, c_void_p, c_void_p,
                                                 c_void_p, c_void_p, c_void_p]),
    "qmc2d_compute_properties_noalloc_status": (c_int, [c_int, c_void_p]),
    "qmc2d_vmc_single": (c_int, [c_void_p, c_int, c_double, c_int]),
    "qmc2d_set_inversion": (c_int, [c_void_p, c_int]),
    "qmc2d_set_pair_lanes": (c_int, [c_void_p, c_int]),
    "qmc2d_set_autotune_scope": (c_int, [c_void_p, c_int]),
    "qmc2d_set_move_inversion": (c_int, [c_void_p, c_int]),
    "qmc2d_get_move_inversion": (c_int, [c_void_p, PI]),
    "qmc2d_get_pair_lanes": (c_int, [c_void_p, PI]),
    "qmc2d_rmc_set_launch": (c_int, [c_void_p, c_int]),
    "qmc2d_get_launch": (c_int, [c_void_p, PI, PI, PI]),
    "qmc2d_dmc_weights": (c_int, [c_void_p, c_int, c_double, c_double, c_double, c_int, PD]),
    "qmc2d_comb_plan": (c_int, [c_int, c_int, PD, c_uint64, ctypes.c_uint32, c_int, PI, PI, PI,
                                PI, PI, PI, PI, PI]),
    "qmc2d_record_len": (c_int, [c_void_p, PI]),
    "qmc2d_records_pack": (c_int, [c_void_p, c_int, PI, c_void_p, c_void_p]),
    "qmc2d_records_unpack": (c_int, [c_void_p, c_int, PI, c_void_p, c_void_p]),
    "qmc2d_population_resample": (c_int, [c_void_p, PI]),
    "qmc2d_single_drift": (c_int, [c_void_p, PD]),
    "qmc2d_compute_properties_dev_status": (c_int, [c_void_p, c_int, c_void_p]),
    "qmc2d_population_set": (c_int, [c_void_p, c_int, PD]),
    "qmc2d_population_size": (c_int, [c_void_p, POINTER(c_int)]),
    "qmc2d_population_get": (c_int, [c_void_p, PD, PD, PD, PD, PD, PD]),
    "qmc2d_population_load_async": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p]),
    "qmc2d_population_load": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p]),
    "qmc2d_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
    "qmc2d_profile": (c_int, [c_void_p, c_int]),
    "qmc2d_profile_get": (c_int, [c_void_p, c_int, PD, POINTER(ctypes.c_long)]),
    "qmc2d_phase_timers": (c_int, [c_void_p, c_int, POINTER(ctypes.c_ulonglong)]),
    "qmc2d_block_reset": (c_int, [c_void_p]),
    "qmc2d_block_get": (c_int, [c_void_p, PD, PD]),
    "qmc2d_counters_get": (c_int, [c_void_p, POINTER(Counters)]),
    "qmc2d_update_twist": (c_int, [c_void_p, SYSP]),
    "qmc2d_set_precision": (c_int, [c_void_p, c_int]),
    "qmc2d_footprint": (c_int, [SYSP, c_int, ctypes.POINTER(c_uint64)]),
    "qmc2d_set_dmc_ecut": (c_int, [c_void_p, c_double]),
    "qmc2d_rmc_estimators_setup": (c_int, [SYSP, c_int, c_int, POINTER(RmcEstimators)]),
    "qmc2d_rmc_path_estimators": (c_int, [c_void_p, POINTER(RmcEstimators), PD]),
    "qmc2d_set_launch": (c_int, [c_void_p, c_int, c_int]),
    "qmc2d_autotune": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), PD]),
    "qmc2d_batch_create": (c_int, [POINTER(c_void_p), c_int, POINTER(c_void_p)]),
    "qmc2d_batch_destroy": (c_int, [c_void_p]),
    "qmc2d_batch_set_lanes": (c_int, [c_void_p, c_int]),
    "qmc2d_batch_vmc": (c_int, [c_void_p, c_int, PD, c_int]),
    "qmc2d_batch_dmc": (c_int, [c_void_p, c_int, PD, PD, c_double, c_int]),
    "qmc2d_stats_create": (c_int, [c_int, POINTER(c_void_p)]),
    "qmc2d_stats_write_estimators": (c_int, [c_void_p, SYSP, POINTER(RmcEstimators), PD, c_double,
                                             ctypes.c_char_p, ctypes.c_char_p]),
    "qmc2d_stats_destroy": (c_int, [c_void_p]),
    "qmc2d_stats_add_block": (c_int, [c_void_p, PD, c_double]),
    "qmc2d_stats_get": (c_int, [c_void_p, PD, PD, PD, POINTER(c_int)]),
    "qmc2d_stats_report": (c_int, [c_void_p, SYSP, PD, c_double, ctypes.c_char_p,
                                   ctypes.c_char_p, ctypes.c_size_t,
                                   POINTER(ctypes.c_size_t)]),
    "qmc2d_stats_write_rhok": (c_int, [c_void_p, SYSP, PD, c_double, ctypes.c_char_p,
                                       ctypes.c_char_p]),
    "qmc2d_write_conf": (c_int, [c_void_p, SYSP, ctypes.c_char_p, c_int]),
    "qmc2d_restart_write": (c_int, [c_void_p, SYSP, c_void_p, c_int, ctypes.c_char_p,
                                    ctypes.c_char_p, ctypes.c_char_p, c_int]),
    "qmc2d_restart_read": (c_int, [c_void_p, SYSP, c_void_p, ctypes.c_char_p, ctypes.c_char_p,
                                   ctypes.c_char_p, c_int, POINTER(c_int), PD]),
    "qmc2d_restart_read_rmc": (c_int, [c_void_p, SYSP, c_void_p, POINTER(RmcParams),
                                       ctypes.c_char_p, ctypes.c_char_p, c_int, POINTER(c_int)]),
    "qmc2d_vmc": (c_int, [c_void_p, c_int, c_double, c_int]),
    "qmc2d_dmc": (c_int, [c_void_p, c_int, c_int, c_double, c_double, c_double, c_int]),
    "qmc2d_rmc_init": (c_int, [c_void_p, c_int, POINTER(RmcParams), PD]),
    "qmc2d_rmc": (c_int, [c_void_p, c_int]),
    "qmc2d_rmc_get_path": (c_int, [c_void_p, c_int, PD, PD]),
}

_lib = None


def load(path=None):
    """Load libqmc2d.so and attach the C signatures. Raises OSError if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libqmc2d.so not built ({p}); run 2degas_b200/build.py")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class QMCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"qmc2d error {code}: {msg}")
        self.code = code


def check(lib, code):
    if code != OK:
        raise QMCError(code, lib.qmc2d_last_error().decode(errors="replace"))
    return code
