"""The product's run-directory reader (qmc2d_system_read, csrc/input.cpp and
system.cpp) against the oracle's own reader (oracle/oracle_input.c), field
by field: every scalar of the system, each table's knots and k-space
trailer, the k vectors, the orbital wave vectors at several twists, the
property layout and the estimator records, and the configurations that
read_conf returns. The two are written independently from reptation.f's
input, readwords, t_read, kread, twistg and read_conf, so that a misread
on either side shows up here and in every parity test instead of hitting
the device path and its checker alike.

Decks: the reference's n26 run directory, its keyword variants, and the
synthetic decks of every benchmark state point (plain split and the
setup program's optimised breakup, with and without twists)."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import N26
from oracle_lib import OracleSystem
from variants import write_variant

SCALARS = ["ndim", "ntypes", "nptot", "npnorm", "nk", "ngvec", "drt", "drti", "drti2",
           "ntables", "nrhok", "v0", "adrift", "delta", "ecut", "value_ecut", "ntheta", "ith",
           "jth", "ibckf", "gstorto", "wpiu", "nodalaction", "rejection", "n_scalar_props",
           "n_props", "jrhok", "ref_underflow_return", "nmstar", "ncmass", "nitc"]


def _view(q, osys):
    """The oracle's qmc2d_system seen through the ctypes layout of
    include/qmc2d.h (both readers fill that struct)."""
    return ctypes.cast(osys.ptr, ctypes.POINTER(q._capi.System)).contents


def _arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy() if n > 0 else np.zeros(0)


def compare(q, prod, osys):
    a, b = prod.s, _view(q, osys)
    for f in SCALARS:
        assert getattr(a, f) == getattr(b, f), f
    nt = a.ntypes
    for f in ("np", "ipfrst", "hbs2m", "irhok"):
        assert list(getattr(a, f))[:nt] == list(getattr(b, f))[:nt], f
    for f in ("el", "eli", "seed"):
        assert list(getattr(a, f)) == list(getattr(b, f)), f
    for t in range(nt):
        assert a.type_name[t].value == b.type_name[t].value
        assert a.x_file[t].value == b.x_file[t].value
    for f in ("iu2", "iu3", "iub", "iv2"):
        for i in range(nt):
            for j in range(nt):
                assert getattr(a, f)[i][j] == getattr(b, f)[i][j], (f, i, j)
    assert np.array_equal(_arr(a.kvec, 2 * a.nk), _arr(b.kvec, 2 * b.nk))
    assert np.array_equal(_arr(a.gvec, 2 * a.ngvec), _arr(b.gvec, 2 * b.ngvec))
    for t in range(a.ntables):
        ta, tb = a.tables[t], b.tables[t]
        assert ta.name == tb.name
        for f in ("ngrid", "tail", "iexp", "nk_ewald"):
            assert getattr(ta, f) == getattr(tb, f), (t, f)
        assert np.array_equal(_arr(ta.ut, 4 * (ta.ngrid + 1)), _arr(tb.ut, 4 * (tb.ngrid + 1)))
        if ta.nk_ewald > 0:
            assert np.array_equal(_arr(ta.vk, ta.nk_ewald + 1), _arr(tb.vk, tb.nk_ewald + 1))
    for f, n in (("mstar_record", a.nmstar), ("cmass_record", a.ncmass), ("itc_record", a.nitc)):
        for i in range(n):
            assert getattr(a, f)[i].value.split() == getattr(b, f)[i].value.split(), f


def _decks(tmp_path):
    tables = importlib.import_module("2degas_b200.tables")
    out = [(N26, "n26", ".0")]
    for name, kw in (("plain", {}), ("nobf", dict(backflow=False)), ("nou3", dict(u3=False)),
                     ("gamma", dict(ntwists=0)), ("nov2", dict(v2=False, rhok=False)),
                     ("est", dict(extra=("  mstar up 2", "  cmass up 1 2 4",
                                         "  itc elocal elocal 1")))):
        d = os.path.join(tmp_path, name)
        os.makedirs(d)
        write_variant(d, "v", **kw)
        out.append((d, "v", ".0"))
    for name, cfg in tables.CONFIGS.items():
        for extra in ({}, dict(twist=True), dict(ewald="fitpn")):
            tag = name + "".join(f"_{k}" for k in extra)
            d = tables.make_run(os.path.join(tmp_path, tag), "c", nconf=3, seed=5,
                                **dict(cfg, **extra))
            out.append((d, "c", ".0"))
    return out


def test_readers_agree_field_by_field(q, tmp_path):
    for d, runid, suffix in _decks(tmp_path):
        prod = q.System.read(d, runid)
        osys = OracleSystem.read(d, runid)
        compare(q, prod, osys)
        xa = prod.read_configs(d, suffix, 1, 2)
        xb = osys.read_configs(d, suffix, 1, 2)
        assert xa.shape == xb.shape and np.array_equal(xa, xb), d


@pytest.mark.parametrize("twist", [(0, 0), (1, 1), (2, 3), (4, 4), (3, 1)])
def test_readers_agree_on_twisted_wave_vectors(q, twist):
    prod = q.System.read(N26, "n26")
    osys = OracleSystem.read(N26, "n26")
    prod.set_twist(*twist)
    osys.set_twist(*twist)
    compare(q, prod, osys)


def test_both_readers_refuse_the_same_decks(q, tmp_path):
    """Keywords outside the walker path and a backflow determinant whose
    orbital wave vectors the reference never builds (ibckf 0 at Gamma)."""
    cases = {
        "gofr": dict(extra=("  gofr up up 2",)),
        "sites": dict(extra=("  sites s 1 n26.up.x",)),
        "ibckf0": None,
    }
    for name, kw in cases.items():
        d = os.path.join(tmp_path, name)
        os.makedirs(d)
        if kw is None:
            write_variant(d, "v", ntwists=0)
            sy = open(os.path.join(d, "v.sy")).read().replace(" 1 n26.b", " 0 n26.b")
            open(os.path.join(d, "v.sy"), "w").write(sy)
        else:
            write_variant(d, "v", **kw)
        with pytest.raises(q.QMCError):
            q.System.read(d, "v")
        with pytest.raises(RuntimeError):
            OracleSystem.read(d, "v")
