"""The run-directory reader (input/t_read/kread/read_conf) and the table
generator, on CPU."""
import importlib
import math
import os

import numpy as np
import pytest

from conftest import N26
from variants import write_variant


def test_n26_system(n26):
    s = n26.s
    assert (s.ntypes, s.nptot, s.npnorm) == (2, 26, 26)
    assert list(s.np[:2]) == [13, 13] and list(s.ipfrst[:2]) == [0, 13]
    assert s.nk == 56 and s.ngvec == 113
    assert s.ntables == 4
    names = [s.tables[i].name.decode() for i in range(4)]
    assert names == ["n26.u2", "n26.u3", "n26.b", "n26.v"]
    assert all(s.tables[i].ngrid == 500 for i in range(4))
    assert s.tables[3].nk_ewald == 56 and s.tables[3].iexp == 1 and s.tables[3].tail == 0.0
    assert abs(s.drt - 0.00903777677) < 1e-15 and abs(s.drti2 - 2 / s.drt ** 2) < 1e-6
    assert s.v0 == -69.0949679 and s.el[0] == 9.03777677
    assert s.ntheta == 4 and (s.ith, s.jth) == (1, 1)
    assert list(s.irhok[:2]) == [1, 2] and s.n_props == 14 + 2 * 2 * 56
    assert list(s.seed) == [3535, 3467, 3262, 1549]
    # first knot of n26.u2 and first v_k
    assert s.tables[0].ut[0] == 0.115781977594e01 and s.tables[0].ut[3] == -0.135165358160e-07
    assert s.tables[3].vk[0] == 0.0805122668 and s.tables[3].vk[56] == 0.0


def test_twist_orbitals(n26):
    s = n26.s
    L = s.el[0]
    k = np.ctypeslib.as_array(s.kvec, shape=(2 * s.nk,)).reshape(-1, 2)
    g = n26.gvec()
    th = 2 * math.pi / L / 4 * np.array([1.0, 1.0])
    want = np.concatenate([[th], k + th, -k + th])
    norms = (g ** 2).sum(1)
    assert np.all(np.diff(norms) >= 0)
    assert np.allclose(np.sort(norms), np.sort((want ** 2).sum(1)))
    assert np.allclose(g[0], th)
    n26.set_twist(0, 0)
    g0 = n26.gvec()
    assert np.all(g0[0] == 0) and np.allclose(g0[1], k[0]) and np.allclose(g0[2], -k[0])


def test_read_configs(n26):
    x = n26.read_configs(N26, ".0", 0, 3)
    first = [float(v) for v in open(os.path.join(N26, "n26.up.x.0")).readline().split()]
    assert x.shape == (3, 52) and list(x[0, :2]) == first
    down = open(os.path.join(N26, "n26.down.x.0")).read().split()
    assert x[1, 26] == float(down[2 * 13])  # second configuration, first down electron
    x2 = n26.read_configs(N26, ".0", 62, 10)
    assert x2.shape[0] == 2  # 64 stored configurations


@pytest.mark.parametrize(
    "extra,code",
    [(("  gofr up up 1",), 4), (("  sites s 1 f",), 4), (("", ), 3)],
)
def test_reader_rejects(q, tmp_path, extra, code):
    d = write_variant(tmp_path, "bad", extra=extra)
    with pytest.raises(q.QMCError) as e:
        q.System.read(d, "bad")
    assert e.value.code == code


def test_partial_table_set_rejected(q, tmp_path):
    d = write_variant(tmp_path, "ok")
    txt = open(os.path.join(d, "ok.sy")).read().replace("  u2 up down n26.u2\n", "")
    open(os.path.join(d, "part.sy"), "w").write(txt)
    with pytest.raises(q.QMCError) as e:
        q.System.read(d, "part")
    assert e.value.code == 4


def test_missing_file(q, tmp_path):
    with pytest.raises(q.QMCError) as e:
        q.System.read(str(tmp_path), "nothere")
    assert e.value.code == 2


def test_generated_tables_round_trip(q, tmp_path):
    """Tables written by the generator (rows wider than 80 columns) read back
    exactly and interpolate the generating functions."""
    T = importlib.import_module("2degas_b200.tables")
    d = T.make_run(str(tmp_path), "g", nconf=2, **T.CONFIGS["dmc_bf_n58_rs5"])
    s = q.System.read(d, "g")
    assert s.N == 58 and s.s.ntables == 3
    u2 = s.s.tables[0]
    rows = np.ctypeslib.as_array(u2.ut, shape=(4 * (u2.ngrid + 1),)).reshape(-1, 4)
    lines = open(os.path.join(d, "g.u2")).read().splitlines()
    assert np.array_equal(rows[5], [float(v) for v in lines[6].split()])
    drt = s.s.drt
    rs = 5.0
    a = math.sqrt(rs)
    L = s.s.el[0]
    rc = L / 2

    def u(x):
        return (1 - math.exp(-a * x)) / x

    du_c = (a * rc * math.exp(-a * rc) - (1 - math.exp(-a * rc))) / rc ** 2
    for r in (0.3, 1.7, 4.2):
        i = int(r / drt)
        rm = (r - i * drt) / drt
        c = rows[i]
        f = c[0] + rm * (c[1] + rm * (c[2] + rm * c[3]))
        assert abs(f - (u(r) - u(rc) - (r - rc) * du_c)) < 1e-9
    gv = s.gvec()[:29]
    assert len(np.unique(np.round((gv ** 2).sum(1), 9))) == 7  # closed shells 0,1,2,4,5,8,9


def test_closed_shells():
    T = importlib.import_module("2degas_b200.tables")
    assert T.closed_shells()[:9] == [1, 5, 9, 13, 21, 25, 29, 37, 45]
