"""The reference's table generators restated in 2degas_b200.tables (tgen
with u2_ob_cos, u2_reatto and eta_yk; reptation.f:5007-5116, 6517-6590,
9474-9513), checked against the golden deck's own tables, which name their
generator and parameters in a trailer.

The trailers print each parameter to about 9 significant digits, while the
tables were built from the unrounded values, so the regenerated tables
agree to what that rounding allows: every column to 1e-6 of its largest
entry (measured: 1e-9 to 7e-8). A wrong form or a wrong joining point
misses by orders of magnitude more."""
import importlib
import os
import shutil

import numpy as np
import pytest

from conftest import N26

tables = importlib.import_module("2degas_b200.tables")


@pytest.mark.parametrize("name", ["n26.b", "n26.u2", "n26.u3"])
def test_generators_regenerate_the_golden_tables(name):
    rows, drt, routine, params = tables.read_table_file(os.path.join(N26, name))
    f, df = tables.GENERATORS[routine](params, drt, rows.shape[0] - 1)
    ours = tables.hermite_table(f, df, drt)
    scale = np.abs(rows).max(axis=0)
    assert np.all(np.abs(ours - rows) <= 1e-6 * scale), name
    assert np.array_equal(ours[-1], rows[-1])  # the zeroed last knot


def test_a_moved_join_misses():
    """A planted mistake: eta_yk built on nt + 1 knots (so the join at
    drt (5 nt / 6) moves by one knot) and cut back to nt + 1 rows misses the
    golden table 50 times beyond the 1e-6 bound of the regeneration test."""
    rows, drt, routine, params = tables.read_table_file(os.path.join(N26, "n26.b"))
    nt = rows.shape[0] - 1
    f, df = tables.eta_yk(params, drt, nt + 1)
    ours = tables.hermite_table(f[: nt + 1], df[: nt + 1], drt)
    assert np.abs(ours - rows).max() > 1e-5 * np.abs(rows).max()  # measured 5.2e-5


def test_tgen_tables_run_through_the_reader(q, oracle_cls, tmp_path):
    """The golden deck with its u2, u3 and backflow tables replaced by
    tgen's: the reader takes them, and the oracle's energies move by no more
    than the parameters' rounding does (1e-6 relative)."""
    d = tmp_path / "n26"
    shutil.copytree(N26, d)
    for name in ("n26.b", "n26.u2", "n26.u3"):
        rows, drt, routine, params = tables.read_table_file(os.path.join(N26, name))
        tables.tgen(str(d / name), routine, params, drt, rows.shape[0] - 1)
    s0 = q.System.read(N26, "n26")
    s1 = q.System.read(d, "n26")
    x = s0.read_configs(N26, ".0", 0, 4)
    o0, o1 = oracle_cls(s0), oracle_cls(s1)
    for k in range(len(x)):
        _, _, p0, _, _ = o0.compute_properties(x[k])
        _, _, p1, _, _ = o1.compute_properties(x[k])
        assert abs(p1[0] - p0[0]) <= 1e-6 * abs(p0[0])
        assert abs(p1[1] - p0[1]) <= 1e-6 * max(1.0, abs(p0[1]))


def test_krlv_regenerates_the_golden_k_list():
    """krlv for the n26 cell (L = sqrt(26 pi), |n| <= 6) gives n26.k's 56
    vectors in its order, to the file's 9 printed digits; the order within
    the |n|^2 = 25 shell comes from the floating-point norm comparisons."""
    import math

    k = np.loadtxt(os.path.join(N26, "n26.k"))
    ours = tables.krlv(math.sqrt(26 * math.pi), 6.0)
    assert ours.shape == k.shape
    assert np.abs(ours - k).max() <= 2e-9 * np.abs(k).max()
