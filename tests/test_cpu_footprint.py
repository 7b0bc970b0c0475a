"""qmc2d_footprint (host only): the device bytes a handle takes grow by the
per-walker determinant blocks exactly when the walker's determinants leave
shared memory (above 45 electrons per spin unpolarised, 49 polarised)."""
import importlib
import os

import pytest

q = importlib.import_module("2degas_b200")
tables = importlib.import_module("2degas_b200.tables")


def per_walker(tmp_path, nu, nd, rs=2.0):
    d = tables.make_run(os.path.join(tmp_path, f"d{nu}_{nd}"), "c", nu, nd, rs,
                        backflow=(0.2, rs, 0.6 * rs))
    s = q.System.read(d, "c")
    return (s.footprint(2048) - s.footprint(1024)) / 1024.0


@pytest.mark.parametrize("small,large", [((45, 45), (49, 49)), ((49, 0), (57, 0))])
def test_matrix_blocks_appear_beyond_shared_memory(tmp_path, small, large):
    a = per_walker(tmp_path, *small)
    b = per_walker(tmp_path, *large)
    n = large[0]
    spins = 2 if large[1] else 1
    # orbital matrix and inversion workspace of every spin (complex n x n
    # each) at least, on top of what the walker needs anyway
    assert b - a >= spins * 2 * 16 * n * n
    # the shared-memory shells carry no such block: growth there is the
    # walker records and move scratch only (well under one matrix per spin)
    assert a < 4 * 16 * 45 * 45 * 8


def test_largest_shells_fit_a_b200(tmp_path):
    # 4096 walkers of 81 + 81 and of 161 polarised stay within 180 GB
    for nu, nd in ((81, 81), (161, 0)):
        d = tables.make_run(os.path.join(tmp_path, f"b{nu}"), "c", nu, nd, 5.0,
                            backflow=(0.2, 5.0, 3.0))
        s = q.System.read(d, "c")
        assert s.footprint(4096) < 20e9
