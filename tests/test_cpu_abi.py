"""The C-ABI library on CPU: it loads, exports what include/qmc2d.h
declares, and fails cleanly (no crash, an error code) without a GPU."""
import ctypes
import importlib
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "qmc2d.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(qmc2d_\w+)\s*\(", hdr)))


def test_header_symbols_exported(q):
    lib = ctypes.CDLL(q._capi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header(q):
    assert set(declared_functions()) == set(q._capi.SIGNATURES)


def test_no_gpu_is_an_error_not_a_crash(q, n26, has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(q.QMCError) as e:
        q.Handle(n26, capacity=4)
    assert e.value.code == q._capi.ERR_CUDA


def test_flops_formula():
    """The per-move flop counts quoted for the benchmark configurations."""
    bench = importlib.import_module("bench")
    f26 = bench.flops_per_move(26, [13, 13], 56, 1, 1)
    f58 = bench.flops_per_move(58, [29, 29], 56, 1, 1)
    f26p = bench.flops_per_move(26, [13, 13], 56, 0, 0)
    assert abs(f26 / 0.60e6 - 1) < 0.05
    assert abs(f58 / 5.75e6 - 1) < 0.05
    assert abs(f26p / 0.08e6 - 1) < 0.15
