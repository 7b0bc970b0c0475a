"""qmc2d_compute_properties_noalloc against qmc2d_compute_properties_dev.

The no-allocation entry point serves callers that own all device memory
themselves (a host code with its own pool, a serving loop that must not
cudaMalloc between requests) and cannot create a handle. It must give the
same walkers' drift, Laplacian, properties and sign as the handle-based
entry point, on consecutive calls that reuse its fixed scratch array, on
the n26 deck and on the N=58 backflow deck (another table layout). A
configuration with two same-spin electrons at one point must come back
through qmc2d_compute_properties_noalloc_status as a zero pivot or a
non-finite result, and a shell whose determinants need device memory of
their own must be refused before launch. This file is collected last so
that a failure here comes after every other test.
"""
import ctypes
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _dev(t):
    return ctypes.c_void_p(t.data_ptr())


def _run_noalloc(q, sysobj, x, torch):
    lib = sysobj.lib
    nw, N, nt, np_ = x.shape[0], sysobj.N, sysobj.ntypes, sysobj.nprops
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    g = torch.zeros((nw, 2 * N), dtype=torch.float64, device="cuda")
    hl = torch.zeros((nw, nt), dtype=torch.float64, device="cuda")
    p = torch.zeros((nw, np_), dtype=torch.float64, device="cuda")
    s = torch.zeros(nw, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    code = lib.qmc2d_compute_properties_noalloc(sysobj.ptr, nw, _dev(xd), _dev(g), _dev(hl),
                                                _dev(p), _dev(s), ctypes.c_void_p(stream))
    q._capi.check(lib, code)
    torch.cuda.synchronize()
    return g.cpu().numpy(), hl.cpu().numpy(), p.cpu().numpy(), s.cpu().numpy()


def _run_handle(q, sysobj, x, torch):
    nw, N, nt, np_ = x.shape[0], sysobj.N, sysobj.ntypes, sysobj.nprops
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    g = torch.zeros((nw, 2 * N), dtype=torch.float64, device="cuda")
    hl = torch.zeros((nw, nt), dtype=torch.float64, device="cuda")
    p = torch.zeros((nw, np_), dtype=torch.float64, device="cuda")
    s = torch.zeros(nw, dtype=torch.float64, device="cuda")
    with q.Handle(sysobj, capacity=nw, seed=5) as h:
        torch.cuda.synchronize()  # inputs written before the handle's stream reads them
        h.compute_properties_dev(nw, _dev(xd), _dev(g), _dev(hl), _dev(p), _dev(s), None)
        torch.cuda.synchronize()  # device-wide: the handle's stream has finished
        out = (g.cpu().numpy(), hl.cpu().numpy(), p.cpu().numpy(), s.cpu().numpy())
    return out


def _close(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return (np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * scale)).max() < RTOL


def test_noalloc_matches_handle_entry_point(q, n26, n26_configs):
    import torch

    assert torch.cuda.is_available()
    for first in (0, 24):  # two calls in a row reuse the same scratch array
        x = n26_configs[first:first + 24].copy()
        ref = _run_handle(q, n26, x, torch)
        got = _run_noalloc(q, n26, x, torch)
        for a, b in zip(got, ref):
            assert _close(a, b)


def test_noalloc_rejects_oversized_batches(q, n26):
    import torch

    lib = n26.lib
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    code = lib.qmc2d_compute_properties_noalloc(n26.ptr, 65537, _dev(buf), _dev(buf), _dev(buf),
                                                _dev(buf), _dev(buf), None)
    assert code == q._capi.ERR_LIMIT
    assert b"at most 65536" in lib.qmc2d_last_error()


@pytest.fixture
def n58(q, tmp_path):
    tables = importlib.import_module("2degas_b200.tables")
    d = tables.make_run(os.path.join(tmp_path, "n58"), "c", nconf=16, seed=23,
                        **tables.CONFIGS["dmc_bf_n58_rs5"])
    s = q.System.read(d, "c")
    return s, s.read_configs(d, ".0", 0, 16)


def test_noalloc_second_deck(q, n58):
    import torch

    s, x = n58
    for first in (0, 8):  # two calls in a row on the N=58 layout
        ref = _run_handle(q, s, x[first:first + 8].copy(), torch)
        got = _run_noalloc(q, s, x[first:first + 8].copy(), torch)
        assert s.lib.qmc2d_compute_properties_noalloc_status(8, None) == q._capi.OK
        for a, b in zip(got, ref):
            assert _close(a, b)


def test_noalloc_reports_failed_walkers(q, n26, n26_configs):
    import torch

    x = n26_configs[:4].copy()
    x[2, 2:4] = x[2, 0:2]  # electrons 0 and 1 (both up) at one point
    lib = n26.lib
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    out = [torch.zeros(4 * k, dtype=torch.float64, device="cuda")
           for k in (2 * n26.N, n26.ntypes, n26.nprops, 1)]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    q._capi.check(lib, lib.qmc2d_compute_properties_noalloc(n26.ptr, 4, _dev(xd),
                                                            *[_dev(t) for t in out], stream))
    code = lib.qmc2d_compute_properties_noalloc_status(4, stream)
    assert code in (q._capi.ERR_SINGULAR, q._capi.ERR_NONFINITE)
    # the next call starts from clean status words
    xd.copy_(torch.tensor(n26_configs[:4], dtype=torch.float64))
    q._capi.check(lib, lib.qmc2d_compute_properties_noalloc(n26.ptr, 4, _dev(xd),
                                                            *[_dev(t) for t in out], stream))
    assert lib.qmc2d_compute_properties_noalloc_status(4, stream) == q._capi.OK


def test_noalloc_refuses_determinants_beyond_shared_memory(q, tmp_path):
    import torch

    tables = importlib.import_module("2degas_b200.tables")
    d = tables.make_run(os.path.join(tmp_path, "n98"), "c", n_up=49, n_down=49, rs=5.0,
                        backflow=(0.2, 5.0, 3.0), nknots=200, nconf=1, seed=3)
    s = q.System.read(d, "c")
    buf = torch.zeros(2 * s.nprops + 4 * s.N, dtype=torch.float64, device="cuda")
    code = s.lib.qmc2d_compute_properties_noalloc(s.ptr, 1, _dev(buf), _dev(buf), _dev(buf),
                                                  _dev(buf), _dev(buf), None)
    assert code == q._capi.ERR_LIMIT
    assert b"shared memory" in s.lib.qmc2d_last_error()
