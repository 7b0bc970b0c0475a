"""qmc2d_compute_properties_noalloc against qmc2d_compute_properties_dev.

The no-allocation entry point serves callers that own all device memory
themselves (a host code with its own pool, a serving loop that must not
cudaMalloc between requests) and cannot create a handle. It must give the
same walkers' drift, Laplacian, properties and sign as the handle-based
entry point, on consecutive calls that reuse its fixed scratch array. This
file is collected last so that a failure here comes after every other test.
"""
import ctypes

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
