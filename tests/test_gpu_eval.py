"""GPU parity of compute_properties against the CPU oracle.

The oracle restates the reference Fortran loop for loop (FP64); the device
path evaluates the same configurations through the C-ABI. Bar: 1e-10
relative on -ln psi, drift, Laplacian and every property (the FP64 path
sums in a different order, so results agree to round-off, not bit for bit).
"""
import numpy as np
import pytest

from variants import write_variant

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def close(a, b, rtol=RTOL):
    """|a-b| <= rtol * max(|b|, scale) elementwise, scale = max|b| of the array."""
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b) / np.maximum(np.abs(b), scale * 1e-3)
    return err.max()


def check_parity(q, oracle_cls, sysobj, x, rtol=RTOL):
    o = oracle_cls(sysobj)
    with q.Handle(sysobj, capacity=len(x), seed=7) as h:
        g, hl, p, s = h.compute_properties(x)
    for k in range(len(x)):
        go, ho, po, so, uf = o.compute_properties(x[k])
        assert close(g[k], go) < rtol, f"drift, config {k}"
        assert close(hl[k], ho) < rtol, f"laplacian, config {k}"
        po = po.copy()
        assert close(p[k], po) < rtol, f"props, config {k}: {np.abs(p[k]-po).max()}"
        assert s[k] == so


def test_n26_full_wavefunction(q, oracle_cls, n26, n26_configs):
    """u2 + u3 + backflow determinant at twist (1,1) + Ewald: the golden deck."""
    check_parity(q, oracle_cls, n26, n26_configs[:32])


def test_n26_gamma_point(q, oracle_cls, n26, n26_configs):
    n26.set_twist(0, 0)
    check_parity(q, oracle_cls, n26, n26_configs[:16])


@pytest.mark.parametrize("twist", [(2, 3), (4, 4)])
def test_n26_other_twists(q, oracle_cls, n26, n26_configs, twist):
    n26.set_twist(*twist)
    check_parity(q, oracle_cls, n26, n26_configs[16:24])


@pytest.mark.parametrize(
    "flags",
    [
        dict(backflow=False, ntwists=0),
        dict(u3=False, backflow=False, ntwists=0),
        dict(u2=False, u3=False, ntwists=0),
        dict(u3=False, v2=False, rhok=False),
        dict(v2=False, rhok=True),
    ],
)
def test_n26_variants(q, oracle_cls, tmp_path, n26_configs, flags):
    d = write_variant(tmp_path, "var", **flags)
    sysobj = q.System.read(d, "var")
    check_parity(q, oracle_cls, sysobj, n26_configs[:12])


def test_unwrapped_coordinates(q, oracle_cls, n26, n26_configs):
    """Positions far outside the cell (the stored walkers are not wrapped)."""
    x = n26_configs[:6].copy()
    x += np.array([3 * 9.03777677, -5 * 9.03777677] * (x.shape[1] // 2))
    check_parity(q, oracle_cls, n26, x)


def test_batch_sizes(q, n26, n26_configs):
    """The same configuration gives the same answer alone and in a batch."""
    x = n26_configs[:40]
    with q.Handle(n26, capacity=64) as h:
        _, _, pall, _ = h.compute_properties(x)
        _, _, pone, _ = h.compute_properties(x[17:18])
    assert np.array_equal(pall[17], pone[0])
