"""The block drivers (vmc, dmc, rmc loops with averages(3)'s output):
their statistics equal the same calls made by hand, the trial energy of dmc
follows the cumulative mean, and every block writes the reference's files."""
import importlib
import os

import numpy as np
import pytest

from variants import write_variant

pytestmark = pytest.mark.gpu

drv = importlib.import_module("2degas_b200.drivers")


def test_vmc_driver(q, n26, n26_configs, tmp_path):
    x = n26_configs[:16]
    with q.Handle(n26, capacity=16, seed=5) as h:
        h.population_set(x)
        st = drv.vmc(h, 2, 5, 0.05, out=tmp_path, runid="v", log=None)
    with q.Handle(n26, capacity=16, seed=5) as h:
        h.population_set(x)
        ref = q.Stats(n26)
        for _ in range(2):
            h.block_reset()
            h.vmc(5, 0.05, 10)
            ref.add_block(*h.block_get())
    np.testing.assert_array_equal(st.get()[0], ref.get()[0])
    names = set(os.listdir(tmp_path))
    assert {"v.res", "v.rhok_up", "v.rhok_down", "n26.up.x.res.0", "n26.down.x.res.0"} <= names


def test_dmc_driver_trial_energy(q, n26, n26_configs, tmp_path):
    with q.Handle(n26, capacity=32, seed=6) as h:
        h.population_set(n26_configs[:32])
        st, et = drv.dmc(h, 3, 4, 0.02, -0.44, out=tmp_path, runid="d", log=None)
    mean, err, norm, nb = st.get()
    assert nb == 3 and et == mean[0]
    assert open(tmp_path / "d.res").readline().split()[1] == "dmc"


def test_rmc_driver_with_estimators(q, n26_configs, tmp_path):
    recs = ("  mstar up 1", "  cmass down 2 1", "  itc 1 elocal 1 elocal 1")
    d = tmp_path / "deck"
    d.mkdir()
    s = q.System.read(write_variant(d, "est", extra=recs), "est")
    ntau, nrep = 12, 3
    est = s.rmc_estimators_setup(ntau, 1)
    out = tmp_path / "out"
    out.mkdir()
    with q.Handle(s, capacity=nrep, seed=7) as h:
        h.rmc_init(nrep, n26_configs[: nrep * ntau], ntau, 1, 2, 0.02, -0.44, 1000, 1000)
        st, est_st = drv.rmc(h, 2, 3, est=est, out=out, runid="r", log=None)
    assert st.get()[3] == 2 and est_st.get()[3] == 2
    names = set(os.listdir(out))
    assert {"r.res", "r.mstar_up", "r.z_cmass_down", "r.cmass_down", "r.elocal_elocal"} <= names
    assert len(open(out / "r.z_cmass_down").read().splitlines()) == 2 * 4
