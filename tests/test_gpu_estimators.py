"""qmc2d_rmc_path_estimators on the GPU against the oracle's numpy
restatement of path_props (reptation.f:1578-1737) on the same paths: the
reptiles' paths are read back with qmc2d_rmc_get_path and the mean over
reptiles of the restated estimators must match to 1e-10 relative."""
import os
import sys

import numpy as np
import pytest

from variants import write_variant

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
from path_estimators import path_estimators  # noqa: E402

RECORDS = ("  mstar up 1", "  mstar down 2", "  cmass up 2 2 1 3", "  cmass down 2 2 0 4",
           "  itc 1 rhok_up complex 1 rhok_up conjg 2", "  itc 2 elocal epot 1 ekin 1")


def test_estimators_match_the_restatement(q, n26_configs, tmp_path):
    s = q.System.read(write_variant(tmp_path, "est", extra=RECORDS), "est")
    nrep, ntau, ntauskip = 4, 20, 2
    est = s.rmc_estimators_setup(ntau, ntauskip)
    info = dict(ipfrst=list(s.s.ipfrst), np=list(s.s.np), eli=list(s.s.eli))
    x0 = np.concatenate([n26_configs[(r * 5) % 40:(r * 5) % 40 + ntau] for r in range(nrep)])
    with q.Handle(s, capacity=nrep, seed=17) as h:
        h.rmc_init(nrep, x0, ntau, ntauskip, 2, 0.02, -0.44, 1000, 1000)
        for nstp in (0, 3, 1):
            h.rmc(nstp)
            got = h.rmc_estimators(est)
            want = np.zeros(est.nvalues)
            for r in range(nrep):
                x, p = h.rmc_get_path(r, ntau)
                want += path_estimators(est, info, x, p)
            want /= nrep
            # relative, with a floor for entries that cancel to near zero (the
            # device fuses multiply-adds, numpy does not)
            scale = np.maximum(np.abs(want), 1e-3 * np.abs(want).max())
            assert np.all(np.abs(got - want) <= 1e-10 * scale), nstp


def test_estimators_need_the_same_path_length(q, n26_configs, tmp_path):
    s = q.System.read(write_variant(tmp_path, "est", extra=RECORDS[:1]), "est")
    est = s.rmc_estimators_setup(16, 2)
    with q.Handle(s, capacity=2, seed=1) as h:
        with pytest.raises(q.QMCError):
            h.rmc_estimators(est)  # no reptiles yet
        h.rmc_init(2, n26_configs[:40], 20, 2, 2, 0.02, -0.44, 1000, 1000)
        with pytest.raises(q.QMCError):
            h.rmc_estimators(est)
