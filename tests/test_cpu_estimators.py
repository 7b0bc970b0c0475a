"""Setup of the reptation path estimators from the deck's 'mstar', 'cmass'
and 'itc' records (mstar_setup, cmass_setup, itc_setup;
reptation.f:1378-1553): fields, the estimator vector's layout, and the
records that are rejected. Host only."""
import os

import pytest

from variants import write_variant

RECORDS = ("  mstar up 1", "  mstar down 2", "  cmass up 2 2 1 3",
           "  itc 1 rhok_up complex 1 rhok_up conjg 2", "  itc 2 elocal epot 1 ekin 1")


def test_records_and_layout(q, tmp_path):
    s = q.System.read(write_variant(tmp_path, "est", extra=RECORDS), "est")
    assert (s.s.nmstar, s.s.ncmass, s.s.nitc) == (2, 1, 2)
    assert s.s.itc_record[0].value.decode() == "1 rhok_up complex 1 rhok_up conjg 2"
    e = s.rmc_estimators_setup(20, 2)
    nk = s.s.nk
    assert (e.mstar_type[0], e.mstar_tau_skip[0], e.mstar_type[1], e.mstar_tau_skip[1]) == \
        (0, 1, 1, 2)
    assert (e.cmass_type[0], e.cmass_tau_skip[0], e.cmass_nskip) == (0, 2, 2)
    assert list(e.cmass_ntauskip[0][:2]) == [1, 3]
    assert (e.itc_add[0], e.itc_count[0], e.itc_complex[0], e.jtc_complex[0]) == (1, 2 * nk, 1, -1)
    assert e.itc_start[0][0] == s.s.jrhok and e.jtc_start[0][0] == s.s.jrhok
    assert (e.itc_add[1], list(e.itc_start[1][:2]), e.jtc_add[1], e.jtc_start[1][0]) == \
        (2, [0, 3], 1, 4)
    assert (e.itc_complex[1], e.itc_count[1], e.itc_tau_skip[1]) == (0, 1, 1)
    # cmass z (4), cmass diffusion (18/2 + 14/2), mstar (16 + 8), itc (8*2nk + 16)
    assert (e.jcmass_z, e.jcmass_d, e.jmstar, e.jitc) == (0, 4, 20, 44)
    assert e.nvalues == 44 + 8 * 2 * nk + 16


def test_cmass_with_one_skip_takes_ntauskip(q, tmp_path):
    s = q.System.read(write_variant(tmp_path, "c1", extra=("  cmass down 1 1",)), "c1")
    e = s.rmc_estimators_setup(12, 3)
    assert e.cmass_nskip == 1 and e.cmass_ntauskip[0][0] == 3
    assert e.nvalues == 4 + 6


@pytest.mark.parametrize("rec", ["  mstar left 1", "  itc 1 nosuch 1 elocal 1",
                                 "  itc 1 rhok_up complex 1 elocal 0",
                                 "  cmass up 1 2 1"])
def test_bad_records(q, tmp_path, rec):
    s = q.System.read(write_variant(tmp_path, "bad", extra=(rec,)), "bad")
    with pytest.raises(q.QMCError):
        s.rmc_estimators_setup(20, 2)


def test_estimator_files(q, tmp_path):
    """averages(3)'s estimator files: names, one line per value in
    write_nonscalar_props' format, z_cmass lines following block by block."""
    import numpy as np

    s = q.System.read(write_variant(tmp_path, "est", extra=RECORDS), "est")
    e = s.rmc_estimators_setup(20, 2)
    st = q.Stats(s, e.nvalues)
    rng = np.random.default_rng(1)
    out = tmp_path / "out"
    out.mkdir()
    for b in range(2):
        blk = rng.normal(size=e.nvalues) * 30.0
        st.add_block(blk, 30.0)
        st.write_estimators(e, blk, 30.0, out, "run")
    names = sorted(os.listdir(out))
    assert names == sorted(["run.mstar_up", "run.mstar_down", "run.z_cmass_up",
                            "run.cmass_up", "run.rhok_up_rhok_up", "run.elocal+epot_ekin"])
    lines = lambda n: open(out / n).read().splitlines()  # noqa: E731
    assert len(lines("run.mstar_up")) == 16 and len(lines("run.mstar_down")) == 8
    assert len(lines("run.cmass_up")) == 9 + 7
    assert len(lines("run.z_cmass_up")) == 2 * 4  # two blocks
    assert len(lines("run.rhok_up_rhok_up")) == 8 * 2 * s.s.nk
    assert len(lines("run.elocal+epot_ekin")) == 16
    ln = lines("run.mstar_up")[3]
    assert len(ln) == 19 + 19 + 9 + 10 + 1 + 7 + 5 and ln[58:65] == " merea " and int(ln[65:]) == 4
    mean, _, _, _ = st.get()
    assert abs(float(ln[19:38]) - mean[e.jmstar + 3]) <= 1e-10 * abs(mean[e.jmstar + 3])
