"""Block statistics of averages(3) (reptation.f:4305-4352) and the report
and rho_k file formats of averages(3) / write_nonscalar_props
(reptation.f:4343-4345, 4582-4616): host-only, no GPU."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "n26")


def _sys(q):
    return q.System.read(GOLDEN, "n26")


def test_cumulative_sums_and_errors(q):
    """cml_av += blk, cml2 += blk^2/norm, cml_norm += norm; err =
    sqrt(|cml2/norm - mean^2| / (iblk-1)), 0 after one block."""
    s = _sys(q)
    n = s.nprops
    rng = np.random.default_rng(3)
    st = q.Stats(s)
    cml, cml2, cn = np.zeros(n), np.zeros(n), 0.0
    for ib in range(1, 5):
        norm = float(rng.uniform(100, 200))
        blk = rng.normal(size=n) * norm
        st.add_block(blk, norm)
        cml += blk
        cml2 += blk ** 2 / norm
        cn += norm
        mean, err, norm_out, nb = st.get()
        assert nb == ib and norm_out == cn
        np.testing.assert_allclose(mean, cml / cn, rtol=1e-14)
        want = np.sqrt(np.abs((cml2 / cn - (cml / cn) ** 2) / (ib - 1))) if ib > 1 else 0 * cml
        np.testing.assert_allclose(err, want, rtol=1e-12, atol=1e-300)


def test_report_fortran_e_fields(q):
    """One line per scalar property: e19.11, e19.11, e9.2, e10.3, 2x, a20."""
    s = _sys(q)
    n = s.nprops
    norm = 4096.0
    vals = np.zeros(n)
    vals[0] = 1.5                      # elocal
    vals[1] = -0.000123456789012345    # -log tf
    vals[2] = 0.0                      # acc.rate
    vals[3] = 1e-120                   # epot: three-digit exponent
    st = q.Stats(s)
    st.add_block(vals * norm, norm)
    lines = st.report(vals * norm, norm, "vmc").splitlines()
    assert lines[0] == " ===>> vmc block 1"
    body = lines[1:]
    assert len(body) == s.s.n_scalar_props
    # hand-derived Fortran Ew.d output for these values
    assert body[0][:19] == "  0.15000000000E+01"
    assert body[0][19:38] == "  0.15000000000E+01"
    assert body[0][38:47] == " 0.00E+00"          # error after one block
    assert body[0][47:57] == " 0.410E+04"         # 4096 -> 0.4096E+04 -> 3 digits
    assert body[0][57:] == "  " + "elocal".ljust(20)
    assert body[1][:19] == " -0.12345678901E-03"
    assert body[1][57:] == "  " + "-log tf".ljust(20)
    assert body[2][:19] == "  0.00000000000E+00"
    assert body[3][:19] == "  0.10000000000-119"
    names = [ln[59:].rstrip() for ln in body]
    assert names[:7] == ["elocal", "-log tf", "acc.rate", "epot", "ekin", "e2", "gg"]
    assert names[-1] == "efp"
    t = [s.s.type_name[i].value.decode() for i in range(s.ntypes)]
    assert names[7:7 + s.ntypes] == ["pot_" + x for x in t]


def test_rhok_files(q, tmp_path):
    """One file per rho_k slot, 2 nk lines of 2e19.11,e9.2,e10.3,1x,a7,i5."""
    s = _sys(q)
    n, nk = s.nprops, s.s.nk
    rng = np.random.default_rng(5)
    st = q.Stats(s)
    b1, b2 = rng.normal(size=n) * 50, rng.normal(size=n) * 50
    st.add_block(b1, 50.0)
    st.add_block(b2, 50.0)
    st.write_rhok(b2, 50.0, tmp_path, "run")
    mean, err, _, _ = st.get()
    t0 = s.s.type_name[0].value.decode()
    lines = open(tmp_path / f"run.rhok_{t0}").read().splitlines()
    assert len(lines) == 2 * nk
    j0 = s.s.jrhok
    for j, ln in enumerate(lines[:5]):
        assert len(ln) == 19 + 19 + 9 + 10 + 1 + 7 + 5
        assert ln[57] == " " and ln[58:65] == " merea " and int(ln[65:]) == j + 1
        f = [float(ln[a:b].replace("E", "e")) for a, b in ((0, 19), (19, 38), (38, 47))]
        assert math.isclose(f[0], b2[j0 + j] / 50.0, rel_tol=1e-10, abs_tol=1e-300)
        assert math.isclose(f[1], mean[j0 + j], rel_tol=1e-10, abs_tol=1e-300)
        assert math.isclose(f[2], err[j0 + j], rel_tol=0.05, abs_tol=1e-300)  # two digits
