"""The setup program's optimised Ewald breakup (2degas_b200/breakup.py)
against the reference's own outputs for N = 26, r_s = 1, nt = 500: the
intermediate file te.vrk (r table, self, constant and k-space energies),
the fit's diagnostics in te.os (points fitted, polynomial, rms error) and
the deck's n26.v that traduci made from te.vrk. A deck written with
ewald="fitpn" gives, through the oracle, the potential energy of an
independent Ewald sum."""
import importlib
import math
import os

import numpy as np
import pytest

breakup = importlib.import_module("2degas_b200.breakup")
GOLD = os.path.join(os.path.dirname(__file__), "golden", "n26")

# te.os (the setup program's output stream for this fit)
TE_OS_NK = 91
TE_OS_RMS = 3.94776845e-07
TE_OS_POLY = [-0.442587, -0.130688, 0.935727, 0.689471, -0.838311, -1.13999, 0.913706]
TE_OS_K = [0.0, 0.695213598, 0.983180499, 1.3904272, 1.55454486, 1.966361, 2.08564079,
           2.19845843, 2.50662827, 2.78085439, 2.8664391, 2.9495415, 3.10908973,
           3.47606799, 3.5449077, 3.7438398, 3.932722, 4.05375705, 4.17128159]
TE_OS_MADELUNG = -0.86310248  # "computed madelung constant"
TE_OS_IDEAL = -0.863102734  # "ideal square madelung constant" (closed form and mdlng)


@pytest.fixture(scope="module")
def fit():
    return breakup.ewald_fitpn(26, 1.0, 500)


def test_fit_reproduces_the_reference_vrk(fit):
    g = breakup.read_vrk(os.path.join(GOLD, "te.vrk"))
    assert fit["nk"] == TE_OS_NK
    assert np.allclose(fit["k"], TE_OS_K, rtol=1e-8, atol=0)
    assert fit["madelung"] == pytest.approx(TE_OS_MADELUNG, rel=1e-7)
    assert fit["rms"] == pytest.approx(TE_OS_RMS, rel=1e-6)
    assert np.allclose(fit["poly"], TE_OS_POLY, rtol=2e-5, atol=0)
    # te.vrk holds 9 significant digits
    assert np.abs(fit["v"] - g["v"]).max() < 2e-8
    assert np.abs(fit["dv"] - g["dv"]).max() < 2e-8
    assert fit["self_energy"] == pytest.approx(g["self_energy"], rel=1e-8)
    assert fit["constant"] == pytest.approx(g["constant"], rel=1e-8)
    vk = np.array([v for v, m in zip(fit["vk_shells"], fit["mult"]) for _ in range(m)])
    assert len(vk) == len(g["vk"]) == 56
    assert np.abs(vk - g["vk"]).max() < 1e-10


def test_madelung_of_the_square_lattice():
    L = math.sqrt(26 * math.pi)
    v = breakup.madelung(L, 2.0)
    assert v == pytest.approx(TE_OS_IDEAL, rel=1e-8)
    assert v == pytest.approx(-3.90026492 * 2.0 / L, rel=1e-8)  # ocpset's closed form


def test_traduci_reproduces_the_reference_v_table():
    g = breakup.read_vrk(os.path.join(GOLD, "te.vrk"))
    lines = open(os.path.join(GOLD, "n26.v")).read().split("\n")
    nt, drt_gold = int(lines[0].split()[0]), float(lines[0].split()[1])
    drt = math.sqrt(26 * math.pi) / 2 / nt
    assert drt == pytest.approx(drt_gold, rel=1e-9)
    rows = breakup.hermite_rows(g["v"], g["dv"], drt)
    gold = np.array([[float(x) for x in lines[1 + i].split()] for i in range(nt + 1)])
    err = np.abs(rows - gold)
    assert (err <= 1e-8 * np.abs(gold) + 1e-16).all()
    # the trailer: routine, no parameters, the k list as in te.vrk, v0 = 0
    fit_like = dict(v=g["v"], dv=g["dv"], vk_shells=g["vk"], mult=[1] * len(g["vk"]),
                    constant=g["constant"], self_energy=g["self_energy"])
    text, v0 = breakup.v_table_text(fit_like, 26, drt, ifv0=1)
    mine = text.split("\n")
    assert [s.strip() for s in mine[nt + 2:nt + 6]] == ["fitpn", "0", "kspace", "56"]
    assert [s.strip() for s in lines[nt + 2:nt + 6]] == ["fitpn", "0", "kspace", "56"]
    assert np.allclose([float(s) for s in mine[nt + 6:nt + 62]],
                       [float(s) for s in lines[nt + 6:nt + 62]], rtol=1e-8, atol=0)
    assert mine[nt + 62].strip() == lines[nt + 62].strip() == "0.d0"
    assert v0 == pytest.approx((g["constant"] * 26 + g["self_energy"]) / 2)


def _ewald(x, L, e2, alpha, nimg=3, kmax=14):
    """Potential energy per electron of N electrons in the periodic square
    cell with a neutralising background: the textbook 2D Ewald sum of e^2/r
    (real-space erfc images, reciprocal erfc(k/2 alpha)/k, self and
    background terms), summed far enough to be exact to 1e-12 here."""
    from scipy.special import erfc

    N, A = len(x), L * L
    img = np.array([(a, b) for a in range(-nimg, nimg + 1) for b in range(-nimg, nimg + 1)]) * L
    ks = np.array([(a, b) for a in range(-kmax, kmax + 1) for b in range(-kmax, kmax + 1)
                   if (a, b) != (0, 0)]) * (2 * math.pi / L)
    kn = np.linalg.norm(ks, axis=1)
    kw = 2 * math.pi / A * erfc(kn / (2 * alpha)) / kn

    def phi(r):
        d = np.linalg.norm(r + img, axis=1)
        d = d[d > 0]
        return (erfc(alpha * d) / d).sum() + (kw * np.cos(ks @ r)).sum() \
            - 2 * math.sqrt(math.pi) / (alpha * A)

    xi = phi(np.zeros(2)) - 2 * alpha / math.sqrt(math.pi)
    E = sum(phi(x[i] - x[j]) for i in range(N) for j in range(i + 1, N))
    return e2 * (E + 0.5 * N * xi) / N


def test_fitpn_deck_at_the_benchmark_shell(tmp_path):
    """N = 58 at r_s = 5 (the fit's shells and grid scale with the cell):
    within 1e-8 Ry per electron of the independent sum."""
    q = importlib.import_module("2degas_b200")
    tables = importlib.import_module("2degas_b200.tables")
    from oracle_lib import Oracle

    d = tables.make_run(str(tmp_path / "f58"), "c", 29, 29, 5.0, nconf=1, seed=5,
                        ewald="fitpn")
    s = q.System.read(d, "c")
    x = s.read_configs(d, ".0", 0, 1)
    pot = Oracle(s).compute_properties(x[0])[2][q._capi.JPOT0]
    L = math.sqrt(58 * math.pi)
    assert abs(pot - _ewald(x[0].reshape(-1, 2), L, 0.4, 4.0 / L)) < 1e-8


def test_fitpn_deck_gives_the_ewald_potential(tmp_path):
    q = importlib.import_module("2degas_b200")
    tables = importlib.import_module("2degas_b200.tables")
    from oracle_lib import Oracle

    L, e2 = math.sqrt(26 * math.pi), 2.0
    pots = {}
    for ew in ("fitpn", "erfc"):
        d = tables.make_run(str(tmp_path / ew), "c", 13, 13, 1.0, nconf=2, seed=3, ewald=ew)
        s = q.System.read(d, "c")
        x = s.read_configs(d, ".0", 0, 2)
        o = Oracle(s)
        pots[ew] = [o.compute_properties(x[k])[2][q._capi.JPOT0] for k in range(2)]
    for k in range(2):
        exact = _ewald(x[k].reshape(-1, 2), L, e2, 4.0 / L)
        assert abs(pots["fitpn"][k] - exact) < 1e-5
        # the plain split at alpha = 5/L truncates erfc(alpha r) at r = L/2
        # (erfc(2.5) = 4e-4): a few 1e-4 Ry per electron
        assert abs(pots["erfc"][k] - exact) < 1e-3
