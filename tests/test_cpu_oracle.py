"""The CPU oracle against the reference's own checks and data.

* testd-style finite differences (reptation.f:2583-2620): the drift and the
  Laplacian the oracle returns must be the derivatives of the -ln psi it
  returns.
* rannyu (reptation.f:5247) against the 48-bit LCG it implements.
* branch2's comb (reptation.f:2162-2273) against a line-by-line Python
  transcription of the Fortran loop.
* the statistical pin: independent 20000-step VMC blocks of the n26 golden
  deck (twist (1,1) of 4x4, delta = 0.05, the reference's seed and first
  stored configuration) must bracket the block the reference wrote to
  n26.res (E_L = -0.4356474067 Ry/electron).
"""
import os

import numpy as np
import pytest

from conftest import N26

GOLD_E = -8712.94813421877 / 20000.0   # n26.res:3 / cml_norm (n26.res:2)


def fd_check(o, x, dx=1e-5):
    g, h, p, _, _ = o.compute_properties(x)
    gfd = np.zeros_like(g)
    lap = np.zeros_like(h)
    N = len(x) // 2
    nup = N // 2
    for j in range(len(x)):
        xp = x.copy()
        xp[j] += dx
        xm = x.copy()
        xm[j] -= dx
        gp, _, pp, _, _ = o.compute_properties(xp)
        gm, _, pm, _, _ = o.compute_properties(xm)
        gfd[j] = (pp[1] - pm[1]) / (2 * dx)
        lap[0 if j < 2 * nup else 1] += (gp[j] - gm[j]) / (2 * dx)
    return g, gfd, h, lap


def test_drift_is_gradient_of_minus_log_psi(oracle_cls, n26, n26_configs):
    o = oracle_cls(n26)
    for k in (0, 5):
        g, gfd, h, lap = fd_check(o, n26_configs[k].copy())
        assert np.abs(g - gfd).max() < 1e-6 * max(1.0, np.abs(g).max())
        assert np.abs(h - lap).max() < 1e-5 * max(1.0, np.abs(h).max())


def test_drift_without_backflow_and_twist(oracle_cls, q, tmp_path, n26_configs):
    from variants import write_variant

    d = write_variant(tmp_path, "nb", backflow=False, ntwists=0)
    s = q.System.read(d, "nb")
    o = oracle_cls(s)
    g, gfd, h, lap = fd_check(o, n26_configs[3].copy())
    assert np.abs(g - gfd).max() < 1e-6 * max(1.0, np.abs(g).max())
    assert np.abs(h - lap).max() < 1e-5 * max(1.0, np.abs(h).max())


def test_spin_swap_and_translation(oracle_cls, n26, n26_configs):
    o = oracle_cls(n26)
    x = n26_configs[2].copy()
    _, h, p, _, _ = o.compute_properties(x)
    xs = np.concatenate([x[26:], x[:26]])
    _, h2, p2, _, _ = o.compute_properties(xs)
    assert abs(p[0] - p2[0]) < 1e-12 and abs(p[1] - p2[1]) < 1e-12
    assert np.allclose(h, h2[::-1], rtol=1e-12)
    # a rigid translation changes only the phase of the twisted determinant
    xt = x + np.tile([0.37, -1.21], 26)
    _, _, p3, _, _ = o.compute_properties(xt)
    assert abs(p[0] - p3[0]) < 1e-11 and abs(p[1] - p3[1]) < 1e-11


def test_rannyu_is_the_48bit_lcg(oracle_cls, n26):
    o = oracle_cls(n26)
    seed = [3535, 3467, 3262, 2 * 1549 + 1]
    draws, state = o.rannyu_stream(seed, 1000)
    m = (502 << 36) | (1521 << 24) | (4071 << 12) | 2107
    ell = (seed[0] << 36) | (seed[1] << 24) | (seed[2] << 12) | seed[3]
    for k in range(1000):
        ell = (ell * m) % (1 << 48)
        assert draws[k] == ell / float(1 << 48)
    assert state == [(ell >> s) & 4095 for s in (36, 24, 12, 0)]


def branch2_python(wate, r):
    """Line-by-line transcription of branch2's comb (reptation.f:2174-2212)
    and prov_dest's in-rank assignment (reptation.f:2260-2271), 1 rank."""
    nconf = len(wate)
    wate = [min(w, 10.0) for w in wate]
    somma = 0.0
    for w in wate:
        somma = somma + w
    tmult, delt, k0 = [], [], 0.0
    for w in wate:
        ww = nconf * w / somma
        tmult.append(int(ww))
        delt.append(ww - int(ww))
        k0 = k0 + (ww - int(ww))
    nw, k, used = 0, 1.0, 0
    for _ in range(int(round(k0))):
        rr = r[used]
        used += 1
        k = k - 1
        while k < rr and nw < nconf:
            nw += 1
            k = k + delt[nw - 1]
        tmult[nw - 1] += 1
        while k < 1 and nw < nconf:
            nw += 1
            k = k + delt[nw - 1]
    mult = list(tmult)
    src = list(range(nconf))
    for j in range(nconf):
        if mult[j] == 0:
            for i in range(nconf):
                if mult[i] >= 2:
                    src[j] = i
                    mult[i] -= 1
                    mult[j] += 1
                    break
    return np.array(tmult), np.array(src), used


def test_branch2_comb(oracle_cls, n26):
    o = oracle_cls(n26)
    rng = np.random.default_rng(5)
    for trial in range(20):
        nw = int(rng.integers(5, 300))
        wate = rng.lognormal(0.0, 0.6 if trial % 2 else 2.0, nw)
        r = rng.uniform(1e-9, 1.0, nw + 1)
        mult, src, used, _ = o.branch2(wate, r)
        pm, ps, pu = branch2_python(list(wate), list(r))
        assert np.array_equal(mult, pm) and np.array_equal(src, ps) and used == pu
        assert mult.sum() == nw
        assert all(mult[s] >= 1 for s in src)


def test_branch2_is_unbiased(oracle_cls, n26):
    """E[mult_i] = nw w_i / sum w for the systematic comb."""
    o = oracle_cls(n26)
    rng = np.random.default_rng(9)
    nw = 40
    wate = rng.uniform(0.2, 3.0, nw)
    acc = np.zeros(nw)
    reps = 3000
    for _ in range(reps):
        mult, _, _, _ = o.branch2(wate, rng.uniform(1e-12, 1.0, nw + 1))
        acc += mult
    expect = nw * wate / wate.sum()
    assert np.abs(acc / reps - expect).max() < 0.05


def _vmc_block(args):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import importlib

    from oracle_lib import Oracle

    seed = args
    q = importlib.import_module("2degas_b200")
    s = q.System.read(N26, "n26")
    x = s.read_configs(N26, ".0", 0, 1)[0]
    o = Oracle(s)
    blk, xf, so, nacc = o.vmc_rannyu(x, 20000, 0.05, 200000, seed, 0)
    return blk[:14] / 20000.0


def test_statistics_against_reference_block():
    """Blocks of 20000 steps of the golden deck from the reference's start
    with different seeds, compared with the block the reference wrote to
    n26.res.

    Coarse agreement only: E_L within 3 %, the potential energy within
    0.5 %, acceptance and nodal distances within 3 %. The recorded block is
    not reproducible to its statistical error: its per-spin kinetic energies
    differ by a factor 2.6 (kin_up 0.302, kin_down 0.799) although the
    deck's wave function is symmetric under up <-> down, for which every
    twist of the 4 x 4 grid gives kin_up = kin_down here. The block was
    therefore written by a different build of the program than the
    sources, and pins the oracle only coarsely."""
    import multiprocessing as mp

    seeds = [[3535, 3467, 3262, 1549]] + [[11 * i + 7, 3467, 100 + i, 2 * i + 1]
                                          for i in range(1, 8)]
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        res = np.array(pool.map(_vmc_block, seeds))
    gold = np.loadtxt(os.path.join(N26, "n26.res"), skiprows=2, max_rows=14)[:, 0] / 20000.0
    assert abs(gold[0] - GOLD_E) < 1e-12
    mean, sd = res.mean(0), res.std(0, ddof=1)
    tol = {0: 0.03, 2: 0.03, 3: 0.005, 11: 0.03, 12: 0.03}
    for j, t in tol.items():
        assert abs(gold[j] - mean[j]) < t * abs(gold[j]), (j, gold[j], mean[j], sd[j])
    # the oracle's wave function is spin-symmetric: kin_up = kin_down
    assert abs(mean[9] - mean[10]) < 5 * np.hypot(sd[9], sd[10])
    assert abs(gold[9] - gold[10]) > 0.4


def _numpy_minus_log_psi(s, x):
    """-ln psi of a Slater-Jastrow deck with an eta = 0 backflow table (so
    q = x) and no u3, restated in numpy independently of the oracle's C: the
    u2 spline of getf (reptation.f:4114) over minimum-image pairs, and
    ln|det| of each spin's plane-wave matrix exp(i g_k . x_j) by LAPACK's LU
    (numpy slogdet)."""
    S = s.s
    N, L = S.nptot, np.array([S.el[0], S.el[1]])
    xy = x.reshape(N, 2)
    u = 0.0
    for a in range(S.ntypes):
        for b in range(S.ntypes):
            t = S.iu2[a][b]
            tb = S.tables[t]
            ut = np.ctypeslib.as_array(tb.ut, shape=(4 * (tb.ngrid + 1),)).reshape(-1, 4)
            ia = range(S.ipfrst[a], S.ipfrst[a] + S.np[a])
            ib = range(S.ipfrst[b], S.ipfrst[b] + S.np[b])
            for i in ia:
                for j in ib:
                    if j <= i:
                        continue
                    d = xy[i] - xy[j]
                    d -= L * np.round(d / L)
                    r = np.hypot(d[0], d[1])
                    ind = int(r * S.drti)
                    rem = r - ind * S.drt
                    c = ut[min(ind, tb.ngrid)]
                    rm = rem * S.drti
                    u += c[0] + rm * (c[1] + rm * (c[2] + rm * c[3]))
    g = np.ctypeslib.as_array(S.gvec, shape=(2 * S.ngvec,)).reshape(-1, 2)
    logdet = 0.0
    for a in range(S.ntypes):
        n, f = S.np[a], S.ipfrst[a]
        A = np.exp(1j * (g[:n] @ xy[f:f + n].T))
        logdet += np.linalg.slogdet(A)[1]
    return u - logdet


@pytest.mark.parametrize("deck", [(13, 13, 1.0), (5, 5, 2.0), (9, 0, 3.0), (1, 1, 1.5)])
def test_minus_log_psi_against_numpy_slogdet(oracle_cls, q, tmp_path, deck):
    """The oracle's -ln psi on plane-wave Slater-Jastrow decks (eta = 0
    backflow tables) equals an independent numpy restatement (spline sum +
    slogdet) to 1e-12 relative."""
    import importlib

    tables = importlib.import_module("2degas_b200.tables")
    nu, nd, rs = deck
    d = tables.make_run(os.path.join(tmp_path, "d"), "c", nu, nd, rs, nconf=6, seed=5,
                        backflow=(0.0, rs, 0.6 * rs))
    s = q.System.read(d, "c")
    x = s.read_configs(d, ".0", 0, 6)
    o = oracle_cls(s)
    for k in range(len(x)):
        _, _, p, _, _ = o.compute_properties(x[k])
        want = _numpy_minus_log_psi(s, x[k])
        assert abs(p[1] - want) <= 1e-12 * max(1.0, abs(want)), (deck, k, p[1], want)
