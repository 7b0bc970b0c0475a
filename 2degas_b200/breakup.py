"""The optimised Ewald breakup of the reference's setup program, restated.

The setup program splits the 2D Coulomb pair potential e^2/r into a
short-range part, tabulated in r up to L/2, and a k-space list over the
first nlamb shells of the square cell's half-space k vectors, by a weighted
least-squares fit (ocpset and fitpn, setup.f:287-542, 1033-1195):

    r v_sr(r) = a sum_i b_i x^(i-1) (x - 1)^3,   x = r / a,  a = L / 2,

with b_1 = -e^2 / a so that r v_sr -> e^2 at r = 0 (the cusp constraint)
and (x - 1)^3 making v_sr, v_sr' and v_sr'' vanish at a. The remaining
b_i minimise sum_k w_k (v_k - vt_k(b))^2 over the shells beyond the first
nlamb, continued by a uniform grid of k up to argek (fillk, setup.f:
968-994), where v_k = 2 pi e^2 / (vol k) is the bare potential's transform
and vt_k(b) the short-range part's:

    vt_k = (2 pi a^2 / vol) sum_i b_i int_0^1 x^(i-1) (x - 1)^3 J0(k a x) dx

(plint2 and pmult, setup.f:1558-1600, 1889-1900; the integrals by
Abramowitz and Stegun 11.1.1, as the reference evaluates them). The
k-space list is v_k - vt_k for the first nlamb shells; the constant energy
is -vt_0 and the self energy -(b_2 - 3 b_1). traduci (setup.f:2227-2314)
turns the r table (values and derivatives) into the reference's cubic
Hermite table format, with the k list expanded by multiplicity.

Host-only table generation; nothing here runs on the GPU.
"""
import math

import numpy as np


def k_shells(L, cut):
    """Norms and cumulative counts of the half-space k-vector shells with
    |k| <= cut of the square cell of side L (shells, setup.f:850-923):
    integer points with the first index fastest, kept when the first
    nonzero index is positive, sorted by norm (a new vector goes before the
    first listed one whose norm is not smaller), and grouped into one shell
    while the squared norm grows by at most 0.1%. Returns (norms, kmult),
    kmult[s] = number of vectors in shells 0..s."""
    a = 2.0 * math.pi / L
    span = int(0.00001 + abs(cut / a))
    c2 = cut * cut
    vecs = []  # squared norms, in the reference's sorted order
    for n2 in range(-span, span + 1):
        for n1 in range(-span, span + 1):
            x1, x2 = n1 * a, n2 * a
            rsq = 0.0 + x1 * x1
            if rsq > c2:
                continue
            rsq = rsq + x2 * x2
            if rsq > c2:
                continue
            first = n1 if n1 != 0 else n2
            if first <= 0:
                continue
            j = 0
            while j < len(vecs) and vecs[j] < rsq:
                j += 1
            vecs.insert(j, rsq)
    norms, kmult = [], []
    rnow = 0.0
    for i, rsq in enumerate(vecs):
        if rsq - rnow > 0.001 * rnow:
            norms.append(0.0)
            kmult.append(0)
        rnow = rsq
        norms[-1] = math.sqrt(rnow)
        kmult[-1] = i + 1
    return norms, kmult


def fill_k(norms, kmult, argek, vol):
    """The k grid and weights of the fit (fillk, setup.f:968-994): k = 0
    with weight 1, the shells with weight 2 x multiplicity (a vector and its
    negative), then a uniform grid of step norms[0]/4 up to argek, each
    point weighted by the number of lattice points its annulus holds
    (vol 2 pi k dk / (2 pi)^2, integrated) less those already counted. The
    grid starts from the norm the reference reads as rknorm(nshlls), which
    with the shells stored from rknorm(2) is the second-to-last shell's,
    and the first annulus takes off every vector of the shells. Returns
    (k, w)."""
    nsh = len(norms)
    k = [0.0] + list(norms)
    w = [1.0, 2.0 * kmult[0]] + [2.0 * (kmult[s] - kmult[s - 1]) for s in range(1, nsh)]
    dk = norms[0] * 0.25
    cutk = norms[-2] if nsh > 1 else 0.0
    nshex = nsh + int((argek - cutk) / dk)
    con = vol * 2.0 * math.pi / (2.0 * (2.0 * math.pi) ** 2)
    vdown = 1 + 2 * kmult[-1]
    for s in range(nsh + 1, nshex + 1):
        vup = con * (cutk + dk * (s - nsh)) ** 2
        k.append(cutk + dk * (s - nsh - 0.5))
        w.append(vup - vdown)
        vdown = vup
    return np.array(k), np.array(w)


def _x_power_j0(r, n, i0):
    """c_i = int_0^1 x^(i+i0-1) J0(r x) dx for i = 1..n (A&S 11.1.1: a
    series in J_1, J_3, J_5, ... of r, cut where the reference cuts it)."""
    from scipy.special import jv

    c = np.empty(n)
    if r < 1e-5:
        for i in range(1, n + 1):
            c[i - 1] = 1.0 / (i + i0)
        return c
    nbf = max(100, 6 * int(r))
    bess = jv(np.arange(nbf + 2), r)  # bess[m] = J_m(r)
    fact, con = 1e-10, 2.0 / (math.e * r)
    for i in range(1, n + 1):
        nn = i + i0 - 2
        s = bess[1]
        rat = 1.0
        for kk in range(4, nbf + 1, 2):
            rat = rat * float(-nn + kk - 4) / float(nn + kk)
            s = s + rat * bess[kk - 1] * (kk - 1)
            if abs(rat) < (con * kk) ** kk * fact:
                break
        c[i - 1] = 2.0 * s / r / (i + i0)
    return c


def _basis(r, m, i0, pn, npow):
    """pn int_0^1 x^(i+i0-1) (x - 1)^npow J0(r x) dx, i = 1..m (plint2 +
    pmult: the powers' integrals differenced npow times)."""
    c = _x_power_j0(r, m + npow, i0)
    for k in range(1, npow + 1):
        c[: m + npow - k] = c[1 : m + npow - k + 1] - c[: m + npow - k]
    return pn * c[:m]


def fit(v, k, w, nf, b0, a, vol, npoly=10, npow=3):
    """fitpn (setup.f:1033-1195) for the 2D Coulomb case (i0 = 0, cusp
    constraint on): returns (b, v_k after the short-range part is
    subtracted, rms error of the fit)."""
    pn = 2.0 * math.pi * a * a / vol
    m = npoly - npow
    anp = 1 - 2 * (npow % 2)
    beta1 = anp * b0 / a
    nk = len(k)
    lhs = np.zeros((m, m))
    rhs = np.zeros(m)
    chisq = 0.0
    for kk in range(nf + 1, nk):
        c = _basis(k[kk] * a, m, 0, pn, npow)
        vv = v[kk] - beta1 * c[0]
        chisq += w[kk] * vv * vv
        rhs[1:] += w[kk] * vv * c[1:]
        lhs[1:, 1:] += w[kk] * np.outer(c[1:], c[1:])
    sol = np.linalg.solve(lhs[1:, 1:], rhs[1:])
    chisq -= float(rhs[1:] @ sol)
    b = np.concatenate([[beta1], sol])
    vout = np.array(v, dtype=float)
    for kk in range(nk):
        vout[kk] -= float(b @ _basis(k[kk] * a, m, 0, pn, npow))
    return b, vout, math.sqrt(chisq) if chisq > 0 else 0.0


def ewald_fitpn(N, rs, nt, cutk=8.0, npoly=10, argek=14.0, nlamb=18):
    """The breakup ocpset computes for N electrons at r_s (reduced units,
    L = sqrt(N pi), e^2 = 2/r_s) on a table of nt + 1 points. Returns a dict
    with the r grid and the table of r v_sr and its derivative (the
    reference's te.vrk r-space part), the self and constant energies, the
    k-space values of the first nlamb shells with their multiplicities, the
    polynomial, the rms error and the number of fitted k points."""
    L = math.sqrt(N * math.pi)
    vol = L * L
    e2 = 2.0 / rs
    lptable = nt + 1
    cutr = 0.5 * L
    eps = 1e-6
    dr = (cutr - eps) / (lptable - 1)
    rv = np.array([eps + i * dr for i in range(lptable)])
    norms, kmult = k_shells(L, cutk)
    k, w = fill_k(norms, kmult, argek, vol)
    v = np.zeros(len(k))
    v[1:] = e2 * 2.0 * math.pi / (vol * k[1:])
    a = rv[-1]
    b, vk, rms = fit(v, k, w, nlamb, e2, a, vol, npoly)
    m = len(b)
    db = np.array([(i + 1) * b[i + 1] for i in range(m - 1)] + [0.0])
    x = rv / a
    v1 = np.polynomial.polynomial.polyval(x, b) * a
    v2 = np.polynomial.polynomial.polyval(x, db) * a
    npow = npoly - m
    v2 = v2 * (x - 1.0) ** npow + npow * (x - 1.0) ** (npow - 1) * v1
    v1 = v1 * (x - 1.0) ** npow
    mult = [int(0.5 * w[s] + 1e-4) for s in range(1, nlamb + 1)]
    self_energy = (-1.0) ** npow * (b[1] - npow * b[0])
    # fitpn's check of the split: the self energy plus the weighted sum of
    # the k-space remainders over every fitted point (the Madelung energy)
    madelung = self_energy + float(w @ vk)
    return dict(r=rv, v=v1, dv=v2 / a, self_energy=self_energy, constant=vk[0],
                vk_shells=vk[1:nlamb + 1], mult=mult, k=k[:nlamb + 1], poly=b, rms=rms,
                nk=len(k), a=a, madelung=madelung)


def madelung(L, e2, p=1.0, ndim=2):
    """Madelung energy of one charge in the square (cubic) lattice of side
    L for an r^-p interaction, e2 times the Ewald sum with the splitting
    alpha = pi / vol^(2/ndim) (mdlng, setup.f:996-1031): the real-space
    images weighted by Gamma(p/2, alpha r^2) / Gamma(p/2), the reciprocal
    ones by Gamma((ndim-p)/2, k^2/(4 alpha)), over |n_l| <= 3 in every
    direction, plus the self and background terms. The upper incomplete
    gamma function is scipy's (the reference evaluates it with its own
    series and continued fraction, gammi)."""
    from scipy.special import gamma, gammaincc

    def ginc(a, x):
        return gammaincc(a, x) * gamma(a)

    limit = int(1 + math.sqrt(-math.log(1e-9) / math.pi))
    vol = L ** ndim
    alpha = math.pi * vol ** (-2.0 / ndim)
    g0 = gamma(0.5 * p)
    v = (-2.0 * alpha ** (0.5 * p) / (p * g0)
         - 2.0 * math.pi ** (0.5 * ndim) / ((ndim - p) * vol * g0 * alpha ** (0.5 * (ndim - p))))
    rng = range(-limit, limit + 1)
    pts = [(i, j) for j in rng for i in rng] if ndim == 2 else \
        [(i, j, l) for l in rng for j in rng for i in rng]
    for n in pts:
        r2 = sum((c * L) ** 2 for c in n)
        if r2 <= 0:
            continue
        rk2 = sum((2.0 * math.pi * c / L) ** 2 for c in n)
        v += (math.pi ** (0.5 * ndim) * (4.0 / rk2) ** (0.5 * (ndim - p))
              * ginc(0.5 * (ndim - p), rk2 / (4.0 * alpha)) / (vol * g0)
              + ginc(0.5 * p, alpha * r2) / (g0 * r2 ** (0.5 * p)))
    return v * e2


def hermite_rows(v, dv, drt):
    """traduci's table (pspline, setup.f:2316-2327): per knot the value, the
    derivative times drt and the cubic's two higher coefficients from the
    next knot's value and derivative; the last knot zeroed."""
    nt = len(v) - 1
    t = np.zeros((nt + 1, 4))
    t[:, 0] = v
    t[:, 1] = np.asarray(dv) * drt
    t[:, 2] = np.asarray(dv) * (drt * drt * 0.5)
    for i in range(nt):
        t[i, 2] = 3.0 * (t[i + 1, 0] - t[i, 0]) - (t[i + 1, 1] + 2.0 * t[i, 1])
        t[i, 3] = -2.0 * (t[i + 1, 0] - t[i, 0]) + (t[i + 1, 1] + t[i, 1])
    t[nt, :] = 0.0
    return t


def v_table_text(fit_out, N, drt, ifv0=1):
    """The reference-format .v table traduci writes (setup.f:2227-2314):
    'nt drt', the rows, 'fitpn', '0', 'kspace', the k-space values expanded
    by multiplicity, then v0 = (N constant + self) / 2 when ifv0 == 0, else
    0 (the deck's v0 record then carries N v0). Returns (text, v0)."""
    rows = hermite_rows(fit_out["v"], fit_out["dv"], drt)
    nt = rows.shape[0] - 1
    out = [f" {nt}  {drt!r}"]
    out += [" " + " ".join(f"{x: .15E}" for x in r) for r in rows]
    out += [" fitpn", " 0", " kspace"]
    vks = [vk for vk, mu in zip(fit_out["vk_shells"], fit_out["mult"]) for _ in range(mu)]
    out.append(f" {len(vks)}")
    out += [f" {x: .15E}" for x in vks]
    v0 = (fit_out["constant"] * N + fit_out["self_energy"]) * 0.5
    out.append(f" {v0: .15E}" if ifv0 == 0 else " 0.d0")
    return "\n".join(out) + "\n", v0


def read_vrk(path):
    """The setup program's intermediate file (te.vrk: writetb's r table,
    then the self, constant and k-space energies). Returns a dict like
    ewald_fitpn's, with the k-space values already expanded."""
    with open(path) as fh:
        lines = [t.strip() for t in fh.read().split("\n")]
    n = int(lines[0].split()[2])
    i = 3
    v = np.array([float(x) for x in lines[i:i + n]])
    dv = np.array([float(x) for x in lines[i + n:i + 2 * n]])
    i += 2 * n
    rest = lines[i:]
    self_e = float(rest[2])
    const = float(rest[5])
    nk = int(rest[6].split()[2])
    vk = np.array([float(x) for x in rest[8:8 + nk]])
    return dict(v=v, dv=dv, self_energy=self_e, constant=const, vk=vk)
