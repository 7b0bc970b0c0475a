"""Run-directory generator for synthetic state points.

Writes a complete reference-format run directory (<runid>.sy, spline tables
in t_read's format, the k-vector file of kread and walker files of
read_conf) for a 2D electron gas at (n_up, n_down, r_s), so any state point
can be run without the reference's interactive setup program. Reduced units
throughout (lengths in r_s a_B, energies in Ry), as the reference's own
setup.f:34-42:
    box side L = sqrt(N pi), hbar^2/2m = 1/r_s^2, e^2 = 2/r_s.

Tables (all cubic Hermite splines through f and f' at the knots, the
reference's `spline`, reptation.f:5223-5245, last knot zeroed):
    u2  u(r) = A/r (1 - exp(-r/F)), A = r_s, F = sqrt(r_s) in Bohr, i.e.
        (1/r)(1 - exp(-sqrt(r_s) r)) in reduced units, shifted so u and u'
        vanish at L/2;
    u3  xi(r) = exp(-(r/2)^2) (the Gaussian exp(-(r/(2 r_s))^2) of Bohr r);
    b   eta(r) = lambda exp(-((r - r0)/w)^2) (r0, w given in Bohr);
    v   plain 2D Ewald: r v_sr(r) = e^2 erfc(alpha r), iexp = 1, with the
        k-space list v_k = e^2 2 pi erfc(k/(2 alpha)) / (k L^2) over the
        half-space k vectors and v0 = -e^2 (N alpha/sqrt(pi)
        + N^2 sqrt(pi)/(alpha L^2)) (self + neutralising background);
        or, with ewald="fitpn", the setup program's optimised breakup over
        the same k vectors (breakup.py).
The k vectors are listed as the reference's krlv lists them. The
reference's own table generators are restated too: tgen with u2_ob_cos,
u2_reatto and eta_yk, which regenerate tables the reference wrote from the
routine name and parameters in their trailer.
"""
import math
import os

import numpy as np


def _f(v):
    """Full-precision decimal of a float (numpy scalars included)."""
    return repr(float(v))


def hermite_table(f, df, drt):
    """t_read rows (ngrid+1, 4) from f, f' at knots (spline, reptation.f:5223)."""
    nt = len(f) - 1
    t = np.zeros((nt + 1, 4))
    t[:, 0] = f
    t[:, 1] = df * drt
    for i in range(nt):
        d = t[i + 1, 0] - t[i, 0]
        t[i, 2] = 3.0 * d - (t[i + 1, 1] + 2.0 * t[i, 1])
        t[i, 3] = -2.0 * d + (t[i + 1, 1] + t[i, 1])
    t[nt, :] = 0.0
    return t


# ---- the reference's table generators: tgen (reptation.f:5007-5036) with
# its pseudopotential routines u2_ob_cos (:5037-5116), u2_reatto
# (:6517-6563) and eta_yk (:9474-9513). Each gives f and f' on the knots
# r_i = i drt: its analytic form below x = drt (5 nt / 6, integer division),
# and from the first knot at or beyond x the quartic tail of obsmooth
# (:6564-6590), which matches the form's value, slope and curvature at x and
# reaches zero value and slope at r = nt drt; the analytic part is shifted by
# beta0 - g(x) to join it. The expressions follow the routines term by term
# (including u2_ob_cos's curvature at x, ddg + ddc + 2 dg dc), so that a
# table the reference wrote is regenerated from the routine name and
# parameters in its trailer.


def _tail(r, x, xi, g, dg, ddg):
    """obsmooth: the quartic tail and beta0."""
    b0 = -0.5 * dg * xi - ddg * xi ** 2 / 12.0
    b1, b2 = dg, 0.5 * ddg
    b3 = -dg / xi ** 2 - 2.0 / 3.0 * ddg / xi
    b4 = 0.5 * dg / xi ** 3 + 0.25 * ddg / xi ** 2
    d = r - x
    f = b0 + b1 * d + b2 * d ** 2 + b3 * d ** 3 + b4 * d ** 4
    df = b1 + 2.0 * b2 * d + 3.0 * b3 * d ** 2 + 4.0 * b4 * d ** 3
    return f, df, b0


def _join(nt, drt, x, xi, g, dg, ddg, form, rmin=None):
    """f, f' on knots 0..nt: form(r) -> (f, f') below x, the tail beyond."""
    f, df = np.zeros(nt + 1), np.zeros(nt + 1)
    i = 0
    while i <= nt:
        r = i * drt
        if rmin is not None:
            r = max(r, rmin)
        if not r < x:
            break
        f[i], df[i] = form(r)
        i += 1
    r = np.arange(i, nt + 1) * drt
    f[i:], df[i:], b0 = _tail(r, x, xi, g, dg, ddg)
    f[:i] += b0 - g
    return f, df


def eta_yk(p, drt, nt):
    """Backflow eta(r) = l (1 + s r)/(r_B + w r + r^3.5) (Kwon et al. 1998),
    p = (l, s, r_B, w); reptation.f:9474."""
    p1, p2, p3, p4 = p[0], p[1], abs(p[2]), p[3]
    c = drt * (nt * 5 // 6)
    xi = drt * nt - c
    g = p1 * (1 + p2 * c) / (p3 + p4 * c + c ** 3.5)
    dg = (p2 * g - (p4 + 3.5 * c ** 2.5) * g ** 2 / p1) / (1 + p2 * c)
    ddg = -(12 * c ** 2 * g ** 2 + 2 * g * dg * (p4 + 3.5 * c ** 2.5)) / (1 + p2 * c) / p1

    def form(r):
        f = p1 * (1 + p2 * r) / (p3 + p4 * r + r ** 3.5)
        return f, (p2 * f - (p4 + 3.5 * r ** 2.5) * f ** 2 / p1) / (1 + p2 * r)

    return _join(nt, drt, c, xi, g, dg, ddg, form)


def u2_ob_cos(p, drt, nt):
    """u(r) = [(a r + b r^2)/(1 + c^2 r + d^2 r^2) + e] [1 + sum_k e_k
    (1 - cos(2 k pi r / (2 nt drt)))], p = (a, b, c, d, e, e_1, ..., e_n);
    reptation.f:5037."""
    n = len(p) - 5
    p1, p2, p3, p4, p5 = p[0], p[1], p[2] ** 2, p[3] ** 2, p[4]
    x = drt * (nt * 5 // 6)
    xi = drt * nt - x
    pl = math.acos(-1.0) / (2.0 * drt * nt)

    def mod(r, second=False):
        c, dc, ddc = 1.0, 0.0, 0.0
        for k in range(1, n + 1):
            kk = 2 * k * pl
            c += p[4 + k] * (1 - math.cos(kk * r))
            dc += p[4 + k] * math.sin(kk * r) * kk
            ddc += p[4 + k] * math.cos(kk * r) * kk ** 2
        return c, dc, ddc

    D = 1 + p3 * x + p4 * x ** 2
    c, dc, ddc = mod(x)
    g = (p1 * x + p2 * x ** 2) / D + p5
    dg = (p1 + 2 * p2 * x) / D - (p1 * x + p2 * x ** 2) * (p3 + 2 * p4 * x) / D ** 2
    ddg = (2 * p2 / D - 2 * (p1 + 2 * p2 * x) * (p3 + 2 * p4 * x) / D ** 2
           - (p1 * x + p2 * x ** 2) * 2 * p4 / D ** 2
           + 2 * (p1 * x + p2 * x ** 2) * (p3 + 2 * p4 * x) ** 2 / D ** 3)
    ddg = ddg + ddc + 2 * dg * dc
    dg = g * dc + c * dg
    g = g * c

    def form(r):
        c, dc, _ = mod(r)
        Dr = 1 + p3 * r + p4 * r ** 2
        f = (p1 * r + p2 * r ** 2) / Dr + p5
        df = (p1 + 2 * p2 * r) / Dr - (p1 * r + p2 * r ** 2) * (p3 + 2 * p4 * r) / Dr ** 2
        return f * c, df * c + f * dc

    return _join(nt, drt, x, xi, g, dg, ddg, form, rmin=1e-10)


def u2_reatto(p, drt, nt):
    """u(r) = a/r^b + c exp(-d (r - e)^2) + f exp(-g (r - h)^2),
    p = (a, b, c, d, e, f, g, h); reptation.f:6517."""
    x = drt * (nt * 5 // 6)
    xi = drt * nt - x

    def parts(r):
        e1 = math.exp(-p[3] * (r - p[4]) ** 2)
        e2 = math.exp(-p[6] * (r - p[7]) ** 2)
        f = p[0] / r ** p[1] + p[2] * e1 + p[5] * e2
        df = (-p[1] * p[0] / r ** (p[1] + 1.0) - 2 * p[2] * p[3] * (r - p[4]) * e1
              - 2 * p[5] * p[6] * (r - p[7]) * e2)
        ddf = ((p[1] + 1.0) * p[1] * p[0] / r ** (p[1] + 2.0)
               - (2 * p[2] * p[3] - 4 * p[2] * p[3] ** 2 * (r - p[4]) ** 2) * e1
               - (2 * p[5] * p[6] - 4 * p[5] * p[6] ** 2 * (r - p[7]) ** 2) * e2)
        return f, df, ddf

    g, dg, ddg = parts(x)
    return _join(nt, drt, x, xi, g, dg, ddg, lambda r: parts(r)[:2], rmin=1e-10)


GENERATORS = {"eta_yk": eta_yk, "u2_ob_cos": u2_ob_cos, "u2_reatto": u2_reatto}


def tgen(path, routine, params, drt, nt):
    """tgen: the table of `routine` with `params` on nt+1 knots of drt,
    splined as `spline` does (last knot zeroed), written in t_read's
    format with the routine name and parameters as the trailer."""
    f, df = GENERATORS[routine](params, drt, nt)
    rows = hermite_table(f, df, drt)
    write_table(path, rows, drt, routine, params)
    return rows


def read_table_file(path):
    """A t_read table file: (rows (nt+1, 4), drt, routine, params)."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip()]
    nt, drt = lines[0].split()
    nt, drt = int(nt), float(drt.replace("D", "E").replace("d", "e"))
    rows = np.array([[float(v.replace("D", "E").replace("d", "e")) for v in ln.split()]
                     for ln in lines[1:nt + 2]])
    routine = lines[nt + 2].strip()
    jp = int(lines[nt + 3].split()[0])
    params = [float(lines[nt + 4 + k].split()[0]) for k in range(jp)]
    return rows, drt, routine, params


def write_table(path, rows, drt, routine, params, kspace=None):
    with open(path, "w") as fh:
        fh.write(f" {rows.shape[0] - 1}  {_f(drt)}\n")
        for r in rows:
            fh.write(" " + " ".join(f"{v: .15E}" for v in r) + "\n")
        fh.write(f" {routine}\n {len(params)}\n")
        for p in params:
            fh.write(f" {_f(p)} 1\n")
        if kspace is not None:
            vk, vk0 = kspace
            fh.write(" kspace\n")
            fh.write(f" {len(vk)}\n")
            for v in vk:
                fh.write(f" {_f(v)}\n")
            fh.write(f" {_f(vk0)}\n")


def krlv(L, cut):
    """The reference's reciprocal-lattice list for a square cell of side L
    (krlv, reptation.f, 2D branch): half-space vectors (first nonzero index
    positive) with |g| <= cut * 2 pi / L, in its order. Points are visited
    with the first index fastest; each vector is inserted before the first
    one already listed with a strictly larger norm, the norms compared in
    floating point as the reference forms them, so that vectors of one
    shell keep the reference's order (rounding included)."""
    pi = math.acos(-1.0)
    vol = L * L - 0.0 * 0.0
    arlv = [[L * 2 * pi / vol, -0.0 * 2 * pi / vol], [-0.0 * 2 * pi / vol, L * 2 * pi / vol]]
    n1 = math.sqrt(arlv[0][0] ** 2 + arlv[0][1] ** 2)
    n2 = math.sqrt(arlv[1][0] ** 2 + arlv[1][1] ** 2)
    tpiba = min(n1, n2)
    cut1 = cut * tpiba
    cut2 = cut1 ** 2
    small = 1e-7
    theta = math.acos((arlv[0][0] * arlv[1][0] + arlv[0][1] * arlv[1][1]) / (n1 * n2))
    span = [int(abs((cut1 + small) / (n1 * math.sin(theta)))),
            int(abs((cut1 + small) / (n2 * math.sin(theta))))]
    out = []
    for i2 in range(-span[1], span[1] + 1):
        for i1 in range(-span[0], span[0] + 1):
            ix = (i1, i2)
            nzero = i1 if i1 != 0 else i2
            g = [0.0, 0.0]
            for idim in range(2):
                for jdim in range(2):
                    g[jdim] = g[jdim] + ix[idim] * arlv[idim][jdim]
            g2 = g[0] * g[0] + g[1] * g[1]
            if g2 > cut2 or nzero <= 0:
                continue
            at = len(out)
            for j, v in enumerate(out):
                if g2 < v[0] * v[0] + v[1] * v[1]:
                    at = j
                    break
            out.insert(at, (g[0], g[1]))
    return np.array(out)


def closed_shells(limit=200):
    """Occupation numbers of closed shells of the square lattice (with k = 0)."""
    norms = sorted(a * a + b * b for a in range(-20, 21) for b in range(-20, 21))
    shells, cnt, last = [], 0, None
    for nn in norms:
        if last is not None and nn != last:
            shells.append(cnt)
        cnt += 1
        last = nn
        if cnt > limit:
            break
    return shells


def make_run(directory, runid, n_up, n_down, rs, nknots=1000, backflow=None, u3=False,
             alpha_L=5.0, nmax2=37, twist=False, nconf=0, seed=1, ewald="erfc"):
    """Write the run directory; returns its path. backflow = (lam, r0_bohr, w_bohr).
    ewald: "erfc" (the plain split above) or "fitpn" (the setup program's
    optimised breakup, breakup.py, over the same k vectors)."""
    os.makedirs(directory, exist_ok=True)
    N = n_up + n_down
    L = math.sqrt(N * math.pi)
    hbs2m = 1.0 / rs ** 2
    e2 = 2.0 / rs
    rc = L / 2.0
    drt = rc / nknots
    r = np.arange(nknots + 1) * drt
    r1 = np.where(r > 0, r, 1e-300)
    # u2 with value and slope shifted to zero at the cutoff
    a = math.sqrt(rs)

    def u(x):
        return (1.0 - np.exp(-a * x)) / x

    def du(x):
        with np.errstate(divide="ignore", invalid="ignore"):
            return (a * x * np.exp(-a * x) - (1.0 - np.exp(-a * x))) / (x * x)

    f = np.where(r > 0, u(r1), a) - u(rc) - (r - rc) * du(rc)
    df = np.where(r > 0, du(r1), -a * a / 2.0) - du(rc)
    write_table(os.path.join(directory, f"{runid}.u2"), hermite_table(f, df, drt), drt, "rpa",
                [rs])
    # Ewald
    alpha = alpha_L / L
    f = e2 * np.array([math.erfc(alpha * x) for x in r])
    df = -e2 * 2.0 * alpha / math.sqrt(math.pi) * np.exp(-(alpha * r) ** 2)
    # |n|^2 <= nmax2, in the reference's order; widened until the k set
    # holds the orbitals of the larger determinant (2 nk + 1 plane waves)
    nmax = max(n_up, n_down)
    while sum(1 for a in range(-nmax, nmax + 1) for b in range(-nmax, nmax + 1)
              if a * a + b * b <= nmax2) < nmax:
        nmax2 += 1
    kv = krlv(L, math.sqrt(nmax2 + 0.5))
    kn = np.sqrt((kv ** 2).sum(1))
    vk = e2 * 2.0 * math.pi * np.array([math.erfc(k / (2 * alpha)) for k in kn]) / (kn * L * L)
    v0 = -e2 * (N * alpha / math.sqrt(math.pi) + N * N * math.sqrt(math.pi) / (alpha * L * L))
    if ewald == "fitpn":
        # the k-space list of the fit covers exactly the shells of the k file
        from . import breakup

        n2 = sorted({int(round((x * x + y * y) * (L / (2.0 * math.pi)) ** 2)) for x, y in kv})
        kcut = 2.0 * math.pi / L * math.sqrt(n2[-1])
        fit = breakup.ewald_fitpn(N, rs, nknots, cutk=max(8.0, 1.5 * kcut), nlamb=len(n2))
        text, v0n = breakup.v_table_text(fit, N, drt, ifv0=1)
        with open(os.path.join(directory, f"{runid}.v"), "w") as fh:
            fh.write(text)
        v0 = v0n * N
    elif ewald == "erfc":
        write_table(os.path.join(directory, f"{runid}.v"), hermite_table(f, df, drt), drt,
                    "ewald", [alpha], kspace=(vk, 0.0))
    else:
        raise ValueError(f"ewald must be 'erfc' or 'fitpn', not {ewald!r}")
    with open(os.path.join(directory, f"{runid}.k"), "w") as fh:
        for k in kv:
            fh.write(f" {_f(k[0])} {_f(k[1])}\n")
    lines = ["  ndim 2"]
    types = [("up", n_up), ("down", n_down)] if n_down > 0 else [("up", n_up)]
    for name, n in types:
        lines.append(f"  type {name} {n} {_f(hbs2m)} {runid}.{name}.x")
    pairs = [(types[i][0], types[j][0]) for i in range(len(types)) for j in range(i, len(types))]
    lines += [f"  u2 {p} {q} {runid}.u2" for p, q in pairs]
    if u3:
        f = np.exp(-(r / 2.0) ** 2)
        df = -r / 2.0 * f
        write_table(os.path.join(directory, f"{runid}.u3"), hermite_table(f, df, drt), drt,
                    "gauss", [2.0])
        lines += [f"  u3 {p} {q} {runid}.u3" for p, q in pairs]
    lines += [f"  rhok {name}" for name, _ in types]
    lines += [f"  pbc {_f(L)} {_f(L)}", f"  kspace {runid}.k"]
    if backflow is not None:
        lam, r0, w = backflow
        r0, w = r0 / rs, w / rs
        f = lam * np.exp(-(((r - r0) / w) ** 2))
        df = -2.0 * (r - r0) / (w * w) * f
        write_table(os.path.join(directory, f"{runid}.b"), hermite_table(f, df, drt), drt,
                    "gauss_bf", [lam, r0, w])
        lines += [f"  backflow {p} {q} 1 {runid}.b" for p, q in pairs]
    if twist:
        lines.append("  ntwists 4")
    lines += [f"  v2 {p} {q} {runid}.v 0. 1 1." for p, q in pairs]
    lines += [f"  v0 {_f(v0)}", "  end"]
    for ln in lines:
        if len(ln) > 80:
            raise ValueError("record longer than 80 columns: " + ln)
    with open(os.path.join(directory, f"{runid}.sy"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    if nconf > 0:
        rng = np.random.Generator(np.random.Philox(seed))
        x = rng.uniform(-L / 2, L / 2, size=(nconf, N, 2))
        off = 0
        for name, n in types:
            with open(os.path.join(directory, f"{runid}.{name}.x.0"), "w") as fh:
                for c in range(nconf):
                    for i in range(off, off + n):
                        fh.write(f" {_f(x[c, i, 0])} {_f(x[c, i, 1])}\n")
            off += n
    return directory


# The state points of the benchmark configurations (reduced units).
CONFIGS = {
    # plain VMC, N=26 r_s=1, u2 only. The reference builds a determinant
    # only inside its backflow routine, so the Slater part is backflow with
    # eta = 0 (identical values and cost in the reference).
    "vmc_n26_rs1": dict(n_up=13, n_down=13, rs=1.0, backflow=(0.0, 1.0, 0.6), nknots=1000),
    # DMC with backflow, N=58 r_s=5: the headline state point.
    "dmc_bf_n58_rs5": dict(n_up=29, n_down=29, rs=5.0, backflow=(0.2, 5.0, 3.0), nknots=1000),
    # reptation, r_s=10, u2 + u3 + backflow.
    "rmc_n26_rs10": dict(n_up=13, n_down=13, rs=10.0, backflow=(0.2, 10.0, 6.0), u3=True),
    "rmc_n58_rs10": dict(n_up=29, n_down=29, rs=10.0, backflow=(0.2, 10.0, 6.0), u3=True),
}
