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
        + N^2 sqrt(pi)/(alpha L^2)) (self + neutralising background).
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


def half_space_kvectors(L, nmax2):
    """Half-space reciprocal vectors 2 pi/L (n1, n2), |n|^2 <= nmax2, by shells."""
    out = []
    m = int(math.isqrt(nmax2)) + 1
    for n1 in range(0, m + 1):
        for n2 in range(-m, m + 1):
            if n1 == 0 and n2 <= 0:
                continue
            if n1 * n1 + n2 * n2 <= nmax2:
                out.append((n1 * n1 + n2 * n2, n1, n2))
    out.sort()
    g = 2.0 * math.pi / L
    return np.array([[g * a, g * b] for _, a, b in out])


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
             alpha_L=5.0, nmax2=37, twist=False, nconf=0, seed=1):
    """Write the run directory; returns its path. backflow = (lam, r0_bohr, w_bohr)."""
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
    kv = half_space_kvectors(L, nmax2)
    kn = np.sqrt((kv ** 2).sum(1))
    vk = e2 * 2.0 * math.pi * np.array([math.erfc(k / (2 * alpha)) for k in kn]) / (kn * L * L)
    v0 = -e2 * (N * alpha / math.sqrt(math.pi) + N * N * math.sqrt(math.pi) / (alpha * L * L))
    write_table(os.path.join(directory, f"{runid}.v"), hermite_table(f, df, drt), drt, "ewald",
                [alpha], kspace=(vk, 0.0))
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
