"""Test infrastructure only (the oracle): a plain numpy/Python restatement of
the imaginary-time estimators of path_props (reptation.f:1578-1737), for
checking the device's qmc2d_rmc_path_estimators on the same paths.

A path is its ntau beads in order from the reptile's first bead: x[ntau, 2N]
(x(2,N) per bead) and p[ntau, nprops] (the stored bead properties). The
estimator layout is the one qmc2d_rmc_estimators_setup returns (cmass z,
cmass diffusion, mstar, itc). Loops follow the reference's, bead index
itau ascending outermost, so that the sums are formed in its order."""
import math

import numpy as np


def path_estimators(est, sysinfo, x, p):
    """est: a qmc2d_rmc_estimators (ctypes); sysinfo: dict with ipfrst, np,
    eli (per dimension); x, p: one path. Returns the estimator vector."""
    ntau, skip0 = est.ntau, est.ntauskip
    nb = ntau - 2 * skip0
    out = np.zeros(est.nvalues)
    ipf, npt, eli = sysinfo["ipfrst"], sysinfo["np"], sysinfo["eli"]

    def cmass(t, itau):  # centre of mass of type t in bead itau (1-based)
        xs = x[itau - 1].reshape(-1, 2)[ipf[t]:ipf[t] + npt[t]]
        return [sum(xs[:, d]) / npt[t] for d in range(2)]

    # cmass z (middle bead ntau/2 + 1)
    for c in range(est.ncmass):
        t = est.cmass_type[c]
        cm = cmass(t, ntau // 2 + 1)
        for d in range(2):
            v = cm[d] * (2.0 * math.pi * eli[d]) * npt[t]
            out[est.jcmass_z + 4 * c + 2 * d] = math.cos(v)
            out[est.jcmass_z + 4 * c + 2 * d + 1] = math.sin(v)
    # cmass diffusion
    off = est.jcmass_d
    for c in range(est.ncmass):
        t, ts = est.cmass_type[c], est.cmass_tau_skip[c]
        cms = [None] + [cmass(t, i) for i in range(1, ntau + 1)]
        for k in range(est.cmass_nskip):
            sk = est.cmass_ntauskip[c][k]
            nij = (ntau - 2 * sk) // ts
            re, nrm = np.zeros(nij), np.zeros(nij)
            for itau in range(1 + sk, ntau - sk + 1):
                for jtau in range(itau, ntau - sk + 1, ts):
                    ij = (jtau - itau) // ts
                    for d in range(2):
                        re[ij] += (cms[itau][d] - cms[jtau][d]) ** 2
                    nrm[ij] += 1.0
            out[off:off + nij] = re / nrm
            off += nij
    # mstar
    off = est.jmstar
    for i in range(est.nmstar):
        t, ts = est.mstar_type[i], est.mstar_tau_skip[i]
        nij = nb // ts
        re, nrm = np.zeros(nij), np.zeros(nij)
        for itau in range(1 + skip0, ntau - skip0 + 1):
            for jtau in range(itau, ntau - skip0 + 1, ts):
                ij = (jtau - itau) // ts
                for ip in range(ipf[t], ipf[t] + npt[t]):
                    for d in range(2):
                        re[ij] += (x[itau - 1][2 * ip + d] - x[jtau - 1][2 * ip + d]) ** 2
                    nrm[ij] += 1.0
        out[off:off + nij] = re / nrm
        off += nij
    # itc
    off = est.jitc
    for i in range(est.nitc):
        ts = est.itc_tau_skip[i]
        nij = nb // ts
        cplx = est.itc_complex[i] != 0
        icounts = range(0, est.itc_count[i], 2) if cplx else range(est.itc_count[i])
        for ic in icounts:
            re, im, nrm = np.zeros(nij), np.zeros(nij), np.zeros(nij)
            for itau in range(1 + skip0, ntau - skip0 + 1):
                ri = sum(p[itau - 1][est.itc_start[i][a] + ic] for a in range(est.itc_add[i]))
                ii = 0.0
                if cplx:
                    ii = sum(p[itau - 1][est.itc_start[i][a] + ic + 1]
                             for a in range(est.itc_add[i])) * est.itc_complex[i]
                for jtau in range(itau, ntau - skip0 + 1, ts):
                    rj = sum(p[jtau - 1][est.jtc_start[i][a] + ic] for a in range(est.jtc_add[i]))
                    ij = (jtau - itau) // ts
                    if cplx:
                        jj = sum(p[jtau - 1][est.jtc_start[i][a] + ic + 1]
                                 for a in range(est.jtc_add[i])) * est.jtc_complex[i]
                        re[ij] += ri * rj - ii * jj
                        im[ij] += ri * jj + ii * rj
                    else:
                        re[ij] += ri * rj
                    nrm[ij] += 1.0
            if cplx:
                out[off:off + nij] = re / nrm
                out[off + nij:off + 2 * nij] = im / nrm
                off += 2 * nij
            else:
                out[off:off + nij] = re / nrm
                off += nij
    return out
