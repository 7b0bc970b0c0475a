"""A line-by-line transcription of the reference's branch2 over several
ranks (reptation.f:2162-2258, 0-based): the cap at wmult = 10, the
all-gathered weights, the comb with the shared rannyu2 stream, the
send/receive loop and prov_dest. Test infrastructure: the checker of
2degas_b200/multirank.py and qmc2d_comb_plan."""
import numpy as np


def transcribed_branch2(recs, wate, uniforms):
    """recs[p]: rank p's records (nconf rows); wate[p]: their weights;
    uniforms: the comb's draws in order. Returns the ranks' records after
    the comb, the exchange and prov_dest."""
    nproc, nconf = len(recs), recs[0].shape[0]
    wwate = np.concatenate([np.minimum(np.asarray(w, float), 10.0) for w in wate])
    somma = 0.0
    for v in wwate:
        somma = somma + v
    tmult, delt, k0 = [], [], 0.0
    for v in wwate:
        ww = nconf * nproc * v / somma
        tmult.append(int(ww))
        delt.append(ww - int(ww))
        k0 = k0 + delt[-1]
    nw, k, used = -1, 1.0, 0
    for _ in range(int(round(k0))):
        r = uniforms[used]
        used += 1
        k = k - 1
        while k < r:
            nw += 1
            k = k + delt[nw]
        tmult[nw] += 1
        while k < 1 and nw < nconf * nproc - 1:
            nw += 1
            k = k + delt[nw]
    mult = [tmult[p * nconf:(p + 1) * nconf] for p in range(nproc)]
    out = [np.array(r, copy=True) for r in recs]
    multproc = [sum(m) for m in mult]
    while True:  # the send/receive loop (:2214-2249)
        ps = next((p for p in range(nproc) if multproc[p] > nconf), None)
        if ps is None:
            break
        pr = next(p for p in range(nproc) if multproc[p] < nconf)
        idest = next(j for j in range(nconf) if mult[pr][j] == 0)
        mult[pr][idest] += 1
        iprov = next(j for j in range(nconf) if mult[ps][j] >= 2)
        mult[ps][iprov] -= 1
        out[pr][idest] = out[ps][iprov]
        multproc[ps] -= 1
        multproc[pr] += 1
    for p in range(nproc):  # prov_dest (:2250-2258)
        m = mult[p]
        for j in range(nconf):
            if m[j] == 0:
                for i in range(nconf):
                    if m[i] >= 2:
                        out[p][j] = out[p][i]
                        m[i] -= 1
                        m[j] += 1
                        break
    return out
