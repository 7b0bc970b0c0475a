// comb.cpp - branch2's fixed-population comb over the walkers of several
// ranks (reptation.f:2162-2273): the host-side plan that every rank computes
// identically from the all-gathered weights, with the walker exchange of
// the reference's send/receive loop (:2214-2249, send :2275, receive :2297)
// and the in-rank distribution of prov_dest (:2250-2258, :2320).
//
// The comb's uniforms are the device comb's (Philox4x32-10, tooth c of
// generation g: u[0] of (c0 = c, c1 = 0xFFFFFFFF, c2 = g, c3 = 1)), shared by
// all ranks as the reference's rannyu2 stream is, so with one rank the plan
// is the single-population comb of qmc2d_dmc.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"

namespace {

uint32_t mulhi(uint32_t a, uint32_t b, uint32_t *lo) {
  const uint64_t p = (uint64_t)a * b;
  *lo = (uint32_t)p;
  return (uint32_t)(p >> 32);
}

double comb_uniform(uint64_t seed, uint32_t c, uint32_t gen) {
  uint32_t x0 = c, x1 = 0xFFFFFFFFu, x2 = gen, x3 = 1u;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; r++) {
    uint32_t lo0, lo1;
    const uint32_t hi0 = mulhi(0xD2511F53u, x0, &lo0);
    const uint32_t hi1 = mulhi(0xCD9E8D57u, x2, &lo1);
    const uint32_t n0 = hi1 ^ x1 ^ k0, n2 = hi0 ^ x3 ^ k1;
    x0 = n0;
    x1 = lo1;
    x2 = n2;
    x3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  const unsigned long long k = ((unsigned long long)(x0 >> 5) << 26) | (x1 >> 6);
  return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" int qmc2d_comb_plan(int nproc, int nconf, const double *wate_all, uint64_t seed,
                               uint32_t gen, int rank, int *src, int *nsend, int *send_rank,
                               int *send_slot, int *nrecv, int *recv_rank, int *recv_slot,
                               int *ncapped) {
  if (nproc < 1 || nconf < 1 || rank < 0 || rank >= nproc || !wate_all || !src || !nsend ||
      !send_rank || !send_slot || !nrecv || !recv_rank || !recv_slot) {
    q2d::set_error("qmc2d_comb_plan: bad argument");
    return QMC2D_ERR_ARG;
  }
  const int ntot = nproc * nconf;
  std::vector<double> w(wate_all, wate_all + ntot);
  // cap each weight at wmult = 10 (reptation.f:2174-2181)
  int cap = 0;
  for (int i = 0; i < ntot; i++)
    if (w[i] > 10.0) {
      w[i] = 10.0;
      if (i / nconf == rank) cap++;
    }
  if (ncapped) *ncapped = cap;
  double somma = 0.0;
  for (int i = 0; i < ntot; i++) somma += w[i];
  if (!(somma > 0.0) || !std::isfinite(somma)) {
    q2d::set_error("qmc2d_comb_plan: weights sum to zero or are not finite");
    return QMC2D_ERR_NONFINITE;
  }
  // multiplicities: integer parts, then the systematic comb over the
  // cumulative fractional parts (copy c lands on the first walker whose
  // cumulative fraction reaches c + r_c)
  std::vector<int> mult(ntot);
  std::vector<double> csum(ntot);
  double run = 0.0;
  for (int i = 0; i < ntot; i++) {
    const double ww = ntot * w[i] / somma;
    mult[i] = (int)ww;
    run += ww - mult[i];
    csum[i] = run;
  }
  const int ncomb = (int)std::llround(csum[ntot - 1]);
  for (int c = 0; c < ncomb; c++) {
    const double target = c + comb_uniform(seed, (uint32_t)c, gen);
    int a0 = 0, a1 = ntot;
    while (a0 < a1) {
      const int mid = (a0 + a1) >> 1;
      if (csum[mid] < target) a0 = mid + 1;
      else a1 = mid;
    }
    mult[a0 < ntot ? a0 : ntot - 1]++;
  }
  // walkers per rank, then the exchange loop: the first rank with a surplus
  // sends a copy of its first walker with multiplicity >= 2 into the first
  // empty slot of the first rank with a deficit, until every rank holds nconf
  std::vector<int> multproc(nproc, 0);
  for (int p = 0; p < nproc; p++)
    for (int j = 0; j < nconf; j++) multproc[p] += mult[p * nconf + j];
  *nsend = *nrecv = 0;
  for (;;) {
    int ps = -1, pr = -1;
    for (int p = 0; p < nproc && ps < 0; p++)
      if (multproc[p] > nconf) ps = p;
    if (ps < 0) break;
    for (int p = 0; p < nproc && pr < 0; p++)
      if (multproc[p] < nconf) pr = p;
    if (pr < 0) {
      q2d::set_error("qmc2d_comb_plan: multiplicities do not add up to the population");
      return QMC2D_ERR_POPULATION;
    }
    int idest = -1, iprov = -1;
    for (int j = 0; j < nconf && idest < 0; j++)
      if (mult[pr * nconf + j] == 0) idest = j;
    for (int j = 0; j < nconf && iprov < 0; j++)
      if (mult[ps * nconf + j] >= 2) iprov = j;
    if (idest < 0 || iprov < 0) {
      q2d::set_error("qmc2d_comb_plan: inconsistent exchange");
      return QMC2D_ERR_POPULATION;
    }
    mult[pr * nconf + idest] += 1;
    mult[ps * nconf + iprov] -= 1;
    if (rank == pr) {
      recv_rank[*nrecv] = ps;
      recv_slot[(*nrecv)++] = idest;
    }
    if (rank == ps) {
      send_rank[*nsend] = pr;
      send_slot[(*nsend)++] = iprov;
    }
    multproc[ps]--;
    multproc[pr]++;
  }
  // in-rank distribution (prov_dest): an empty slot takes a copy of the
  // first walker that still has copies to spare
  int *m = mult.data() + (size_t)rank * nconf;
  for (int j = 0; j < nconf; j++) src[j] = j;
  for (int j = 0; j < nconf; j++) {
    if (m[j] != 0) continue;
    for (int i = 0; i < nconf; i++)
      if (m[i] >= 2) {
        src[j] = i;
        m[i]--;
        m[j]++;
        break;
      }
  }
  return QMC2D_OK;
}
