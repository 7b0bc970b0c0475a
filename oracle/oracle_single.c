/*
 * oracle_single.c - CPU oracle (TEST INFRASTRUCTURE ONLY) for the device's
 * single-electron VMC sweeps (qmc2d_vmc_single). The reference moves all
 * electrons at once (move, reptation.f:4617-4680); the device applies the
 * same importance-sampled Metropolis step to one electron at a time. Here
 * every ratio and drift comes from a full evaluation of the configuration
 * with the one electron moved (oracle_compute_properties, the reference's
 * compute_properties restated): no inverse is kept, so the device's
 * Sherman-Morrison updates and refreshes are checked against an independent
 * route. The draws replay the device's Philox streams:
 *   electron i, coordinate d of walker w in sweep t: (u_cos, u_log) =
 *   philox(seed, c0 = 2i+d, c1 = w, c2 = t, c3 = 0x5100); its acceptance
 *   draw u[0] of (c0 = 0x80000000|i, c1 = w, c2 = t, c3 = 0x5100).
 */
#include "oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TAG_SINGLE 0x5100u

int oracle_vmc_single(const qmc2d_system *sys, int nw, int nsweep, double delta, uint64_t seed,
                      long sweep0, double *x, double *g, double *hl, double *p, double *s,
                      double *age, double *blk, long *naccept) {
  const int N = sys->nptot, npr = sys->n_props, nt = sys->ntypes;
  qmc2d_system s2 = *sys;
  s2.delta = delta; /* kinetic's drift cutoff reads the time step */
  oracle_work *w = oracle_work_new(&s2);
  double *xn = malloc(sizeof(double) * 2 * N), *gn = malloc(sizeof(double) * 2 * N);
  double *pn = malloc(sizeof(double) * npr);
  const double pi = acos(-1.0);
  long nacc = 0;
  int st = 0;
  for (int k = 0; k < nw && st == 0; k++) {
    double *xk = x + (size_t)2 * N * k, *gk = g + (size_t)2 * N * k, *pk = p + (size_t)npr * k;
    double *hk = hl + (size_t)nt * k, sk, hn[QMC2D_MAX_TYPES], sn;
    int uf = 0;
    st = oracle_compute_properties(&s2, w, xk, gk, hk, pk, &sk, &uf);
    for (int sw = 0; sw < nsweep && st == 0; sw++) {
      const uint32_t t = (uint32_t)(sweep0 + sw);
      double psum = 0.0;
      for (int i = 0; i < N && st == 0; i++) {
        int ti = (nt > 1 && i >= sys->ipfrst[1]) ? 1 : 0;
        double var = 2.0 * sys->hbs2m[ti] * delta, vari = 1.0 / var;
        double chi[2], wold = 0.0;
        memcpy(xn, xk, sizeof(double) * 2 * N);
        for (int d = 0; d < 2; d++) {
          double u[2];
          oracle_philox_uniform2(seed, (uint32_t)(2 * i + d), (uint32_t)k, t, TAG_SINGLE, u);
          chi[d] = cos(pi * u[0]) * sqrt(-2.0 * var * log(u[1]));
          wold = wold - chi[d] * chi[d] * vari;
          xn[2 * i + d] = xk[2 * i + d] - var * gk[2 * i + d] + chi[d];
        }
        st = oracle_compute_properties(&s2, w, xn, gn, hn, pn, &sn, &uf);
        if (st) break;
        double wnew = 0.0;
        for (int d = 0; d < 2; d++) {
          double b = xk[2 * i + d] - xn[2 * i + d] + var * gn[2 * i + d];
          wnew = wnew - b * b * vari;
        }
        double pr = (pk[QMC2D_JLTF] - pn[QMC2D_JLTF]) * 2 + 0.5 * (wnew - wold);
        pr = pr < -50.0 ? -50.0 : pr;
        pr = pr > 0.0 ? 0.0 : pr;
        pr = exp(pr);
        double u[2];
        oracle_philox_uniform2(seed, 0x80000000u | (uint32_t)i, (uint32_t)k, t, TAG_SINGLE, u);
        psum += pr;
        if (pr >= u[0]) {
          memcpy(xk, xn, sizeof(double) * 2 * N);
          memcpy(gk, gn, sizeof(double) * 2 * N);
          memcpy(pk, pn, sizeof(double) * npr);
          for (int q = 0; q < nt; q++) hk[q] = hn[q];
          nacc++;
        }
      }
      pk[QMC2D_JACC] = psum / N;
      if (blk)
        for (int q = 0; q < npr; q++) blk[q] = blk[q] + pk[q];
    }
    s[k] = 1.0;
    age[k] = 0.0;
  }
  if (naccept) *naccept = nacc;
  free(xn);
  free(gn);
  free(pn);
  oracle_work_free(w);
  return st;
}
