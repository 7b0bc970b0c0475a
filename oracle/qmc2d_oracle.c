/*
 * qmc2d_oracle.c - CPU oracle (TEST INFRASTRUCTURE ONLY) for the walker
 * propagation path of 2degas. A loop-for-loop FP64 restatement of the
 * reference's Fortran; every routine cites the reptation.f lines it follows.
 * Indices are 0-based; Fortran arrays are addressed through the macros below
 * with the reference's column-major index order so loops read as in the
 * original.
 *
 * Parity pin: see qmc2d_oracle.h (re-run of the reference's recorded n26
 * VMC block).
 */
#include "oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ RNG */

/* rannyu (reptation.f:5247-5291): l <- l*m mod 2^48 in 12-bit limbs. */
double oracle_rannyu(oracle_rng *r) {
  const double twom12 = 0.000244140625;
  int m1 = r->m[0], m2 = r->m[1], m3 = r->m[2], m4 = r->m[3];
  int l1 = r->l[0], l2 = r->l[1], l3 = r->l[2], l4 = r->l[3];
  int i1 = l1 * m4 + l2 * m3 + l3 * m2 + l4 * m1;
  int i2 = l2 * m4 + l3 * m3 + l4 * m2;
  int i3 = l3 * m4 + l4 * m3;
  int i4 = l4 * m4;
  l4 = i4 % 4096;
  i3 = i3 + i4 / 4096;
  l3 = i3 % 4096;
  i2 = i2 + i3 / 4096;
  l2 = i2 % 4096;
  l1 = (i1 + i2 / 4096) % 4096;
  r->l[0] = l1;
  r->l[1] = l2;
  r->l[2] = l3;
  r->l[3] = l4;
  return twom12 * (l1 + twom12 * (l2 + twom12 * (l3 + twom12 * (l4))));
}

/* setrn (reptation.f:5292-5318) with nbit = 48 and the multiplier of
 * block data randat (reptation.f:5347-5352). */
void oracle_setrn(oracle_rng *r, const int seed[4]) {
  r->m[0] = 502;
  r->m[1] = 1521;
  r->m[2] = 4071;
  r->m[3] = 2107;
  for (int i = 0; i < 4; i++) r->l[i] = seed[i] % 4096;
  r->l[3] = 2 * (r->l[3] / 2) + 1;
}

/* savern (reptation.f:5319-5345) with nbit = 48. */
void oracle_savern(const oracle_rng *r, int seed[4]) {
  for (int i = 0; i < 4; i++) seed[i] = r->l[i];
}

/* Philox4x32-10: 10 rounds of the published round function with the
 * Weyl key schedule. */
static uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t *hi) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
}

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; round++) {
    uint32_t hi0, hi1;
    uint32_t lo0 = mulhilo32(0xD2511F53u, c0, &hi0);
    uint32_t lo1 = mulhilo32(0xCD9E8D57u, c2, &hi1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* 53 random bits from two words, offset by half an ulp so u is in (0,1). */
static double bits_to_open01(uint32_t a, uint32_t b) {
  uint64_t k = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
}

void oracle_philox_uniform2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                            double u[2]) {
  uint32_t ctr[4] = {c0, c1, c2, c3};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  oracle_philox4x32_10(ctr, key, o);
  u[0] = bits_to_open01(o[0], o[1]);
  u[1] = bits_to_open01(o[2], o[3]);
}

/* ------------------------------------------------------------ scratch */

oracle_work *oracle_work_new(const qmc2d_system *sys) {
  oracle_work *w = (oracle_work *)calloc(1, sizeof(oracle_work));
  if (!w) return NULL;
  int N = sys->nptot;
  w->N = N;
  w->P = N * (N - 1) / 2;
  w->nk = sys->nk;
  int nm = 1;
  for (int t = 0; t < sys->ntypes; t++)
    if (sys->np[t] > nm) nm = sys->np[t];
  w->nmax = nm;
  size_t P = (size_t)(w->P > 0 ? w->P : 1);
  w->pp_r = (double *)calloc(P, sizeof(double));
  w->pp_byr = (double *)calloc(P, sizeof(double));
  w->pp_rem = (double *)calloc(P, sizeof(double));
  w->pp_rvec = (double *)calloc(2 * P, sizeof(double));
  w->pp_ind = (int *)calloc(P, sizeof(int));
  w->rhok = (double *)calloc((size_t)2 * (sys->nk > 0 ? sys->nk : 1) * QMC2D_MAX_TYPES,
                             sizeof(double));
  w->g3 = (double *)calloc((size_t)2 * N, sizeof(double));
  w->dg = (double *)calloc((size_t)4 * N * N, sizeof(double));
  w->ddg = (double *)calloc((size_t)2 * N * N, sizeof(double));
  w->qx = (double *)calloc((size_t)2 * N, sizeof(double));
  w->qa = (double *)calloc((size_t)4 * N * N, sizeof(double));
  w->qb = (double *)calloc((size_t)2 * N * N, sizeof(double));
  size_t nn = (size_t)nm * nm;
  w->zorb = (zc *)calloc(nn, sizeof(zc));
  w->dzorb = (zc *)calloc(2 * nn, sizeof(zc));
  w->ddzorb = (zc *)calloc(4 * nn, sizeof(zc));
  w->sorb = (zc *)calloc(nn * QMC2D_MAX_TYPES, sizeof(zc));
  w->dsorb = (zc *)calloc(2 * nn * QMC2D_MAX_TYPES, sizeof(zc));
  w->ddsorb = (zc *)calloc(4 * nn * QMC2D_MAX_TYPES, sizeof(zc));
  w->zv = (zc *)calloc(2 * nn, sizeof(zc));
  w->zwork = (zc *)calloc((size_t)nm, sizeof(zc));
  w->ipvt = (int *)calloc((size_t)nm, sizeof(int));
  /* pp_dist: a pair of types is in the pair list if any pair table links
   * them (u2, u3, backflow, v2 keywords set pp_dist, reptation.f:243-347). */
  for (int a = 0; a < sys->ntypes; a++)
    for (int b = 0; b < sys->ntypes; b++)
      w->pp_dist[a][b] = (sys->iu2[a][b] >= 0 || sys->iu3[a][b] >= 0 ||
                          sys->iub[a][b] >= 0 || sys->iv2[a][b] >= 0);
  return w;
}

void oracle_work_free(oracle_work *w) {
  if (!w) return;
  free(w->pp_r); free(w->pp_byr); free(w->pp_rem); free(w->pp_rvec); free(w->pp_ind);
  free(w->rhok); free(w->g3); free(w->dg); free(w->ddg); free(w->qx); free(w->qa);
  free(w->qb); free(w->zorb); free(w->dzorb); free(w->ddzorb); free(w->sorb);
  free(w->dsorb); free(w->ddsorb); free(w->zv); free(w->zwork); free(w->ipvt);
  free(w);
}

/* ----------------------------------------------------------- distances */

/* distances (reptation.f:4127-4243): minimum-image pair vectors in the
 * order same-type block of type it, then cross blocks (it, jt>it); rho_k. */
void oracle_distances(const qmc2d_system *sys, oracle_work *w, const double *x) {
  int ij = 0;
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    if (w->pp_dist[it][it]) {
      for (int ip = f0; ip < l0; ip++)
        for (int jp = ip + 1; jp < l0; jp++) {
          w->pp_r[ij] = 0.0;
          for (int d = 0; d < 2; d++) {
            PRV(d, ij) = x[2 * ip + d] - x[2 * jp + d];
            PRV(d, ij) = PRV(d, ij) - sys->el[d] * fnint(sys->eli[d] * PRV(d, ij));
            w->pp_r[ij] = w->pp_r[ij] + PRV(d, ij) * PRV(d, ij);
          }
          w->pp_r[ij] = sqrt(w->pp_r[ij]);
          w->pp_ind[ij] = (int)(w->pp_r[ij] * sys->drti);
          w->pp_rem[ij] = w->pp_r[ij] - w->pp_ind[ij] * sys->drt;
          w->pp_byr[ij] = 1.0 / w->pp_r[ij];
          ij++;
        }
    }
    for (int jt = it + 1; jt < sys->ntypes; jt++) {
      if (!w->pp_dist[it][jt]) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++) {
          w->pp_r[ij] = 0.0;
          for (int d = 0; d < 2; d++) {
            PRV(d, ij) = x[2 * ip + d] - x[2 * jp + d];
            PRV(d, ij) = PRV(d, ij) - sys->el[d] * fnint(sys->eli[d] * PRV(d, ij));
            w->pp_r[ij] = w->pp_r[ij] + PRV(d, ij) * PRV(d, ij);
          }
          w->pp_r[ij] = sqrt(w->pp_r[ij]);
          w->pp_ind[ij] = (int)(w->pp_r[ij] * sys->drti);
          w->pp_rem[ij] = w->pp_r[ij] - w->pp_ind[ij] * sys->drt;
          w->pp_byr[ij] = 1.0 / w->pp_r[ij];
          ij++;
        }
    }
  }
  /* rhok (reptation.f:4225-4243): stored in slot irhok(it). */
  if (sys->nrhok != 0) {
    for (int it = 0; it < sys->ntypes; it++) {
      if (sys->irhok[it] == 0) continue;
      double *rk = w->rhok + (size_t)2 * sys->nk * (sys->irhok[it] - 1);
      memset(rk, 0, sizeof(double) * 2 * sys->nk);
      int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
      for (int ip = f0; ip < l0; ip++)
        for (int ik = 0; ik < sys->nk; ik++) {
          double kr = 0.0;
          for (int d = 0; d < 2; d++) kr = kr + sys->kvec[2 * ik + d] * x[2 * ip + d];
          rk[2 * ik] = rk[2 * ik] + cos(kr);
          rk[2 * ik + 1] = rk[2 * ik + 1] + sin(kr);
        }
    }
  }
}

/* ------------------------------------------------------------ two_body */

/* two_body (reptation.f:2981-3046): u2 pair sum, gradient, Laplacian. */
void oracle_two_body(const qmc2d_system *sys, oracle_work *w, double *ltf_out, double *g_new,
                     double *h_new) {
  int N = w->N;
  double ltf = 0.0, h[QMC2D_MAX_TYPES] = {0.0, 0.0};
  double *g = (double *)calloc((size_t)2 * N, sizeof(double));
  double t, dt, ddt;
  int ij = 0;
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    int i = sys->iu2[it][it];
    if (i >= 0) {
      for (int ip = f0; ip < l0; ip++)
        for (int jp = ip + 1; jp < l0; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          ltf = ltf + t;
          dt = dt * w->pp_byr[ij];
          for (int d = 0; d < 2; d++) {
            g[2 * ip + d] = g[2 * ip + d] + dt * PRV(d, ij);
            g[2 * jp + d] = g[2 * jp + d] - dt * PRV(d, ij);
          }
          h[it] = h[it] + 2 * (ddt + (2 - 1) * dt);
          ij++;
        }
    }
    for (int jt = it + 1; jt < sys->ntypes; jt++) {
      i = sys->iu2[it][jt];
      if (i < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          ltf = ltf + t;
          dt = dt * w->pp_byr[ij];
          for (int d = 0; d < 2; d++) {
            g[2 * ip + d] = g[2 * ip + d] + dt * PRV(d, ij);
            g[2 * jp + d] = g[2 * jp + d] - dt * PRV(d, ij);
          }
          h[it] = h[it] + ddt + (2 - 1) * dt;
          h[jt] = h[jt] + ddt + (2 - 1) * dt;
          ij++;
        }
    }
  }
  *ltf_out = *ltf_out + ltf;
  for (int it = 0; it < sys->ntypes; it++) {
    if (sys->hbs2m[it] == 0.0) continue;
    for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
      for (int d = 0; d < 2; d++) g_new[2 * ip + d] = g_new[2 * ip + d] + g[2 * ip + d];
  }
  for (int it = 0; it < sys->ntypes; it++)
    if (sys->hbs2m[it] != 0.0) h_new[it] = h_new[it] + h[it];
  free(g);
}

/* ---------------------------------------------------------- three_body */

/* makeg (reptation.f:2866-2901); rij is 1/r as passed by three_body. */
static void makeg(oracle_work *w, int jp, int ip, double t, double dt, double ddt,
                  const double *delx, double rij) {
  int N = w->N;
  double aux1 = t, aux2, aux3;
  for (int id = 0; id < 2; id++) {
    aux2 = -aux1 * delx[id];
    G3(id, ip) = G3(id, ip) + aux2;
    G3(id, jp) = G3(id, jp) - aux2;
  }
  aux2 = dt * rij;
  for (int id = 0; id < 2; id++) {
    aux3 = aux1 + aux2 * delx[id] * delx[id];
    DG(id, id, jp, ip) = -aux3;
    DG(id, id, ip, ip) = DG(id, id, ip, ip) + aux3;
    DG(id, id, jp, jp) = DG(id, id, jp, jp) + aux3;
    for (int jd = id + 1; jd < 2; jd++) {
      aux3 = aux2 * delx[id] * delx[jd];
      DG(jd, id, jp, ip) = -aux3;
      DG(jd, id, ip, ip) = DG(jd, id, ip, ip) + aux3;
      DG(jd, id, jp, jp) = DG(jd, id, jp, jp) + aux3;
    }
  }
  aux2 = (2 + 1) * dt * rij + ddt;
  for (int id = 0; id < 2; id++) {
    aux3 = aux2 * delx[id];
    DDG(id, jp, ip) = aux3;
    DDG(id, ip, ip) = DDG(id, ip, ip) - aux3;
    DDG(id, jp, jp) = DDG(id, jp, jp) + aux3;
  }
}

/* dotg (reptation.f:2903-2979) */
static void dotg(const qmc2d_system *sys, oracle_work *w, double *ltf, double *g_new,
                 double *h_new) {
  int N = w->N;
  for (int ip = 0; ip < sys->nptot; ip++)
    for (int id = 0; id < 2; id++) *ltf = *ltf - 0.5 * G3(id, ip) * G3(id, ip);
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    if (sys->iu3[it][it] >= 0) {
      for (int ip = f0; ip < l0; ip++) {
        for (int id = 0; id < 2; id++) {
          g_new[2 * ip + id] = g_new[2 * ip + id] + G3(id, ip) * DG(id, id, ip, ip);
          h_new[it] = h_new[it] - DG(id, id, ip, ip) * DG(id, id, ip, ip);
          h_new[it] = h_new[it] - G3(id, ip) * DDG(id, ip, ip);
          for (int jd = id + 1; jd < 2; jd++) {
            g_new[2 * ip + id] = g_new[2 * ip + id] + G3(jd, ip) * DG(jd, id, ip, ip);
            g_new[2 * ip + jd] = g_new[2 * ip + jd] + G3(id, ip) * DG(jd, id, ip, ip);
            h_new[it] = h_new[it] - 2 * DG(jd, id, ip, ip) * DG(jd, id, ip, ip);
          }
        }
        for (int jp = ip + 1; jp < l0; jp++) {
          for (int id = 0; id < 2; id++) {
            g_new[2 * ip + id] = g_new[2 * ip + id] + G3(id, jp) * DG(id, id, jp, ip);
            g_new[2 * jp + id] = g_new[2 * jp + id] + G3(id, ip) * DG(id, id, jp, ip);
            h_new[it] = h_new[it] - 2 * DG(id, id, jp, ip) * DG(id, id, jp, ip);
            h_new[it] = h_new[it] + G3(id, ip) * DDG(id, jp, ip);
            h_new[it] = h_new[it] - G3(id, jp) * DDG(id, jp, ip);
            for (int jd = id + 1; jd < 2; jd++) {
              g_new[2 * ip + id] = g_new[2 * ip + id] + G3(jd, jp) * DG(jd, id, jp, ip);
              g_new[2 * ip + jd] = g_new[2 * ip + jd] + G3(id, jp) * DG(jd, id, jp, ip);
              g_new[2 * jp + id] = g_new[2 * jp + id] + G3(jd, ip) * DG(jd, id, jp, ip);
              g_new[2 * jp + jd] = g_new[2 * jp + jd] + G3(id, ip) * DG(jd, id, jp, ip);
              h_new[it] = h_new[it] - 4 * DG(jd, id, jp, ip) * DG(jd, id, jp, ip);
            }
          }
        }
      }
    }
    for (int jt = it + 1; jt < sys->ntypes; jt++) {
      if (sys->iu3[it][jt] < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++)
          for (int id = 0; id < 2; id++) {
            g_new[2 * ip + id] = g_new[2 * ip + id] + G3(id, jp) * DG(id, id, jp, ip);
            g_new[2 * jp + id] = g_new[2 * jp + id] + G3(id, ip) * DG(id, id, jp, ip);
            h_new[it] = h_new[it] - DG(id, id, jp, ip) * DG(id, id, jp, ip);
            h_new[jt] = h_new[jt] - DG(id, id, jp, ip) * DG(id, id, jp, ip);
            h_new[it] = h_new[it] - G3(id, jp) * DDG(id, jp, ip);
            h_new[jt] = h_new[jt] + G3(id, ip) * DDG(id, jp, ip);
            for (int jd = id + 1; jd < 2; jd++) {
              g_new[2 * ip + id] = g_new[2 * ip + id] + G3(jd, jp) * DG(jd, id, jp, ip);
              g_new[2 * ip + jd] = g_new[2 * ip + jd] + G3(id, jp) * DG(jd, id, jp, ip);
              g_new[2 * jp + id] = g_new[2 * jp + id] + G3(jd, ip) * DG(jd, id, jp, ip);
              g_new[2 * jp + jd] = g_new[2 * jp + jd] + G3(id, ip) * DG(jd, id, jp, ip);
              h_new[it] = h_new[it] - 2 * DG(jd, id, jp, ip) * DG(jd, id, jp, ip);
              h_new[jt] = h_new[jt] - 2 * DG(jd, id, jp, ip) * DG(jd, id, jp, ip);
            }
          }
    }
  }
}

/* three_body (reptation.f:2777-2864): l=1 factorised triplets. */
void oracle_three_body(const qmc2d_system *sys, oracle_work *w, double *ltf, double *g_new,
                       double *h_new) {
  int N = w->N;
  int any = 0;
  for (int it = 0; it < sys->ntypes; it++)
    for (int jt = it; jt < sys->ntypes; jt++) any |= (sys->iu3[it][jt] >= 0);
  if (!any) return;
  memset(w->g3, 0, sizeof(double) * 2 * N);
  memset(w->dg, 0, sizeof(double) * 4 * N * N);
  memset(w->ddg, 0, sizeof(double) * 2 * N * N);
  double t, dt, ddt;
  int ij = 0;
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    int i = sys->iu3[it][it];
    if (i >= 0) {
      for (int ip = f0; ip < l0; ip++)
        for (int jp = ip + 1; jp < l0; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          makeg(w, jp, ip, t, dt, ddt, &PRV(0, ij), w->pp_byr[ij]);
          double r = w->pp_r[ij];
          ddt = 2 * (t * t + 4 * r * t * dt + r * r * (dt * dt + ddt * t));
          dt = 2 * t * (t + r * dt);
          t = (t * r) * (t * r);
          *ltf = *ltf + t;
          for (int d = 0; d < 2; d++) {
            g_new[2 * ip + d] = g_new[2 * ip + d] + dt * PRV(d, ij);
            g_new[2 * jp + d] = g_new[2 * jp + d] - dt * PRV(d, ij);
          }
          h_new[it] = h_new[it] + 2 * (ddt + (2 - 1) * dt);
          ij++;
        }
    }
    for (int jt = it + 1; jt < sys->ntypes; jt++) {
      i = sys->iu3[it][jt];
      if (i < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          makeg(w, jp, ip, t, dt, ddt, &PRV(0, ij), w->pp_byr[ij]);
          double r = w->pp_r[ij];
          ddt = 2 * (t * t + 4 * r * t * dt + r * r * (dt * dt + ddt * t));
          dt = 2 * t * (t + r * dt);
          t = (t * r) * (t * r);
          *ltf = *ltf + t;
          for (int d = 0; d < 2; d++) {
            g_new[2 * ip + d] = g_new[2 * ip + d] + dt * PRV(d, ij);
            g_new[2 * jp + d] = g_new[2 * jp + d] - dt * PRV(d, ij);
          }
          h_new[it] = h_new[it] + ddt + (2 - 1) * dt;
          h_new[jt] = h_new[jt] + ddt + (2 - 1) * dt;
          ij++;
        }
    }
  }
  dotg(sys, w, ltf, g_new, h_new);
}
