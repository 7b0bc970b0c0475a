/*
 * oracle_props.c - CPU oracle (TEST INFRASTRUCTURE ONLY): kinetic and
 * potential energy and compute_properties, restated from reptation.f.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* kinetic (reptation.f:2729-2775) */
static void kinetic(const qmc2d_system *sys, oracle_work *w, double *g_new, const double *h_new,
                    double *p) {
  int nt = sys->ntypes;
  int n_jgg = 0;
  double gg = 1.0;
  p[QMC2D_JKIN0] = 0.0;
  p[QMC2D_JGG] = 0.0;
  for (int it = 0; it < nt; it++) {
    if (sys->hbs2m[it] == 0.0) continue;
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    double g2 = 0.0;
    if (sys->adrift == 0.0) {
      for (int ip = f0; ip < l0; ip++)
        for (int d = 0; d < 2; d++) g2 = g2 + g_new[2 * ip + d] * g_new[2 * ip + d];
      p[QMC2D_JGG] = 1.0;
      n_jgg = 1;
    } else {
      double vari = 1.0 / (2.0 * sys->hbs2m[it] * sys->delta);
      for (int ip = f0; ip < l0; ip++) {
        double x2 = 0.0;
        for (int d = 0; d < 2; d++) x2 = x2 + g_new[2 * ip + d] * g_new[2 * ip + d];
        gg = x2 * sys->adrift * sys->delta * sys->delta * vari;
        gg = (-1.0 + sqrt(1.0 + 2.0 * gg)) / gg;
        p[QMC2D_JGG] = p[QMC2D_JGG] + gg;
        n_jgg = n_jgg + 1;
        for (int d = 0; d < 2; d++) g_new[2 * ip + d] = g_new[2 * ip + d] * gg;
        g2 = g2 + x2;
      }
    }
    int jk = QMC2D_JKIN(nt, it);
    p[jk] = sys->hbs2m[it] * (h_new[it] - g2);
    p[QMC2D_JKIN0] = p[QMC2D_JKIN0] + p[jk];
    p[jk] = p[jk] / sys->np[it];
    p[QMC2D_JUN(nt, it)] = 1.0 / sqrt(g2);
  }
  p[QMC2D_JKIN0] = p[QMC2D_JKIN0] / sys->npnorm;
  p[QMC2D_JGG] = p[QMC2D_JGG] / n_jgg;
  if (sys->ntheta != 0) p[QMC2D_JEFP(nt)] = w->grad2_ph / sys->npnorm;
}

/* potential (reptation.f:3986-4101): real-space spline of the pair
 * potential times (1/r)**iexp plus tails, and the k-space sum over ordered
 * type pairs of v_k (rho_k^a . rho_k^b) plus v_k0*npnorm. rho_k is read by
 * type index as the reference does (rhok(ik,it), reptation.f:4042). */
static void potential(const qmc2d_system *sys, oracle_work *w, double *p) {
  int nt = sys->ntypes;
  double p2t[QMC2D_MAX_TYPES] = {0.0, 0.0}, p2tot = 0.0;
  const double v = 1.0; /* v2value: the 7th word of 'v2' is not read (reptation.f:252) */
  int ij = 0;
  for (int it = 0; it < nt; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    int i = sys->iv2[it][it];
    if (i >= 0) {
      double aux = sys->np[it] * (sys->np[it] - 1) * 0.5 * sys->tables[i].tail * v;
      p2t[it] = p2t[it] + aux;
      p2tot = p2tot + aux;
      for (int ip = f0; ip < l0; ip++)
        for (int jp = ip + 1; jp < l0; jp++) {
          double f = getf_0(sys, i, w->pp_ind[ij], w->pp_rem[ij], w->pp_byr[ij]);
          p2t[it] = p2t[it] + f * v;
          p2tot = p2tot + f * v;
          ij++;
        }
    }
    for (int jt = it + 1; jt < nt; jt++) {
      i = sys->iv2[it][jt];
      if (i < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      double aux = sys->np[it] * sys->np[jt] * sys->tables[i].tail * v;
      p2t[it] = p2t[it] + 0.5 * aux;
      p2t[jt] = p2t[jt] + 0.5 * aux;
      p2tot = p2tot + aux;
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++) {
          double f = getf_0(sys, i, w->pp_ind[ij], w->pp_rem[ij], w->pp_byr[ij]);
          p2t[it] = p2t[it] + 0.5 * f * v;
          p2t[jt] = p2t[jt] + 0.5 * f * v;
          p2tot = p2tot + f * v;
          ij++;
        }
    }
  }
  for (int it = 0; it < nt; it++)
    for (int jt = 0; jt < nt; jt++) {
      int iv = sys->iv2[it][jt];
      if (iv < 0) continue;
      const qmc2d_table *tb = &sys->tables[iv];
      if (tb->nk_ewald == 0) continue;
      const double *ra = w->rhok + (size_t)2 * sys->nk * it;
      const double *rb = w->rhok + (size_t)2 * sys->nk * jt;
      double aux = 0.0;
      for (int ik = 0; ik < tb->nk_ewald; ik++)
        aux = aux + tb->vk[ik] * (ra[2 * ik] * rb[2 * ik] + ra[2 * ik + 1] * rb[2 * ik + 1]);
      p2t[it] = p2t[it] + aux + tb->vk[tb->nk_ewald] * sys->npnorm;
      p2tot = p2tot + aux + tb->vk[tb->nk_ewald] * sys->npnorm;
    }
  p[QMC2D_JPOT0] = p2tot;
  for (int it = 0; it < nt; it++) p[QMC2D_JPOT(nt, it)] = p2t[it] / sys->np[it];
  p[QMC2D_JPOT0] = (p[QMC2D_JPOT0] + sys->v0) / sys->npnorm;
}

/* compute_properties(1) (reptation.f:2661-2727) with trial_function
 * (reptation.f:3048-3063). */
int oracle_compute_properties(const qmc2d_system *sys, oracle_work *w, const double *x,
                              double *g, double *hl, double *p, double *s, int *underflow) {
  int nt = sys->ntypes;
  int N = sys->nptot;
  int uf = 0;
  memset(p, 0, sizeof(double) * sys->n_props);
  oracle_distances(sys, w, x);
  double ltf = 0.0;
  memset(g, 0, sizeof(double) * 2 * N);
  for (int it = 0; it < nt; it++) hl[it] = 0.0;
  *s = 1.0;
  oracle_two_body(sys, w, &ltf, g, hl);
  oracle_three_body(sys, w, &ltf, g, hl);
  int st = oracle_slater(sys, w, x, &ltf, g, hl, &uf);
  if (underflow) *underflow = uf;
  if (st) return st;
  p[QMC2D_JLTF] = ltf;
  kinetic(sys, w, g, hl, p);
  potential(sys, w, p);
  p[QMC2D_JETOT] = p[QMC2D_JPOT0] + p[QMC2D_JKIN0] + p[QMC2D_JEFP(nt)];
  p[QMC2D_JE2] = p[QMC2D_JETOT] * p[QMC2D_JETOT];
  int i = 0;
  for (int it = 0; it < nt; it++) {
    if (sys->irhok[it] == 0) continue;
    const double *rk = w->rhok + (size_t)2 * sys->nk * it;
    for (int ik = 0; ik < sys->nk; ik++) {
      p[sys->jrhok + i] = rk[2 * ik];
      p[sys->jrhok + i + 1] = rk[2 * ik + 1];
      i += 2;
    }
  }
  return 0;
}
