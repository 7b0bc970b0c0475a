/*
 * oracle_walk.c - CPU oracle (TEST INFRASTRUCTURE ONLY): the walker moves
 * of VMC and DMC and the fixed-population branching, restated from
 * reptation.f.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* sigma (reptation.f:855-870) */
static double var_of(const qmc2d_system *sys, int it, double delta) {
  return sys->hbs2m[it] != 0.0 ? 2.0 * sys->hbs2m[it] * delta : 0.0;
}

/* move (reptation.f:4617-4680) + metropolis_test (reptation.f:2622-2659). */
double oracle_move(const qmc2d_system *sys, oracle_work *w, oracle_walker *wk, double delta,
                   int mage, oracle_uniform_fn U, void *ctx, double *xn, double *gn, double *pn,
                   int *accepted, double *elocal, int *status) {
  int nt = sys->ntypes;
  double hn[QMC2D_MAX_TYPES], sn;
  double wold = 0.0;
  const double pi = acos(-1.0);
  for (int it = 0; it < nt; it++) {
    if (sys->hbs2m[it] == 0.0) continue;
    double var = var_of(sys, it, delta), vari = 1.0 / var;
    double ww = 0.0;
    for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
      for (int d = 0; d < 2; d++) {
        int j = 2 * ip + d;
        double uc = U(ctx, 0, j);
        double ul = U(ctx, 1, j);
        double chi = cos(pi * uc) * sqrt(-2.0 * var * log(ul));
        ww = ww - chi * chi;
        double drift = -var * wk->g[j];
        xn[j] = chi + drift + wk->x[j];
      }
    wold = wold + ww * vari;
  }
  int uf = 0;
  *status = oracle_compute_properties(sys, w, xn, gn, hn, pn, &sn, &uf);
  double p;
  if (wk->age == mage) {
    p = 1.0;
  } else {
    double wnew = 0.0;
    for (int it = 0; it < nt; it++) {
      if (sys->hbs2m[it] == 0.0) continue;
      double var = var_of(sys, it, delta), vari = 1.0 / var;
      double ww = 0.0;
      for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
        for (int d = 0; d < 2; d++) {
          int j = 2 * ip + d;
          double drift = -var * gn[j];
          double chi = wk->x[j] - xn[j] - drift;
          ww = ww - chi * chi;
        }
      wnew = wnew + ww * vari;
    }
    p = (wk->p[QMC2D_JLTF] - pn[QMC2D_JLTF]) * 2 + 0.5 * (wnew - wold);
    p = p < -50.0 ? -50.0 : p;
    p = p > 0.0 ? 0.0 : p;
    p = exp(p);
  }
  /* metropolis_test */
  double xr = 1.0;
  if (p < 1.0) xr = U(ctx, 2, 0);
  if (p >= xr) {
    *accepted = 1;
    wk->age = 0;
    *elocal = 0.5 * (pn[QMC2D_JETOT] + wk->p[QMC2D_JETOT]);
    memcpy(wk->x, xn, sizeof(double) * 2 * sys->nptot);
    memcpy(wk->g, gn, sizeof(double) * 2 * sys->nptot);
    for (int it = 0; it < nt; it++) wk->h[it] = hn[it];
    memcpy(wk->p, pn, sizeof(double) * sys->n_props);
    wk->s = sn;
  } else {
    *accepted = 0;
    wk->age = wk->age + 1;
    *elocal = wk->p[QMC2D_JETOT];
  }
  wk->p[QMC2D_JACC] = p;
  return p;
}

/* ------------------------------------------- the reference's own stream */

typedef struct {
  oracle_rng rng;
  int order;
  int have;
  double cached;
} rannyu_ctx;

/* Both draws of a Gaussian come from one rannyu() each, in the order the
 * compiled reference evaluated cos(pi*rannyu())*sqrt(-2 var log(rannyu())). */
static double rannyu_draw(void *vctx, int kind, int j) {
  (void)j;
  rannyu_ctx *c = (rannyu_ctx *)vctx;
  if (kind == 2 || c->order == 0) return oracle_rannyu(&c->rng);
  if (kind == 0) {
    c->cached = oracle_rannyu(&c->rng); /* log argument drawn first */
    c->have = 1;
    return oracle_rannyu(&c->rng);
  }
  c->have = 0;
  return c->cached;
}

int oracle_vmc_rannyu(const qmc2d_system *sys, const double *x0, int nstp, double delta,
                      int mage, const int seed[4], int rng_order, double *blk, double *x_final,
                      int seed_out[4], long *naccept) {
  int N = sys->nptot, np_ = sys->n_props;
  qmc2d_system s2 = *sys;
  s2.delta = delta;
  oracle_work *w = oracle_work_new(&s2);
  rannyu_ctx ctx;
  int sd[4] = {seed[0], seed[1], seed[2], 2 * (seed[3] + 0) + 1}; /* reptation.f:38 */
  oracle_setrn(&ctx.rng, sd);
  ctx.order = rng_order;
  ctx.have = 0;
  oracle_walker wk;
  wk.x = (double *)malloc(sizeof(double) * 2 * N);
  wk.g = (double *)malloc(sizeof(double) * 2 * N);
  wk.p = (double *)malloc(sizeof(double) * np_);
  double *xn = (double *)malloc(sizeof(double) * 2 * N);
  double *gn = (double *)malloc(sizeof(double) * 2 * N);
  double *pn = (double *)malloc(sizeof(double) * np_);
  /* read_conf: evaluate, then metropolis_test(1) accepts (reptation.f:2480-2489) */
  int st = oracle_compute_properties(&s2, w, x0, wk.g, wk.h, wk.p, &wk.s, NULL);
  memcpy(wk.x, x0, sizeof(double) * 2 * N);
  wk.age = 0;
  wk.p[QMC2D_JACC] = 1.0;
  memset(blk, 0, sizeof(double) * np_);
  long nacc = 0;
  for (int istp = 0; istp < nstp && st == 0; istp++) {
    int acc;
    double el;
    oracle_move(&s2, w, &wk, delta, mage, rannyu_draw, &ctx, xn, gn, pn, &acc, &el, &st);
    nacc += acc;
    for (int i = 0; i < np_; i++) blk[i] = blk[i] + wk.p[i] * 1.0; /* averages(2) */
  }
  memcpy(x_final, wk.x, sizeof(double) * 2 * N);
  oracle_savern(&ctx.rng, seed_out);
  if (naccept) *naccept = nacc;
  free(wk.x); free(wk.g); free(wk.p); free(xn); free(gn); free(pn);
  oracle_work_free(w);
  return st;
}

/* -------------------------------------------------- Philox device streams */

typedef struct {
  uint64_t seed;
  uint32_t c1, c2, c3;
} philox_ctx;

static double philox_draw(void *vctx, int kind, int j) {
  philox_ctx *c = (philox_ctx *)vctx;
  double u[2];
  if (kind == 2) {
    oracle_philox_uniform2(c->seed, 0xFFFFFFFEu, c->c1, c->c2, c->c3, u);
    return u[0];
  }
  oracle_philox_uniform2(c->seed, (uint32_t)j, c->c1, c->c2, c->c3, u);
  return u[kind];
}

int oracle_population_init(const qmc2d_system *sys, int nw, const double *x, double *g,
                           double *hl, double *p, double *s, double *age) {
  int N = sys->nptot, np_ = sys->n_props, nt = sys->ntypes;
  oracle_work *w = oracle_work_new(sys);
  int st = 0;
  for (int k = 0; k < nw && st == 0; k++) {
    st = oracle_compute_properties(sys, w, x + (size_t)2 * N * k, g + (size_t)2 * N * k,
                                   hl + (size_t)nt * k, p + (size_t)np_ * k, s + k, NULL);
    p[(size_t)np_ * k + QMC2D_JACC] = 1.0;
    age[k] = 0.0;
  }
  oracle_work_free(w);
  return st;
}

static void walker_view(const qmc2d_system *sys, oracle_walker *wk, int k, double *x, double *g,
                        double *hl, double *p, double *s, double *age) {
  int N = sys->nptot, np_ = sys->n_props, nt = sys->ntypes;
  wk->x = x + (size_t)2 * N * k;
  wk->g = g + (size_t)2 * N * k;
  wk->p = p + (size_t)np_ * k;
  for (int it = 0; it < nt; it++) wk->h[it] = hl[(size_t)nt * k + it];
  wk->s = s[k];
  wk->age = age[k];
}

static void walker_store(const qmc2d_system *sys, const oracle_walker *wk, int k, double *hl,
                         double *s, double *age) {
  int nt = sys->ntypes;
  for (int it = 0; it < nt; it++) hl[(size_t)nt * k + it] = wk->h[it];
  s[k] = wk->s;
  age[k] = wk->age;
}

int oracle_vmc_philox(const qmc2d_system *sys, int nw, int nstp, double delta, int mage,
                      uint64_t seed, long step0, double *x, double *g, double *hl, double *p,
                      double *s, double *age, double *blk, long *naccept) {
  int N = sys->nptot, np_ = sys->n_props;
  qmc2d_system s2 = *sys;
  s2.delta = delta;
  oracle_work *w = oracle_work_new(&s2);
  double *xn = (double *)malloc(sizeof(double) * 2 * N);
  double *gn = (double *)malloc(sizeof(double) * 2 * N);
  double *pn = (double *)malloc(sizeof(double) * np_);
  long nacc = 0;
  int st = 0;
  for (int k = 0; k < nw && st == 0; k++) {
    oracle_walker wk;
    walker_view(&s2, &wk, k, x, g, hl, p, s, age);
    for (int istp = 0; istp < nstp && st == 0; istp++) {
      philox_ctx ctx = {seed, (uint32_t)k, (uint32_t)(step0 + istp), 0u};
      int acc;
      double el;
      oracle_move(&s2, w, &wk, delta, mage, philox_draw, &ctx, xn, gn, pn, &acc, &el, &st);
      nacc += acc;
      if (blk)
        for (int i = 0; i < np_; i++) blk[i] = blk[i] + wk.p[i];
    }
    walker_store(&s2, &wk, k, hl, s, age);
  }
  if (naccept) *naccept = nacc;
  free(xn); free(gn); free(pn);
  oracle_work_free(w);
  return st;
}

/* branch2 for one rank (reptation.f:2162-2273) with prov_dest's in-rank
 * redistribution (reptation.f:2260-2271, 2320-2345). */
int oracle_branch2(int nw, double *wate, const double *r, int *mult, int *src, int *ncapped) {
  const double wmult = 10.0;
  int nc = 0;
  for (int i = 0; i < nw; i++)
    if (wate[i] > wmult) {
      wate[i] = wmult;
      nc++;
    }
  if (ncapped) *ncapped = nc;
  double somma = 0.0;
  for (int i = 0; i < nw; i++) somma = somma + wate[i];
  double *delt = (double *)malloc(sizeof(double) * nw);
  double k0 = 0.0;
  for (int i = 0; i < nw; i++) {
    double ww = nw * wate[i] / somma;
    mult[i] = (int)ww;
    delt[i] = ww - mult[i];
    k0 = k0 + delt[i];
  }
  int ncomb = (int)round(k0);
  int nwi = -1; /* 0-based: the reference's nw - 1 */
  double k = 1.0;
  int used = 0;
  for (int i = 0; i < ncomb; i++) {
    double rr = r[used++];
    k = k - 1.0;
    while (k < rr && nwi < nw - 1) {
      nwi++;
      k = k + delt[nwi];
    }
    if (nwi < 0) nwi = 0;
    mult[nwi] = mult[nwi] + 1;
    while (k < 1.0 && nwi < nw - 1) {
      nwi++;
      k = k + delt[nwi];
    }
  }
  free(delt);
  int *m = (int *)malloc(sizeof(int) * nw);
  memcpy(m, mult, sizeof(int) * nw);
  for (int j = 0; j < nw; j++) src[j] = j;
  for (int j = 0; j < nw; j++) {
    if (m[j] != 0) continue;
    for (int i = 0; i < nw; i++)
      if (m[i] >= 2) {
        src[j] = i;
        m[i]--;
        m[j]++;
        break;
      }
  }
  free(m);
  return used;
}

int oracle_dmc_philox(const qmc2d_system *sys, int nw, int ngen, int mmstep, double delta,
                      double etrial, double mmult, int mage, uint64_t seed, long gen0,
                      long move0, double *x, double *g, double *hl, double *p, double *s,
                      double *age, double *blk, double *blk_norm, long *naccept) {
  int N = sys->nptot, np_ = sys->n_props, nt = sys->ntypes;
  qmc2d_system s2 = *sys;
  s2.delta = delta;
  oracle_work *w = oracle_work_new(&s2);
  double *xn = (double *)malloc(sizeof(double) * 2 * N);
  double *gn = (double *)malloc(sizeof(double) * 2 * N);
  double *pn = (double *)malloc(sizeof(double) * np_);
  double *wate = (double *)malloc(sizeof(double) * nw);
  double *r = (double *)malloc(sizeof(double) * (nw + 1));
  int *mult = (int *)malloc(sizeof(int) * nw);
  int *src = (int *)malloc(sizeof(int) * nw);
  double *x2 = (double *)malloc(sizeof(double) * 2 * N * nw);
  double *g2 = (double *)malloc(sizeof(double) * 2 * N * nw);
  double *h2 = (double *)malloc(sizeof(double) * nt * nw);
  double *p2 = (double *)malloc(sizeof(double) * np_ * nw);
  double *sv = (double *)malloc(sizeof(double) * nw);
  double *av = (double *)malloc(sizeof(double) * nw);
  long nacc = 0;
  int st = 0;
  for (int gen = 0; gen < ngen && st == 0; gen++) {
    for (int k = 0; k < nw; k++) wate[k] = 1.0;
    for (int k = 0; k < nw && st == 0; k++) {
      oracle_walker wk;
      walker_view(&s2, &wk, k, x, g, hl, p, s, age);
      for (int ms = 0; ms < mmstep && st == 0; ms++) {
        long mv = move0 + (long)gen * mmstep + ms;
        philox_ctx ctx = {seed, (uint32_t)k, (uint32_t)mv, 0u};
        int acc;
        double el;
        oracle_move(&s2, w, &wk, delta, mage, philox_draw, &ctx, xn, gn, pn, &acc, &el, &st);
        nacc += acc;
        double peso = exp(-sys->npnorm * (el - etrial) * delta);
        if (peso > mmult) peso = mmult;
        wate[k] = wate[k] * peso;
        for (int i = 0; i < np_; i++) blk[i] = blk[i] + wk.p[i] * wate[k];
        *blk_norm = *blk_norm + wate[k];
      }
      walker_store(&s2, &wk, k, hl, s, age);
    }
    if (st) break;
    for (int i = 0; i < nw; i++) {
      double u[2];
      oracle_philox_uniform2(seed, (uint32_t)i, 0xFFFFFFFFu, (uint32_t)(gen0 + gen), 1u, u);
      r[i] = u[0];
    }
    r[nw] = 0.5;
    oracle_branch2(nw, wate, r, mult, src, NULL);
    memcpy(x2, x, sizeof(double) * 2 * N * nw);
    memcpy(g2, g, sizeof(double) * 2 * N * nw);
    memcpy(h2, hl, sizeof(double) * nt * nw);
    memcpy(p2, p, sizeof(double) * np_ * nw);
    memcpy(sv, s, sizeof(double) * nw);
    memcpy(av, age, sizeof(double) * nw);
    for (int j = 0; j < nw; j++) {
      int i = src[j];
      memcpy(x + (size_t)2 * N * j, x2 + (size_t)2 * N * i, sizeof(double) * 2 * N);
      memcpy(g + (size_t)2 * N * j, g2 + (size_t)2 * N * i, sizeof(double) * 2 * N);
      memcpy(hl + (size_t)nt * j, h2 + (size_t)nt * i, sizeof(double) * nt);
      memcpy(p + (size_t)np_ * j, p2 + (size_t)np_ * i, sizeof(double) * np_);
      s[j] = sv[i];
      age[j] = av[i];
    }
  }
  if (naccept) *naccept = nacc;
  free(xn); free(gn); free(pn); free(wate); free(r); free(mult); free(src);
  free(x2); free(g2); free(h2); free(p2); free(sv); free(av);
  oracle_work_free(w);
  return st;
}
