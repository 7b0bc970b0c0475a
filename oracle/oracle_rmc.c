/*
 * oracle_rmc.c - CPU oracle (TEST INFRASTRUCTURE ONLY): reptation QMC for
 * one reptile, restated from reptation.f (rmc :1286, read_path :1775,
 * get_w_stack :1804, fgg :1853, reptation_metropolis_test :1865,
 * reptation_move :1897, path_props scalar part :1556-1577). Random draws
 * come from the Philox streams documented in qmc2d_oracle.h.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

enum { JBRA = 0, JDTP = 1, JITP = 2, JLNG = 3, JNDS = 4 };

struct oracle_reptile {
  qmc2d_rmc_params prm;
  qmc2d_system sys; /* copy with delta set */
  int nbuf, N, npr, nt;
  double *x, *g, *p, *h, *s, *age_stack, *w;
  int jfirst, jlast, kfirst, klast;
  double *pp_new, *pp_old;
  double age;
  int idir, ndelta;
  oracle_work *wk;
  double *xn, *gn, *pn;
  double hn[QMC2D_MAX_TYPES], sn;
  double var[QMC2D_MAX_TYPES], vari[QMC2D_MAX_TYPES];
};

#define XS(r, j) ((r)->x + (size_t)2 * (r)->N * (j))
#define GS(r, j) ((r)->g + (size_t)2 * (r)->N * (j))
#define PS(r, j) ((r)->p + (size_t)(r)->npr * (j))
#define WS(r, j, k) ((r)->w[(size_t)5 * (j) + (k)])

oracle_reptile *oracle_reptile_new(const qmc2d_system *sys, const qmc2d_rmc_params *prm) {
  oracle_reptile *r = (oracle_reptile *)calloc(1, sizeof(oracle_reptile));
  r->prm = *prm;
  r->sys = *sys;
  r->sys.delta = prm->delta;
  r->nbuf = prm->ntau + prm->mdelta;
  r->N = sys->nptot;
  r->npr = sys->n_props;
  r->nt = sys->ntypes;
  size_t nb = (size_t)r->nbuf;
  r->x = (double *)calloc(nb * 2 * r->N, sizeof(double));
  r->g = (double *)calloc(nb * 2 * r->N, sizeof(double));
  r->p = (double *)calloc(nb * r->npr, sizeof(double));
  r->h = (double *)calloc(nb * r->nt, sizeof(double));
  r->s = (double *)calloc(nb, sizeof(double));
  r->age_stack = (double *)calloc(nb, sizeof(double));
  r->w = (double *)calloc(nb * 5, sizeof(double));
  r->pp_new = (double *)calloc((size_t)r->npr, sizeof(double));
  r->pp_old = (double *)calloc((size_t)r->npr, sizeof(double));
  r->xn = (double *)calloc((size_t)2 * r->N, sizeof(double));
  r->gn = (double *)calloc((size_t)2 * r->N, sizeof(double));
  r->pn = (double *)calloc((size_t)r->npr, sizeof(double));
  r->wk = oracle_work_new(&r->sys);
  for (int it = 0; it < r->nt; it++) {
    r->var[it] = sys->hbs2m[it] != 0.0 ? 2.0 * sys->hbs2m[it] * prm->delta : 0.0;
    r->vari[it] = r->var[it] != 0.0 ? 1.0 / r->var[it] : 0.0;
  }
  return r;
}

void oracle_reptile_free(oracle_reptile *r) {
  if (!r) return;
  free(r->x); free(r->g); free(r->p); free(r->h); free(r->s); free(r->age_stack);
  free(r->w); free(r->pp_new); free(r->pp_old); free(r->xn); free(r->gn); free(r->pn);
  oracle_work_free(r->wk);
  free(r);
}

/* fgg (reptation.f:1853-1863) */
static double fgg(const oracle_reptile *r, double e, double gg) {
  if (r->sys.ecut == 0) return e;
  return r->sys.value_ecut + (e - r->sys.value_ecut) * gg;
}

/* path_props, scalar part (reptation.f:1567-1577) */
static void path_props(oracle_reptile *r) {
  int ntau = r->prm.ntau, sk = r->prm.ntauskip;
  for (int ip = 0; ip < r->npr; ip++) {
    r->pp_new[ip] = 0.0;
    for (int i = 1 + sk; i <= ntau - sk; i++) {
      int j = (r->kfirst + i - 1) % r->nbuf;
      r->pp_new[ip] = r->pp_new[ip] + PS(r, j)[ip];
    }
    r->pp_new[ip] = r->pp_new[ip] / (ntau - 2 * sk);
  }
  r->pp_new[QMC2D_JETOT] = 0.5 * (PS(r, r->klast)[QMC2D_JETOT] + PS(r, r->kfirst)[QMC2D_JETOT]);
}

/* get_w_stack (reptation.f:1804-1851) */
static void get_w_stack(oracle_reptile *r, int j, int jn, double *wnew, double *wold) {
  const qmc2d_system *sys = &r->sys;
  int nt = r->nt;
  double lng = 0.0;
  *wold = 0.0;
  *wnew = 0.0;
  for (int it = 0; it < nt; it++) {
    if (sys->hbs2m[it] == 0.0) continue;
    double wf = 0.0, wb = 0.0, wg = 0.0;
    for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
      for (int d = 0; d < 2; d++) {
        int k = 2 * ip + d;
        double a = XS(r, j)[k] - XS(r, jn)[k];
        wg = wg - a * a;
        double df = -r->var[it] * GS(r, j)[k];
        double b = XS(r, j)[k] + df - XS(r, jn)[k];
        wf = wf - b * b;
        double db = -r->var[it] * GS(r, jn)[k];
        double c = XS(r, j)[k] - db - XS(r, jn)[k];
        wb = wb - c * c;
      }
    *wnew = *wnew + wb * r->vari[it];
    *wold = *wold + wf * r->vari[it];
    lng = lng + wg * r->vari[it];
  }
  lng = lng + r->prm.delta * sys->npnorm * (PS(r, j)[QMC2D_JKIN0] + PS(r, jn)[QMC2D_JKIN0]);
  WS(r, j, JLNG) = 0.5 * lng;
  WS(r, j, JDTP) = 0.5 * *wold;
  WS(r, j, JBRA) = -.5 * r->prm.delta * sys->npnorm *
                   (fgg(r, PS(r, j)[QMC2D_JETOT], PS(r, j)[QMC2D_JGG]) +
                    fgg(r, PS(r, jn)[QMC2D_JETOT], PS(r, jn)[QMC2D_JGG]) - 2.0 * r->prm.etrial);
  WS(r, jn, JITP) = 0.5 * *wnew;
  WS(r, j, JNDS) = 0.0;
  for (int it = 0; it < nt; it++) {
    if (sys->hbs2m[it] == 0.0) continue;
    int ju = QMC2D_JUN(nt, it);
    WS(r, j, JNDS) = WS(r, j, JNDS) -
                     log(1.0 - exp(-PS(r, j)[ju] * PS(r, jn)[ju] / (0.5 * r->var[it])));
  }
}

int oracle_reptile_init(const qmc2d_system *sys, oracle_reptile *r, const double *x) {
  (void)sys;
  int N = r->N, ntau = r->prm.ntau;
  /* read_conf with ntarget = ntau: bead i in stack slot i (reptation.f:1780) */
  for (int i = 0; i < ntau; i++) {
    memcpy(XS(r, i), x + (size_t)2 * N * i, sizeof(double) * 2 * N);
    int st = oracle_compute_properties(&r->sys, r->wk, XS(r, i), GS(r, i), r->h + r->nt * i,
                                       PS(r, i), &r->s[i], NULL);
    if (st) return st;
    PS(r, i)[QMC2D_JACC] = 1.0;
    r->age_stack[i] = 0.0;
  }
  r->kfirst = 0;
  r->klast = ntau - 1;
  path_props(r);
  r->jfirst = r->kfirst;
  r->jlast = r->klast;
  for (int i = 1; i <= ntau - 1; i++) {
    int j = (r->jfirst + i - 1) % r->nbuf;
    int jn = (r->jfirst + i) % r->nbuf;
    double wnew, wold;
    get_w_stack(r, j, jn, &wnew, &wold);
    double p = 2 * (PS(r, j)[QMC2D_JLTF] - PS(r, jn)[QMC2D_JLTF]) + 0.5 * (wnew - wold);
    p = p < -50.0 ? -50.0 : p;
    p = p > 0.0 ? 0.0 : p;
    PS(r, jn)[QMC2D_JACC] = exp(p);
  }
  memcpy(r->pp_old, r->pp_new, sizeof(double) * r->npr);
  r->age = 0.0;
  return 0;
}

static double u1(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, int k) {
  double u[2];
  oracle_philox_uniform2(seed, c0, c1, c2, c3, u);
  return u[k];
}

/* reptation_move (reptation.f:1897-2160); returns wnew, sets *st. */
static double reptation_move(oracle_reptile *r, int rid, uint64_t seed, uint32_t t, int *st) {
  const qmc2d_system *sys = &r->sys;
  int nt = r->nt, nb = r->nbuf;
  double half = 0.5, one = 0.0, one_nds = 0.0, mezzo = 0.0;
  if (sys->wpiu != 0) {
    mezzo = 0.5;
  } else if (sys->gstorto != 0) {
    half = 0.0;
    one = 1.0;
    if (sys->nodalaction != 0) one_nds = 1.0;
  }
  const double pi = acos(-1.0);
  double ud = u1(seed, 0xFFFFFFF0u, (uint32_t)rid, t, 2u, 0);
  double ul = u1(seed, 0xFFFFFFF0u, (uint32_t)rid, t, 2u, 1);
  r->idir = (ud - 0.5) >= 0.0 ? 1 : -1; /* int(sign(1, rannyu()-0.5)) */
  r->ndelta = 1 + (int)(ul * r->prm.mdelta);
  int jstart = r->idir == 1 ? r->jlast : r->jfirst;
  *st = 0;
  for (int idelta = 1; idelta <= r->ndelta; idelta++) {
    int j = (jstart + r->idir * (idelta - 1) + nb) % nb;
    int jn = (jstart + r->idir * idelta + nb) % nb;
    uint32_t c3 = 3u + (uint32_t)(idelta - 1);
    double wold = 0.0, lng = 0.0, dold = 0.0;
    for (int it = 0; it < nt; it++) {
      if (sys->hbs2m[it] == 0.0) continue;
      double ww = 0.0, wg = 0.0, d = 0.0;
      for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
        for (int dd = 0; dd < 2; dd++) {
          int k = 2 * ip + dd;
          double drift = -r->var[it] * GS(r, j)[k];
          d = d + drift * drift;
          double u[2];
          oracle_philox_uniform2(seed, (uint32_t)k, (uint32_t)rid, t, c3, u);
          double chi = cos(pi * u[0]) * sqrt(-2.0 * r->var[it] * log(u[1]));
          ww = ww - chi * chi;
          r->xn[k] = chi + drift + XS(r, j)[k];
          wg = wg - (chi + drift) * (chi + drift);
        }
      wold = wold + ww * r->vari[it];
      dold = dold + d * r->vari[it];
      lng = lng + wg * r->vari[it];
    }
    *st = oracle_compute_properties(sys, r->wk, r->xn, r->gn, r->hn, r->pn, &r->sn, NULL);
    if (*st) return 0.0;
    double wnew = 0.0;
    for (int it = 0; it < nt; it++) {
      if (sys->hbs2m[it] == 0.0) continue;
      double ww = 0.0;
      for (int ip = sys->ipfrst[it]; ip < sys->ipfrst[it] + sys->np[it]; ip++)
        for (int dd = 0; dd < 2; dd++) {
          int k = 2 * ip + dd;
          double drift = -r->var[it] * r->gn[k];
          double chi = XS(r, j)[k] - r->xn[k] - drift;
          ww = ww - chi * chi;
        }
      wnew = wnew + ww * r->vari[it];
    }
    double p = 2 * (PS(r, j)[QMC2D_JLTF] - r->pn[QMC2D_JLTF]) + 0.5 * (wnew - wold);
    p = p < -50.0 ? -50.0 : p;
    p = p > 0.0 ? 0.0 : p;
    p = exp(p);
    if (sys->rejection == 0) {
      p = 1.0;
    } else if (r->age_stack[j] == r->prm.mage) {
      p = 1.0;
    }
    if (r->s[j] * r->sn < 0.0) p = 0.0;
    double wg = r->prm.delta * sys->npnorm * (PS(r, j)[QMC2D_JKIN0] + r->pn[QMC2D_JKIN0]);
    double ua = u1(seed, 0xFFFFFFFEu, (uint32_t)rid, t, c3, 0);
    const double *pj = PS(r, j);
    if (p < ua) {
      /* reject this bead: copy bead j forward (reptation.f:2023-2075) */
      int a = r->idir == 1 ? j : jn, b = r->idir == 1 ? jn : j;
      WS(r, a, JDTP) = 0.5 * dold;
      WS(r, a, JBRA) = -r->prm.delta * sys->npnorm *
                       (fgg(r, pj[QMC2D_JETOT], pj[QMC2D_JGG]) - r->prm.etrial);
      WS(r, b, JITP) = 0.5 * dold;
      WS(r, a, JLNG) = 0.5 * wg;
      WS(r, a, JNDS) = 0.0;
      for (int it = 0; it < nt; it++) {
        if (sys->hbs2m[it] == 0.0) continue;
        int ju = QMC2D_JUN(nt, it);
        WS(r, a, JNDS) = WS(r, a, JNDS) - log(1.0 - exp(-pj[ju] * pj[ju] / (0.5 * r->var[it])));
      }
      r->age_stack[jn] = r->age_stack[j] + 1;
      r->s[jn] = r->s[j];
      memcpy(XS(r, jn), XS(r, j), sizeof(double) * 2 * r->N);
      memcpy(GS(r, jn), GS(r, j), sizeof(double) * 2 * r->N);
      for (int it = 0; it < nt; it++) r->h[nt * jn + it] = r->h[nt * j + it];
      memcpy(PS(r, jn), PS(r, j), sizeof(double) * r->npr);
    } else {
      /* accept this bead (reptation.f:2076-2126) */
      lng = lng + wg;
      int a = r->idir == 1 ? j : jn, b = r->idir == 1 ? jn : j;
      WS(r, a, JDTP) = r->idir == 1 ? 0.5 * wold : 0.5 * wnew;
      WS(r, a, JBRA) = -0.5 * r->prm.delta * sys->npnorm *
                       ((fgg(r, pj[QMC2D_JETOT], pj[QMC2D_JGG]) +
                         fgg(r, r->pn[QMC2D_JETOT], r->pn[QMC2D_JGG])) -
                        2.0 * r->prm.etrial);
      WS(r, b, JITP) = r->idir == 1 ? 0.5 * wnew : 0.5 * wold;
      WS(r, a, JLNG) = 0.5 * lng;
      WS(r, a, JNDS) = 0.0;
      for (int it = 0; it < nt; it++) {
        if (sys->hbs2m[it] == 0.0) continue;
        int ju = QMC2D_JUN(nt, it);
        WS(r, a, JNDS) =
            WS(r, a, JNDS) - log(1.0 - exp(-pj[ju] * r->pn[ju] / (0.5 * r->var[it])));
      }
      r->age_stack[jn] = 0.0;
      r->s[jn] = r->sn;
      memcpy(XS(r, jn), r->xn, sizeof(double) * 2 * r->N);
      memcpy(GS(r, jn), r->gn, sizeof(double) * 2 * r->N);
      for (int it = 0; it < nt; it++) r->h[nt * jn + it] = r->hn[it];
      memcpy(PS(r, jn), r->pn, sizeof(double) * r->npr);
    }
    PS(r, jn)[QMC2D_JACC] = p;
  }
  r->kfirst = (r->jfirst + r->idir * r->ndelta + nb) % nb;
  r->klast = (r->jlast + r->idir * r->ndelta + nb) % nb;
  path_props(r);
  double wn = (-PS(r, r->kfirst)[QMC2D_JLTF] * (1 + 2 * mezzo) -
               PS(r, r->klast)[QMC2D_JLTF] * (1 - 2 * mezzo) +
               PS(r, r->jfirst)[QMC2D_JLTF] * (1 + 2 * mezzo) +
               PS(r, r->jlast)[QMC2D_JLTF] * (1 - 2 * mezzo));
  if (r->idir == 1) {
    for (int idelta = 1; idelta <= r->ndelta; idelta++) {
      int j = (r->jfirst + r->idir * (idelta - 1) + nb) % nb;
      int jn = (r->jfirst + r->idir * idelta + nb) % nb;
      wn = wn - WS(r, j, JBRA) - WS(r, j, JDTP) * (half + mezzo) +
           WS(r, jn, JITP) * (one + half + mezzo) - WS(r, j, JLNG) * one +
           WS(r, j, JNDS) * one_nds;
    }
    for (int idelta = 1; idelta <= r->ndelta; idelta++) {
      int j = (r->jlast + r->idir * (idelta - 1) + nb) % nb;
      int jn = (r->jlast + r->idir * idelta + nb) % nb;
      wn = wn + WS(r, j, JBRA) - WS(r, j, JDTP) * (one + half - mezzo) +
           WS(r, jn, JITP) * (half - mezzo) + WS(r, j, JLNG) * one -
           WS(r, j, JNDS) * one_nds;
    }
  } else {
    for (int idelta = 1; idelta <= r->ndelta; idelta++) {
      int j = (r->jlast + r->idir * (idelta - 1) + nb) % nb;
      int jn = (r->jlast + r->idir * idelta + nb) % nb;
      wn = wn - WS(r, jn, JBRA) + WS(r, jn, JDTP) * (one + half - mezzo) -
           WS(r, j, JITP) * (half - mezzo) - WS(r, jn, JLNG) * one +
           WS(r, jn, JNDS) * one_nds;
    }
    for (int idelta = 1; idelta <= r->ndelta; idelta++) {
      int j = (r->jfirst + r->idir * (idelta - 1) + nb) % nb;
      int jn = (r->jfirst + r->idir * idelta + nb) % nb;
      wn = wn + WS(r, jn, JBRA) + WS(r, jn, JDTP) * (half + mezzo) -
           WS(r, j, JITP) * (one + half + mezzo) + WS(r, jn, JLNG) * one -
           WS(r, jn, JNDS) * one_nds;
    }
  }
  return wn;
}

int oracle_reptile_run(const qmc2d_system *sys, oracle_reptile *r, int rid, uint64_t seed,
                       long step0, int nstp, double *blk, long *naccept) {
  (void)sys;
  long nacc = 0;
  for (int istp = 0; istp < nstp; istp++) {
    uint32_t t = (uint32_t)(step0 + istp);
    int st;
    double wnew = reptation_move(r, rid, seed, t, &st);
    if (st) return st;
    /* reptation_metropolis_test (reptation.f:1865-1895) */
    double p;
    if (r->age == r->prm.mage_r) {
      p = 1.0;
    } else {
      p = wnew < -50.0 ? -50.0 : wnew;
      p = p > 0.0 ? 0.0 : p;
      p = exp(p);
    }
    double ua = u1(seed, 0xFFFFFFFDu, (uint32_t)rid, t, 2u, 0);
    if (p >= ua) {
      r->jfirst = r->kfirst;
      r->jlast = r->klast;
      memcpy(r->pp_old, r->pp_new, sizeof(double) * r->npr);
      r->age = 0.0;
      nacc++;
    } else {
      r->age = r->age + 1;
      r->ndelta = 0;
    }
    if (blk)
      for (int i = 0; i < r->npr; i++) blk[i] = blk[i] + r->pp_old[i];
  }
  if (naccept) *naccept += nacc;
  return 0;
}

void oracle_reptile_path(const oracle_reptile *r, double *x, double *p) {
  for (int i = 0; i < r->prm.ntau; i++) {
    int j = (r->jfirst + i) % r->nbuf;
    if (x) memcpy(x + (size_t)2 * r->N * i, XS(r, j), sizeof(double) * 2 * r->N);
    if (p) memcpy(p + (size_t)r->npr * i, PS(r, j), sizeof(double) * r->npr);
  }
}
