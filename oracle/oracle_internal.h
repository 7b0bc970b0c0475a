/*
 * oracle_internal.h - shared internals of the CPU oracle (TEST
 * INFRASTRUCTURE ONLY): scratch layout standing in for the reference's
 * /c_dist/ and /scratch/ COMMON blocks (ewald.h), complex helpers and the
 * spline evaluators.
 */
#ifndef QMC2D_ORACLE_INTERNAL_H
#define QMC2D_ORACLE_INTERNAL_H

#include <math.h>
#include <stddef.h>

#include "qmc2d_oracle.h"

typedef struct { double re, im; } zc;

static inline zc zmul(zc a, zc b) {
  zc r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline zc zadd(zc a, zc b) {
  zc r = {a.re + b.re, a.im + b.im};
  return r;
}
/* Complex division a/b, componentwise formula. */
static inline zc zdiv(zc a, zc b) {
  double d = b.re * b.re + b.im * b.im;
  zc r = {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
  return r;
}
/* dcabs1 (reptation.f:9219-9226) */
static inline double cabs1(zc z) { return fabs(z.re) + fabs(z.im); }

struct oracle_work {
  int N, P, nk, nmax;
  /* /c_dist/ pair arrays (ewald.h) */
  double *pp_r, *pp_byr, *pp_rvec, *pp_rem;
  int *pp_ind;
  int pp_dist[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES];
  double *rhok; /* rhok(2*nk, slot) */
  /* three_body scratch: g(2,N), dg(2,2,N,N), ddg(2,N,N) */
  double *g3, *dg, *ddg;
  /* slater scratch */
  double *qx, *qa, *qb;
  zc *zorb, *dzorb, *ddzorb; /* zorb(n,n), dzorb(2,n,n), ddzorb(2,2,n,n) */
  zc *sorb, *dsorb, *ddsorb; /* saved per type */
  zc *zv, *zwork;
  int *ipvt;
  double grad2_ph;
};

/* Column-major addressing with the reference's index order. */
#define PRV(d, ij) (w->pp_rvec[2 * (ij) + (d)])
#define DG(jd, id, jp, ip) (w->dg[(((size_t)(ip) * N + (jp)) * 2 + (id)) * 2 + (jd)])
#define DDG(id, jp, ip) (w->ddg[((size_t)(ip) * N + (jp)) * 2 + (id)])
#define G3(id, ip) (w->g3[2 * (ip) + (id)])
#define QA(jd, id, jp, ip) (w->qa[(((size_t)(ip) * N + (jp)) * 2 + (id)) * 2 + (jd)])
#define QB(id, jp, ip) (w->qb[((size_t)(ip) * N + (jp)) * 2 + (id)])
#define QX(id, ip) (w->qx[2 * (ip) + (id)])
#define ZORB(a, b) (w->zorb[(size_t)(b) * nm + (a)])
#define DZORB(id, a, b) (w->dzorb[((size_t)(b) * nm + (a)) * 2 + (id)])
#define DDZORB(jd, id, a, b) (w->ddzorb[(((size_t)(b) * nm + (a)) * 2 + (id)) * 2 + (jd)])
#define ZV(id, a, b) (w->zv[((size_t)(b) * nm + (a)) * 2 + (id)])

/* getf (reptation.f:4114-4126): f, f', f'' of the cubic at knot ind. */
static inline void getf(const qmc2d_system *sys, int itab, int ind, double rem, double *f,
                        double *df, double *ddf) {
  const qmc2d_table *t = &sys->tables[itab];
  int i = ind < t->ngrid ? ind : t->ngrid;
  double rm = rem * sys->drti;
  const double *u = t->ut + 4 * i;
  *f = u[0] + rm * (u[1] + rm * (u[2] + rm * u[3]));
  *df = (u[1] + rm * (2 * u[2] + rm * (3 * u[3]))) * sys->drti;
  *ddf = (u[2] + rm * (3 * u[3])) * sys->drti2;
}

/* getf_0 (reptation.f:4103-4112): f times (1/r)**iexp. */
static inline double getf_0(const qmc2d_system *sys, int itab, int ind, double rem,
                            double byr) {
  const qmc2d_table *t = &sys->tables[itab];
  int i = ind < t->ngrid ? ind : t->ngrid;
  double rm = rem * sys->drti;
  const double *u = t->ut + 4 * i;
  double f = u[0] + rm * (u[1] + rm * (u[2] + rm * u[3]));
  double p = 1.0;
  for (int k = 0; k < t->iexp; k++) p *= byr;
  return f * p;
}

/* Fortran nint: nearest integer, halves away from zero. */
static inline double fnint(double x) { return round(x); }

/* Wavefunction pieces, in evaluation order (trial_function, reptation.f:3048). */
void oracle_distances(const qmc2d_system *sys, oracle_work *w, const double *x);
void oracle_two_body(const qmc2d_system *sys, oracle_work *w, double *ltf, double *g_new,
                     double *h_new);
void oracle_three_body(const qmc2d_system *sys, oracle_work *w, double *ltf, double *g_new,
                       double *h_new);
/* slater_excitations; returns 0 or QMC2D_ERR_SINGULAR, sets *underflow. */
int oracle_slater(const qmc2d_system *sys, oracle_work *w, const double *x, double *ltf,
                  double *g_new, double *h_new, int *underflow);

#endif
