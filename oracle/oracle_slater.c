/*
 * oracle_slater.c - CPU oracle (TEST INFRASTRUCTURE ONLY): the backflow
 * Slater determinant of complex plane waves and the LINPACK complex LU it
 * relies on, restated from reptation.f.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* izamax (reptation.f:9079-9118), unit stride. Returns a 0-based offset. */
static int izamax(int n, const zc *zx) {
  if (n < 1) return -1;
  int imax = 0;
  if (n == 1) return 0;
  double smax = cabs1(zx[0]);
  for (int i = 1; i < n; i++) {
    if (cabs1(zx[i]) <= smax) continue;
    imax = i;
    smax = cabs1(zx[i]);
  }
  return imax;
}

/* zscal (reptation.f:9190-9217), unit stride. */
static void zscal(int n, zc za, zc *zx) {
  for (int i = 0; i < n; i++) zx[i] = zmul(za, zx[i]);
}

/* zaxpy (reptation.f:9156-9188), unit stride. */
static void zaxpy(int n, zc za, const zc *zx, zc *zy) {
  if (n <= 0) return;
  if (cabs1(za) == 0.0) return;
  for (int i = 0; i < n; i++) zy[i] = zadd(zy[i], zmul(za, zx[i]));
}

/* zswap (reptation.f:9120-9154), unit stride. */
static void zswap(int n, zc *zx, zc *zy) {
  for (int i = 0; i < n; i++) {
    zc t = zx[i];
    zx[i] = zy[i];
    zy[i] = t;
  }
}

/* zgefa (reptation.f:9227-9337): LU with partial pivoting, column-major
 * a(lda, n). ipvt 0-based. Returns info (0, or 1-based zero-pivot column). */
static int zgefa(zc *a, int lda, int n, int *ipvt) {
#define A(i, j) a[(size_t)(j) * lda + (i)]
  int info = 0;
  int nm1 = n - 1;
  for (int k = 0; k < nm1; k++) {
    int kp1 = k + 1;
    int l = izamax(n - k, &A(k, k)) + k;
    ipvt[k] = l;
    if (cabs1(A(l, k)) == 0.0) {
      info = k + 1;
      continue;
    }
    if (l != k) {
      zc t = A(l, k);
      A(l, k) = A(k, k);
      A(k, k) = t;
    }
    zc one = {1.0, 0.0};
    zc t = zdiv(one, A(k, k));
    t.re = -t.re;
    t.im = -t.im;
    zscal(n - kp1, t, &A(kp1, k));
    for (int j = kp1; j < n; j++) {
      t = A(l, j);
      if (l != k) {
        A(l, j) = A(k, j);
        A(k, j) = t;
      }
      zaxpy(n - kp1, t, &A(kp1, k), &A(kp1, j));
    }
  }
  ipvt[n - 1] = n - 1;
  if (cabs1(A(n - 1, n - 1)) == 0.0) info = n;
  return info;
#undef A
}

/* zgedi (reptation.f:9338-9470) with job = 11: determinant as
 * det[0] * 10**det[1] and the inverse in place. */
static void zgedi(zc *a, int lda, int n, const int *ipvt, zc det[2], zc *work) {
#define A(i, j) a[(size_t)(j) * lda + (i)]
  const double ten = 10.0;
  det[0].re = 1.0;
  det[0].im = 0.0;
  det[1].re = 0.0;
  det[1].im = 0.0;
  for (int i = 0; i < n; i++) {
    if (ipvt[i] != i) {
      det[0].re = -det[0].re;
      det[0].im = -det[0].im;
    }
    det[0] = zmul(A(i, i), det[0]);
    if (cabs1(det[0]) == 0.0) break;
    while (cabs1(det[0]) < 1.0) {
      zc tt = {ten, 0.0};
      det[0] = zmul(tt, det[0]);
      det[1].re = det[1].re - 1.0;
    }
    while (cabs1(det[0]) >= ten) {
      zc tt = {ten, 0.0};
      det[0] = zdiv(det[0], tt);
      det[1].re = det[1].re + 1.0;
    }
  }
  /* inverse(u) */
  for (int k = 0; k < n; k++) {
    zc one = {1.0, 0.0};
    A(k, k) = zdiv(one, A(k, k));
    zc t = {-A(k, k).re, -A(k, k).im};
    zscal(k, t, &A(0, k));
    for (int j = k + 1; j < n; j++) {
      t = A(k, j);
      A(k, j).re = 0.0;
      A(k, j).im = 0.0;
      zaxpy(k + 1, t, &A(0, k), &A(0, j));
    }
  }
  /* inverse(u) * inverse(l) */
  for (int kb = 1; kb <= n - 1; kb++) {
    int k = n - 1 - kb;
    for (int i = k + 1; i < n; i++) {
      work[i] = A(i, k);
      A(i, k).re = 0.0;
      A(i, k).im = 0.0;
    }
    for (int j = k + 1; j < n; j++) {
      zc t = work[j];
      zaxpy(n, t, &A(0, j), &A(0, k));
    }
    int l = ipvt[k];
    if (l != k) zswap(n, &A(0, k), &A(0, l));
  }
#undef A
}

/* paho_orbitals with iex = 1 and no excitation (reptation.f:10268-10320):
 * zorb(jk,i) = exp(i g_jk . q_i) for orbital jk and particle i of type jt,
 * its derivatives, then LU and inverse. zorb is left holding the inverse. */
static int paho_orbitals(const qmc2d_system *sys, oracle_work *w, int jt, zc zdet[2]) {
  int nm = w->nmax;
  int n = sys->np[jt];
  int f0 = sys->ipfrst[jt];
  for (int jk = 0; jk < n; jk++) {
    const double *gv = sys->gvec + 2 * jk;
    for (int jp = f0; jp < f0 + n; jp++) {
      double kr = 0.0;
      for (int d = 0; d < 2; d++) kr = kr + QX(d, jp) * gv[d];
      int i = jp - f0;
      ZORB(jk, i).re = cos(kr);
      ZORB(jk, i).im = sin(kr);
      for (int d = 0; d < 2; d++) {
        zc ig = {0.0, gv[d]};
        DZORB(d, jk, i) = zmul(ig, ZORB(jk, i));
      }
      for (int id = 0; id < 2; id++)
        for (int jd = 0; jd < 2; jd++) {
          zc mg = {-(gv[id] * gv[jd]), -0.0};
          DDZORB(jd, id, jk, i) = zmul(mg, ZORB(jk, i));
        }
    }
  }
  int info = zgefa(w->zorb, nm, n, w->ipvt);
  if (info != 0) return QMC2D_ERR_SINGULAR;
  zgedi(w->zorb, nm, n, w->ipvt, zdet, w->zwork);
  return 0;
}

/* slater_excitations (reptation.f:9967-10266): symmetric backflow
 * q_i = r_i + sum_j eta(r_ij) r_ij, determinant per type, drift and
 * Laplacian through the backflow Jacobian qa and its divergence qb. */
int oracle_slater(const qmc2d_system *sys, oracle_work *w, const double *x, double *ltf,
                  double *g_new, double *h_new, int *underflow) {
  int N = w->N;
  int nm = w->nmax;
  size_t nn = (size_t)nm * nm;
  int any = 0;
  for (int it = 0; it < sys->ntypes; it++)
    for (int jt = it; jt < sys->ntypes; jt++) any |= (sys->iub[it][jt] >= 0);
  *underflow = 0;
  if (!any) return 0;
  /* initialize (reptation.f:10009-10020) */
  for (int ip = 0; ip < sys->nptot; ip++) {
    for (int jp = 0; jp < sys->nptot; jp++)
      for (int id = 0; id < 2; id++) {
        QB(id, jp, ip) = 0.0;
        for (int jd = 0; jd < 2; jd++) QA(jd, id, jp, ip) = 0.0;
      }
    for (int id = 0; id < 2; id++) {
      QX(id, ip) = x[2 * ip + id];
      QA(id, id, ip, ip) = 1.0;
    }
  }
  /* quasi-coordinates (reptation.f:10021-10057) */
  double t, dt, ddt;
  int ij = 0;
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    int i = sys->iub[it][it];
    if (i >= 0) {
      for (int ip = f0; ip < l0; ip++)
        for (int jp = ip + 1; jp < l0; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          for (int d = 0; d < 2; d++) {
            double wk = t * PRV(d, ij);
            QX(d, ip) = QX(d, ip) + wk;
            QX(d, jp) = QX(d, jp) - wk;
          }
          ij++;
        }
    }
    for (int jt = it + 1; jt < sys->ntypes; jt++) {
      i = sys->iub[it][jt];
      if (i < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = f1; jp < l1; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          for (int d = 0; d < 2; d++) {
            double wk = t * PRV(d, ij);
            QX(d, ip) = QX(d, ip) + wk;
            QX(d, jp) = QX(d, jp) - wk;
          }
          ij++;
        }
    }
  }
  /* determinants (reptation.f:10058-10086) */
  for (int jt = 0; jt < sys->ntypes; jt++) {
    zc zdet[2];
    int st = paho_orbitals(sys, w, jt, zdet);
    if (st) return st;
    /* -Re(log(det1) + det2*log(10)) */
    double lg = log(sqrt(zdet[0].re * zdet[0].re + zdet[0].im * zdet[0].im));
    *ltf = *ltf - (lg + zdet[1].re * log(10.0));
    memcpy(w->sorb + nn * jt, w->zorb, sizeof(zc) * nn);
    memcpy(w->dsorb + 2 * nn * jt, w->dzorb, sizeof(zc) * 2 * nn);
    memcpy(w->ddsorb + 4 * nn * jt, w->ddzorb, sizeof(zc) * 4 * nn);
  }
  double wgt = exp(-*ltf * 2);
  if (sys->ref_underflow_return && wgt <= 0.0) {
    *underflow = 1;
    w->grad2_ph = 0.0;
    return 0;
  }
  /* qa, qb (reptation.f:10093-10168) */
  ij = 0;
  for (int it = 0; it < sys->ntypes; it++) {
    int f0 = sys->ipfrst[it], l0 = f0 + sys->np[it];
    for (int jt = it; jt < sys->ntypes; jt++) {
      int i = sys->iub[it][jt];
      if (i < 0) continue;
      int f1 = sys->ipfrst[jt], l1 = f1 + sys->np[jt];
      for (int ip = f0; ip < l0; ip++)
        for (int jp = (jt == it ? ip + 1 : f1); jp < l1; jp++) {
          getf(sys, i, w->pp_ind[ij], w->pp_rem[ij], &t, &dt, &ddt);
          double byr = w->pp_byr[ij];
          for (int id = 0; id < 2; id++) {
            double w2 = (dt * byr * (2 + 1) + ddt) * PRV(id, ij);
            QB(id, ip, ip) = QB(id, ip, ip) + w2;
            QB(id, jp, jp) = QB(id, jp, jp) - w2;
            QB(id, jp, ip) = QB(id, jp, ip) + w2;
            QB(id, ip, jp) = QB(id, ip, jp) - w2;
            QA(id, id, ip, ip) = QA(id, id, ip, ip) + t;
            QA(id, id, jp, jp) = QA(id, id, jp, jp) + t;
            QA(id, id, jp, ip) = QA(id, id, jp, ip) - t;
            QA(id, id, ip, jp) = QA(id, id, ip, jp) - t;
            for (int jd = 0; jd < 2; jd++) {
              double w3 = dt * byr * PRV(jd, ij) * PRV(id, ij);
              QA(jd, id, ip, ip) = QA(jd, id, ip, ip) + w3;
              QA(jd, id, jp, jp) = QA(jd, id, jp, jp) + w3;
              QA(jd, id, jp, ip) = QA(jd, id, jp, ip) - w3;
              QA(jd, id, ip, jp) = QA(jd, id, ip, jp) - w3;
            }
          }
          ij++;
        }
    }
  }
  /* drift and Laplacian per determinant (reptation.f:10169-10265) */
  double aux = 0.0;
  for (int jt = 0; jt < sys->ntypes; jt++) {
    int n = sys->np[jt];
    int fj = sys->ipfrst[jt], lj = fj + n;
    memcpy(w->zorb, w->sorb + nn * jt, sizeof(zc) * nn);
    memcpy(w->dzorb, w->dsorb + 2 * nn * jt, sizeof(zc) * 2 * nn);
    memcpy(w->ddzorb, w->ddsorb + 4 * nn * jt, sizeof(zc) * 4 * nn);
    /* zv(id,lf,jf) = sum_kf Ainv(lf,kf) dA(id,kf,jf)  (F of Kwon et al.) */
    for (int jf = 0; jf < n; jf++)
      for (int lf = 0; lf < n; lf++) {
        for (int id = 0; id < 2; id++) {
          ZV(id, lf, jf).re = 0.0;
          ZV(id, lf, jf).im = 0.0;
        }
        for (int id = 0; id < 2; id++)
          for (int kf = 0; kf < n; kf++)
            ZV(id, lf, jf) = zadd(ZV(id, lf, jf), zmul(ZORB(lf, kf), DZORB(id, kf, jf)));
      }
    w->grad2_ph = 0.0;
    for (int it = 0; it < sys->ntypes; it++) {
      int lo = it < jt ? it : jt, hi = it < jt ? jt : it;
      if (sys->iub[lo][hi] < 0) continue;
      int fi = sys->ipfrst[it], li = fi + sys->np[it];
      double aux2 = 0.0;
      for (int ip = fi; ip < li; ip++)
        for (int id = 0; id < 2; id++) {
          zc z1 = {0.0, 0.0};
          for (int jp = fj; jp < lj; jp++) {
            int jf = jp - fj;
            for (int jd = 0; jd < 2; jd++) {
              double q = QA(jd, id, jp, ip);
              z1.re = z1.re + ZV(jd, jf, jf).re * q;
              z1.im = z1.im + ZV(jd, jf, jf).im * q;
            }
          }
          g_new[2 * ip + id] = g_new[2 * ip + id] - z1.re;
          w->grad2_ph = w->grad2_ph + z1.im * z1.im;
          aux2 = aux2 + z1.im * z1.im;
        }
      for (int ip = fi; ip < li; ip++)
        for (int jp = fj; jp < lj; jp++) {
          int jf = jp - fj;
          for (int jd = 0; jd < 2; jd++)
            h_new[it] = h_new[it] - ZV(jd, jf, jf).re * QB(jd, ip, jp);
        }
      for (int ip = fi; ip < li; ip++)
        for (int jp = fj; jp < lj; jp++) {
          int jf = jp - fj;
          for (int id = 0; id < 2; id++)
            for (int jd = 0; jd < 2; jd++) {
              zc z1 = {0.0, 0.0};
              for (int kf = 0; kf < n; kf++)
                z1 = zadd(z1, zmul(ZORB(jf, kf), DDZORB(jd, id, kf, jf)));
              double z2 = 0.0;
              for (int kd = 0; kd < 2; kd++)
                z2 = z2 + QA(kd, jd, jp, ip) * QA(kd, id, jp, ip);
              h_new[it] = h_new[it] - z1.re * z2;
            }
        }
      for (int ip = fi; ip < li; ip++)
        for (int jp = fj; jp < lj; jp++) {
          int jf = jp - fj;
          for (int kp = fj; kp < lj; kp++) {
            int kf = kp - fj;
            for (int id = 0; id < 2; id++) {
              zc z1 = {0.0, 0.0}, z2 = {0.0, 0.0};
              for (int jd = 0; jd < 2; jd++) {
                double q = QA(jd, id, jp, ip);
                z1.re = z1.re + q * ZV(jd, kf, jf).re;
                z1.im = z1.im + q * ZV(jd, kf, jf).im;
              }
              for (int jd = 0; jd < 2; jd++) {
                double q = QA(jd, id, kp, ip);
                z2.re = z2.re + q * ZV(jd, jf, kf).re;
                z2.im = z2.im + q * ZV(jd, jf, kf).im;
              }
              h_new[it] = h_new[it] + zmul(z1, z2).re;
            }
          }
        }
      aux = aux + aux2 * sys->hbs2m[it];
    }
  }
  w->grad2_ph = aux;
  return 0;
}
