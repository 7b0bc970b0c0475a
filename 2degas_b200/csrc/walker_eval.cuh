// walker_eval.cuh - FP64 evaluation of one walker by one CTA: the
// reference's compute_properties (reptation.f:2661) = distances :4127,
// two_body :2981, three_body :2777, slater_excitations :9967, kinetic :2729,
// potential :3986, restated for a 256-thread CTA with every intermediate in
// shared memory.
//
// Layout and parallel decomposition
//   * pair sums: 8 threads per particle i sweep j != i (each unordered pair
//     is visited from both ends, so per-particle sums need no atomics); the
//     8 partial sums meet by warp shuffles in a fixed order.
//   * u3 (l=1 factorised triplets): with G_i = -sum_j xi(r_ij) r_ij and
//     M_ij = xi I + (xi'/r) r r^T, the gradient of -1/2 sum|G|^2 on k is
//     sum_j M_kj (G_k - G_j) and its Laplacian is
//     sum_j (xi'' + 3 xi'/r) r_kj.(G_k - G_j) - tr(S_k^2) - sum_j tr(M_kj^2),
//     S_k = sum_j M_kj: the dense dg/ddg of makeg/dotg are never formed.
//   * determinant per spin: A(k,j) = exp(i g_k.q_j) in shared memory,
//     Gauss-Jordan inversion with partial pivoting (log|det| from the
//     pivots), F_a = A^-1 diag(i g_a) A, and the backflow cross term
//     sum_{j,k} Re[(J_j.F(k,j))(J_k.F(j,k))] as the quadratic form of the
//     symmetric 2n x 2n matrix M_ac(j,k) = Re[F_a(k,j) F_c(j,k)] against the
//     Jacobian columns of every electron.
#pragma once

#include <cuda_runtime.h>

#include "devsys.h"

namespace q2d {

struct EvalSmem {
  double *x, *g, *q, *G3, *S3, *Sb, *qbd, *lap, *ltf, *vp, *ph2;
  double *gd, *lapd, *ph2d;  // determinant contributions (added unless underflow)
  double *rhok;              // 2*nk per rhok slot
  double2 *A, *Ai, *F0, *F1;
  double *D2, *U, *red, *colk;
  int *perm, *iscal;
  double *dscal;
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// Carve the dynamic shared memory; returns bytes used.
__host__ __device__ inline size_t eval_carve(const DevSys &s, char *base, EvalSmem *m) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base ? base + off : nullptr;
    off += align16(bytes);
    return p;
  };
  int N = s.N, n = s.nmax > 0 ? s.nmax : 1;
  EvalSmem t;
  t.x = (double *)take(sizeof(double) * 2 * N);
  t.g = (double *)take(sizeof(double) * 2 * N);
  t.q = (double *)take(sizeof(double) * 2 * N);
  t.G3 = (double *)take(sizeof(double) * 2 * N);
  t.S3 = (double *)take(sizeof(double) * 3 * N);
  t.Sb = (double *)take(sizeof(double) * 3 * N);
  t.qbd = (double *)take(sizeof(double) * 2 * N);
  t.lap = (double *)take(sizeof(double) * N);
  t.ltf = (double *)take(sizeof(double) * N);
  t.vp = (double *)take(sizeof(double) * N);
  t.ph2 = (double *)take(sizeof(double) * N);
  t.gd = (double *)take(sizeof(double) * 2 * N);
  t.lapd = (double *)take(sizeof(double) * N);
  t.ph2d = (double *)take(sizeof(double) * N);
  t.rhok = (double *)take(sizeof(double) * 2 * (s.nk > 0 ? s.nk : 1) * 2);
  // A and Ai are contiguous so the 2n x 2n real matrix of the cross term can
  // overlay them once F0/F1 are formed.
  t.A = (double2 *)take(sizeof(double2) * 2 * n * n);
  t.Ai = t.A ? t.A + n * n : nullptr;
  t.F0 = (double2 *)take(sizeof(double2) * n * n);
  t.F1 = (double2 *)take(sizeof(double2) * n * n);
  t.D2 = (double *)take(sizeof(double) * 3 * n);
  t.U = (double *)take(sizeof(double) * 2 * n * kChunk);
  t.red = (double *)take(sizeof(double) * kThreads);
  t.colk = (double *)take(sizeof(double2) * n);
  t.perm = (int *)take(sizeof(int) * n);
  t.iscal = (int *)take(sizeof(int) * 8);
  t.dscal = (double *)take(sizeof(double) * 16);
  if (m) *m = t;
  return off;
}

// ----------------------------------------------------------------- helpers

__device__ __forceinline__ int type_of(const DevSys &S, int i) {
  return (S.nt > 1 && i >= S.ipfrst[1]) ? 1 : 0;
}

// getf (reptation.f:4114): cubic at knot min(ngrid, ind), f, f', f''.
__device__ __forceinline__ void spline3(const DevSys &S, int t, int ind, double rem, double &f,
                                        double &df, double &ddf) {
  int i = max(0, min(S.tab_ngrid[t], ind));  // NaN/negative -> knot 0
  const double2 *u = reinterpret_cast<const double2 *>(S.coef + S.tab_off[t] + 4 * i);
  double2 a = __ldg(u), b = __ldg(u + 1);
  double rm = rem * S.drti;
  f = a.x + rm * (a.y + rm * (b.x + rm * b.y));
  df = (a.y + rm * (2.0 * b.x + rm * (3.0 * b.y))) * S.drti;
  ddf = (b.x + rm * (3.0 * b.y)) * S.drti2;
}

// getf_0 (reptation.f:4103): f * (1/r)**iexp.
__device__ __forceinline__ double spline0(const DevSys &S, int t, int ind, double rem,
                                          double byr) {
  int i = max(0, min(S.tab_ngrid[t], ind));  // NaN/negative -> knot 0
  const double2 *u = reinterpret_cast<const double2 *>(S.coef + S.tab_off[t] + 4 * i);
  double2 a = __ldg(u), b = __ldg(u + 1);
  double rm = rem * S.drti;
  double f = a.x + rm * (a.y + rm * (b.x + rm * b.y));
  for (int k = 0; k < S.tab_iexp[t]; k++) f *= byr;
  return f;
}

// Minimum-image pair geometry (distances, reptation.f:4136-4160).
__device__ __forceinline__ void pair_geom(const DevSys &S, const double *x, int i, int j,
                                          double &rx, double &ry, double &r, double &byr,
                                          int &ind, double &rem) {
  rx = x[2 * i] - x[2 * j];
  ry = x[2 * i + 1] - x[2 * j + 1];
  rx = rx - S.el[0] * round(S.eli[0] * rx);
  ry = ry - S.el[1] * round(S.eli[1] * ry);
  r = sqrt(rx * rx + ry * ry);
  ind = (int)(r * S.drti);
  rem = r - ind * S.drt;
  byr = 1.0 / r;
}

// Sum within aligned groups of 8 lanes; every lane of the warp must call it.
__device__ __forceinline__ double group8_sum(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  return v;
}

// Deterministic block sum; result valid in every thread. Uses red[0..8].
__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
  __syncthreads();
  return t;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// ---------------------------------------------------------- the evaluation
//
// Input: m.x holds the configuration. Output (in shared memory): m.g (drift
// -grad ln psi), hl[nt] (-lap ln psi per type), props[nprops], *sign.
// Returns a status word (ST_*), identical in all threads.
__device__ inline int eval_walker(const DevSys &S, const EvalSmem &m, double *hl, double *props,
                                  double *sign) {
  const int tid = threadIdx.x;
  const int N = S.N, nt = S.nt;
  const int lane8 = tid & (kGroup - 1);
  const int per_round = kThreads / kGroup;

  // ---- pass A: pair sums of u2, the pair part of u3, u3 G vectors and S,
  // backflow displacement, Jacobian diagonal and Laplacian, pair potential.
  for (int base = 0; base < N; base += per_round) {
    int i = base + tid / kGroup;
    bool valid = i < N;
    int ti = valid ? type_of(S, i) : 0;
    double ltf = 0, gx = 0, gy = 0, lap = 0, vp = 0;
    double Gx = 0, Gy = 0, s3xx = 0, s3xy = 0, s3yy = 0;
    double qx = 0, qy = 0, sbxx = 0, sbxy = 0, sbyy = 0, qbx = 0, qby = 0;
    if (valid) {
      for (int j = lane8; j < N; j += kGroup) {
        if (j == i) continue;
        int tj = type_of(S, j);
        double rx, ry, r, byr, rem;
        int ind;
        pair_geom(S, m.x, i, j, rx, ry, r, byr, ind, rem);
        double t, dt, ddt;
        if (S.has_u2) {
          spline3(S, S.iu2[ti][tj], ind, rem, t, dt, ddt);
          ltf += 0.5 * t;
          double dtr = dt * byr;
          gx += dtr * rx;
          gy += dtr * ry;
          lap += ddt + dtr;
        }
        if (S.has_u3) {
          spline3(S, S.iu3[ti][tj], ind, rem, t, dt, ddt);
          Gx -= t * rx;
          Gy -= t * ry;
          double c = dt * byr;
          s3xx += t + c * rx * rx;
          s3xy += c * rx * ry;
          s3yy += t + c * ry * ry;
          // the two-body piece (xi r)^2 removed from sum |G|^2 (three_body :2824-2832)
          double d3 = 2.0 * (t * t + 4.0 * r * t * dt + r * r * (dt * dt + ddt * t));
          double c3 = 2.0 * t * (t + r * dt);
          double tr = t * r;
          ltf += 0.5 * tr * tr;
          gx += c3 * rx;
          gy += c3 * ry;
          lap += d3 + c3;
        }
        if (S.has_bf) {
          spline3(S, S.iub[ti][tj], ind, rem, t, dt, ddt);
          qx += t * rx;
          qy += t * ry;
          double c = dt * byr;
          sbxx += t + c * rx * rx;
          sbxy += c * rx * ry;
          sbyy += t + c * ry * ry;
          double w2 = dt * byr * 3.0 + ddt;
          qbx += w2 * rx;
          qby += w2 * ry;
        }
        if (S.has_v2) vp += 0.5 * spline0(S, S.iv2[ti][tj], ind, rem, byr);
      }
    }
    ltf = group8_sum(ltf);
    gx = group8_sum(gx);
    gy = group8_sum(gy);
    lap = group8_sum(lap);
    vp = group8_sum(vp);
    if (S.has_u3) {
      Gx = group8_sum(Gx);
      Gy = group8_sum(Gy);
      s3xx = group8_sum(s3xx);
      s3xy = group8_sum(s3xy);
      s3yy = group8_sum(s3yy);
    }
    if (S.has_bf) {
      qx = group8_sum(qx);
      qy = group8_sum(qy);
      sbxx = group8_sum(sbxx);
      sbxy = group8_sum(sbxy);
      sbyy = group8_sum(sbyy);
      qbx = group8_sum(qbx);
      qby = group8_sum(qby);
    }
    if (valid && lane8 == 0) {
      m.ltf[i] = ltf;
      m.g[2 * i] = gx;
      m.g[2 * i + 1] = gy;
      m.lap[i] = lap;
      m.vp[i] = vp;
      m.G3[2 * i] = Gx;
      m.G3[2 * i + 1] = Gy;
      m.S3[3 * i] = s3xx;
      m.S3[3 * i + 1] = s3xy;
      m.S3[3 * i + 2] = s3yy;
      m.q[2 * i] = m.x[2 * i] + qx;
      m.q[2 * i + 1] = m.x[2 * i + 1] + qy;
      m.Sb[3 * i] = sbxx;
      m.Sb[3 * i + 1] = sbxy;
      m.Sb[3 * i + 2] = sbyy;
      m.qbd[2 * i] = qbx;
      m.qbd[2 * i + 1] = qby;
      m.gd[2 * i] = 0.0;
      m.gd[2 * i + 1] = 0.0;
      m.lapd[i] = 0.0;
      m.ph2[i] = 0.0;
      m.ph2d[i] = 0.0;
    }
  }
  // ---- rho_k per rhok slot (distances, reptation.f:4225-4243)
  for (int e = tid; e < nt * S.nk; e += kThreads) {
    int t = e / S.nk, k = e - t * S.nk;
    if (S.irhok[t] == 0) continue;
    double kx = __ldg(S.kvec + 2 * k), ky = __ldg(S.kvec + 2 * k + 1);
    double c = 0.0, sn = 0.0;
    for (int i = S.ipfrst[t]; i < S.ipfrst[t] + S.np[t]; i++) {
      double kr = kx * m.x[2 * i] + ky * m.x[2 * i + 1];
      double sv, cv;
      sincos(kr, &sv, &cv);
      c += cv;
      sn += sv;
    }
    int slot = S.irhok[t] - 1;
    m.rhok[2 * (slot * S.nk + k)] = c;
    m.rhok[2 * (slot * S.nk + k) + 1] = sn;
  }
  __syncthreads();

  // ---- pass B: u3 gradient and Laplacian from the G vectors.
  if (S.has_u3) {
    for (int base = 0; base < N; base += per_round) {
      int k = base + tid / kGroup;
      bool valid = k < N;
      int tk = valid ? type_of(S, k) : 0;
      double gx = 0, gy = 0, lap = 0;
      double Gkx = valid ? m.G3[2 * k] : 0.0, Gky = valid ? m.G3[2 * k + 1] : 0.0;
      if (valid) {
        for (int j = lane8; j < N; j += kGroup) {
          if (j == k) continue;
          int tj = type_of(S, j);
          double rx, ry, r, byr, rem;
          int ind;
          pair_geom(S, m.x, k, j, rx, ry, r, byr, ind, rem);
          double t, dt, ddt;
          spline3(S, S.iu3[tk][tj], ind, rem, t, dt, ddt);
          double c = dt * byr;
          double mxx = t + c * rx * rx, mxy = c * rx * ry, myy = t + c * ry * ry;
          double dGx = Gkx - m.G3[2 * j], dGy = Gky - m.G3[2 * j + 1];
          gx += mxx * dGx + mxy * dGy;
          gy += mxy * dGx + myy * dGy;
          double w = ddt + 3.0 * c;
          lap += w * (rx * dGx + ry * dGy) - (mxx * mxx + 2.0 * mxy * mxy + myy * myy);
        }
      }
      gx = group8_sum(gx);
      gy = group8_sum(gy);
      lap = group8_sum(lap);
      if (valid && lane8 == 0) {
        double sxx = m.S3[3 * k], sxy = m.S3[3 * k + 1], syy = m.S3[3 * k + 2];
        m.g[2 * k] += gx;
        m.g[2 * k + 1] += gy;
        m.lap[k] += lap - (sxx * sxx + 2.0 * sxy * sxy + syy * syy);
        m.ltf[k] -= 0.5 * (Gkx * Gkx + Gky * Gky);
      }
    }
  }
  __syncthreads();

  // ---- backflow Slater determinants (slater_excitations, reptation.f:9967)
  int status = ST_OK;
  double logdet_sum = 0.0;
  if (S.has_bf) {
    for (int sp = 0; sp < nt; sp++) {
      const int n = S.np[sp], f0 = S.ipfrst[sp], nn = n * n;
      // orbitals (paho_orbitals, reptation.f:10298-10315): A(k,j), column-major
      for (int e = tid; e < nn; e += kThreads) {
        int k = e % n, j = e / n;
        double gkx = __ldg(S.gvec + 2 * k), gky = __ldg(S.gvec + 2 * k + 1);
        double kr = m.q[2 * (f0 + j)] * gkx + m.q[2 * (f0 + j) + 1] * gky;
        double sv, cv;
        sincos(kr, &sv, &cv);
        m.A[e] = make_double2(cv, sv);
        m.Ai[e] = make_double2(cv, sv);
      }
      if (tid == 0) {
        m.dscal[0] = 0.0;  // log|det|
        m.iscal[1] = 0;    // singular flag
      }
      __syncthreads();
      // Gauss-Jordan inversion with partial pivoting (pivot = first row of
      // largest |re|+|im|, as izamax/dcabs1, reptation.f:9079, 9219).
      for (int k = 0; k < n; k++) {
        if (tid < 32) {
          double best = -1.0;
          int bi = k;
          for (int r = k + tid; r < n; r += 32) {
            double v = cabs1(m.Ai[r + k * n]);
            if (v > best) {
              best = v;
              bi = r;
            }
          }
          for (int o = 16; o > 0; o >>= 1) {
            double ob = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) {
              best = ob;
              bi = oi;
            }
          }
          if (tid == 0) {
            m.perm[k] = bi;
            m.iscal[0] = bi;
            if (!(best > 0.0)) m.iscal[1] = 1;
          }
        }
        __syncthreads();
        int p = m.iscal[0];
        if (p != k)
          for (int c = tid; c < n; c += kThreads) {
            double2 a = m.Ai[k + c * n];
            m.Ai[k + c * n] = m.Ai[p + c * n];
            m.Ai[p + c * n] = a;
          }
        __syncthreads();
        double2 piv = m.Ai[k + k * n];
        double d = piv.x * piv.x + piv.y * piv.y;
        double2 inv = make_double2(piv.x / d, -piv.y / d);
        double2 *colk = reinterpret_cast<double2 *>(m.colk);
        for (int r = tid; r < n; r += kThreads) colk[r] = m.Ai[r + k * n];
        if (tid == 0) m.dscal[0] += 0.5 * log(d);
        __syncthreads();
        for (int c = tid; c < n; c += kThreads)
          m.Ai[k + c * n] = (c == k) ? inv : cmul(m.Ai[k + c * n], inv);
        __syncthreads();
        for (int e = tid; e < nn; e += kThreads) {
          int r = e % n, c = e / n;
          if (r == k) continue;
          double2 f = colk[r];
          if (c == k) {
            double2 v = cmul(f, inv);
            m.Ai[e] = make_double2(-v.x, -v.y);
          } else {
            double2 a = m.Ai[k + c * n];
            double2 v = m.Ai[e];
            v.x -= f.x * a.x - f.y * a.y;
            v.y -= f.x * a.y + f.y * a.x;
            m.Ai[e] = v;
          }
        }
        __syncthreads();
      }
      // undo the row interchanges on the columns of the inverse
      for (int k = n - 1; k >= 0; k--) {
        int p = m.perm[k];
        if (p != k)
          for (int r = tid; r < n; r += kThreads) {
            double2 a = m.Ai[r + k * n];
            m.Ai[r + k * n] = m.Ai[r + p * n];
            m.Ai[r + p * n] = a;
          }
        __syncthreads();
      }
      if (m.iscal[1]) status |= ST_SINGULAR;
      logdet_sum += m.dscal[0];
      // F_a(l,j) = sum_k Ainv(l,k) (i g_k[a]) A(k,j)  (zv, reptation.f:10189-10200)
      for (int e = tid; e < nn; e += kThreads) {
        int l = e % n, j = e / n;
        double2 f0v = make_double2(0, 0), f1v = make_double2(0, 0);
        for (int k = 0; k < n; k++) {
          double2 pr = cmul(m.Ai[l + k * n], m.A[k + j * n]);
          double gkx = __ldg(S.gvec + 2 * k), gky = __ldg(S.gvec + 2 * k + 1);
          f0v.x -= gkx * pr.y;
          f0v.y += gkx * pr.x;
          f1v.x -= gky * pr.y;
          f1v.y += gky * pr.x;
        }
        m.F0[e] = f0v;
        m.F1[e] = f1v;
      }
      // D2(j)[ab] = Re sum_k Ainv(j,k) (-g_ka g_kb) A(k,j)  (ddzorb term)
      for (int j = tid; j < n; j += kThreads) {
        double dxx = 0, dxy = 0, dyy = 0;
        for (int k = 0; k < n; k++) {
          double2 pr = cmul(m.Ai[j + k * n], m.A[k + j * n]);
          double gkx = __ldg(S.gvec + 2 * k), gky = __ldg(S.gvec + 2 * k + 1);
          dxx -= gkx * gkx * pr.x;
          dxy -= gkx * gky * pr.x;
          dyy -= gky * gky * pr.x;
        }
        m.D2[3 * j] = dxx;
        m.D2[3 * j + 1] = dxy;
        m.D2[3 * j + 2] = dyy;
      }
      __syncthreads();
      // drift, phase gradient and the first two Laplacian terms for every
      // electron i against this determinant (reptation.f:10201-10237).
      for (int base = 0; base < N; base += per_round) {
        int i = base + tid / kGroup;
        bool valid = i < N;
        int ti = valid ? type_of(S, i) : 0;
        double zxr = 0, zxi = 0, zyr = 0, zyi = 0, t12 = 0;
        if (valid) {
          for (int jl = lane8; jl < n; jl += kGroup) {
            int j = f0 + jl;
            double jxx, jxy, jyx, jyy, qbx, qby;  // J[a][b] = dq_j[a]/dx_i[b]
            if (j == i) {
              jxx = 1.0 + m.Sb[3 * i];
              jxy = m.Sb[3 * i + 1];
              jyx = jxy;
              jyy = 1.0 + m.Sb[3 * i + 2];
              qbx = m.qbd[2 * i];
              qby = m.qbd[2 * i + 1];
            } else {
              double rx, ry, r, byr, rem;
              int ind;
              pair_geom(S, m.x, i, j, rx, ry, r, byr, ind, rem);
              double t, dt, ddt;
              spline3(S, S.iub[ti][sp], ind, rem, t, dt, ddt);
              double c = dt * byr;
              jxx = -(t + c * rx * rx);
              jxy = -(c * rx * ry);
              jyx = jxy;
              jyy = -(t + c * ry * ry);
              double w2 = dt * byr * 3.0 + ddt;
              qbx = -w2 * rx;
              qby = -w2 * ry;
            }
            double2 fx = m.F0[jl + jl * n], fy = m.F1[jl + jl * n];
            zxr += fx.x * jxx + fy.x * jyx;
            zxi += fx.y * jxx + fy.y * jyx;
            zyr += fx.x * jxy + fy.x * jyy;
            zyi += fx.y * jxy + fy.y * jyy;
            t12 -= fx.x * qbx + fy.x * qby;
            // (J^T J)[a][b]
            double jtj_xx = jxx * jxx + jyx * jyx;
            double jtj_xy = jxx * jxy + jyx * jyy;
            double jtj_yy = jxy * jxy + jyy * jyy;
            t12 -= m.D2[3 * jl] * jtj_xx + 2.0 * m.D2[3 * jl + 1] * jtj_xy +
                   m.D2[3 * jl + 2] * jtj_yy;
          }
        }
        zxr = group8_sum(zxr);
        zxi = group8_sum(zxi);
        zyr = group8_sum(zyr);
        zyi = group8_sum(zyi);
        t12 = group8_sum(t12);
        if (valid && lane8 == 0) {
          m.gd[2 * i] -= zxr;
          m.gd[2 * i + 1] -= zyr;
          m.ph2d[i] += zxi * zxi + zyi * zyi;
          m.lapd[i] += t12;
        }
      }
      __syncthreads();
      // cross term: M (2n x 2n, overlaying A and Ainv) then quadratic forms.
      const int n2 = 2 * n;
      double *M = reinterpret_cast<double *>(m.A);
      for (int e = tid; e < n2 * n2; e += kThreads) {
        int p = e % n2, qq = e / n2;
        int a = p / n, j = p - a * n, c = qq / n, k = qq - c * n;
        double2 fa = (a == 0 ? m.F0 : m.F1)[k + j * n];
        double2 fc = (c == 0 ? m.F0 : m.F1)[j + k * n];
        M[e] = fa.x * fc.x - fa.y * fc.y;
      }
      __syncthreads();
      for (int i0 = 0; i0 < N; i0 += kChunk / 2) {
        // U[(a,j)][(i,b)] = J_{j,i}[a][b] for electrons i0 .. i0+15
        for (int e = tid; e < n * (kChunk / 2); e += kThreads) {
          int jl = e % n, il = e / n;
          int i = i0 + il, j = f0 + jl;
          double jxx = 0, jxy = 0, jyy = 0;
          if (i < N) {
            if (j == i) {
              jxx = 1.0 + m.Sb[3 * i];
              jxy = m.Sb[3 * i + 1];
              jyy = 1.0 + m.Sb[3 * i + 2];
            } else {
              double rx, ry, r, byr, rem;
              int ind;
              pair_geom(S, m.x, i, j, rx, ry, r, byr, ind, rem);
              double t, dt, ddt;
              spline3(S, S.iub[type_of(S, i)][sp], ind, rem, t, dt, ddt);
              double c = dt * byr;
              jxx = -(t + c * rx * rx);
              jxy = -(c * rx * ry);
              jyy = -(t + c * ry * ry);
            }
          }
          m.U[(0 * n + jl) * kChunk + 2 * il + 0] = jxx;  // a=x, b=x
          m.U[(0 * n + jl) * kChunk + 2 * il + 1] = jxy;  // a=x, b=y
          m.U[(1 * n + jl) * kChunk + 2 * il + 0] = jxy;  // a=y, b=x
          m.U[(1 * n + jl) * kChunk + 2 * il + 1] = jyy;  // a=y, b=y
        }
        __syncthreads();
        {
          int col = tid & (kChunk - 1), rg = tid / kChunk;
          const int nrg = kThreads / kChunk;
          double part = 0.0;
          for (int p = rg; p < n2; p += nrg) {
            double y = 0.0;
            for (int qq = 0; qq < n2; qq++) y += M[p + qq * n2] * m.U[qq * kChunk + col];
            part += m.U[p * kChunk + col] * y;
          }
          m.red[rg * kChunk + col] = part;
        }
        __syncthreads();
        if (tid < kChunk / 2) {
          int i = i0 + tid;
          if (i < N) {
            double t3 = 0.0;
            for (int rg = 0; rg < kThreads / kChunk; rg++)
              t3 += m.red[rg * kChunk + 2 * tid] + m.red[rg * kChunk + 2 * tid + 1];
            m.lapd[i] += t3;
          }
        }
        __syncthreads();
      }
    }
  }

  // ---- assemble: -ln psi, kinetic (reptation.f:2729), potential (:3986)
  double ltf_j = 0.0;
  for (int i = tid; i < N; i += kThreads) ltf_j += m.ltf[i];
  ltf_j = block_sum(ltf_j, m.red);
  double ltf = ltf_j - logdet_sum;
  bool underflow = false;
  if (S.has_bf && S.ref_underflow) underflow = exp(-ltf * 2.0) <= 0.0;
  if (underflow) status |= ST_UNDERFLOW;
  if (S.has_bf && !underflow) {
    for (int i = tid; i < N; i += kThreads) {
      m.g[2 * i] += m.gd[2 * i];
      m.g[2 * i + 1] += m.gd[2 * i + 1];
      m.lap[i] += m.lapd[i];
      m.ph2[i] = m.ph2d[i];
    }
  }
  __syncthreads();
  // drift cutoff (kinetic, reptation.f:2748-2763)
  double ngg = 0.0, ggsum = 0.0;
  if (S.adrift != 0.0) {
    for (int i = tid; i < N; i += kThreads) {
      int ti = type_of(S, i);
      double vari = 1.0 / (2.0 * S.hbs2m[ti] * S.delta);
      double x2 = m.g[2 * i] * m.g[2 * i] + m.g[2 * i + 1] * m.g[2 * i + 1];
      double gg = x2 * S.adrift * S.delta * S.delta * vari;
      gg = (-1.0 + sqrt(1.0 + 2.0 * gg)) / gg;
      ggsum += gg;
      m.ph2d[i] = x2;  // raw |g|^2 for the kinetic energy
      m.g[2 * i] *= gg;
      m.g[2 * i + 1] *= gg;
    }
    ggsum = block_sum(ggsum, m.red);
    ngg = N;
  }
  double kin0 = 0.0, pot0 = 0.0, efp = 0.0;
  double kin_t[2] = {0, 0}, un_t[2] = {0, 0}, pot_t[2] = {0, 0};
  for (int t = 0; t < nt; t++) {
    double hs = 0.0, g2 = 0.0, vs = 0.0, ph = 0.0;
    for (int i = S.ipfrst[t] + tid; i < S.ipfrst[t] + S.np[t]; i += kThreads) {
      hs += m.lap[i];
      g2 += S.adrift != 0.0 ? m.ph2d[i]
                            : m.g[2 * i] * m.g[2 * i] + m.g[2 * i + 1] * m.g[2 * i + 1];
      vs += m.vp[i];
      ph += m.ph2[i];
    }
    hs = block_sum(hs, m.red);
    g2 = block_sum(g2, m.red);
    vs = block_sum(vs, m.red);
    ph = block_sum(ph, m.red);
    hl[t] = hs;
    kin_t[t] = S.hbs2m[t] * (hs - g2);
    kin0 += kin_t[t];
    kin_t[t] /= S.np[t];
    un_t[t] = 1.0 / sqrt(g2);
    pot_t[t] = vs;
    efp += S.hbs2m[t] * ph;
  }
  kin0 /= S.npnorm;
  // v2 tails (potential, reptation.f:4001-4022)
  for (int it = 0; it < nt; it++) {
    int i = S.iv2[it][it];
    if (i >= 0) pot_t[it] += S.np[it] * (S.np[it] - 1) * 0.5 * S.tab_tail[i];
    for (int jt = it + 1; jt < nt; jt++) {
      i = S.iv2[it][jt];
      if (i < 0) continue;
      double aux = S.np[it] * S.np[jt] * S.tab_tail[i];
      pot_t[it] += 0.5 * aux;
      pot_t[jt] += 0.5 * aux;
    }
  }
  pot0 = 0.0;
  for (int t = 0; t < nt; t++) pot0 += pot_t[t];
  // k space (reptation.f:4034-4052): rho_k read by type index
  for (int it = 0; it < nt; it++)
    for (int jt = 0; jt < nt; jt++) {
      int iv = S.iv2[it][jt];
      if (iv < 0 || S.tab_nkew[iv] == 0) continue;
      const double *vk = S.coef + S.tab_vkoff[iv];
      double aux = 0.0;
      for (int k = tid; k < S.tab_nkew[iv]; k += kThreads)
        aux += __ldg(vk + k) * (m.rhok[2 * (it * S.nk + k)] * m.rhok[2 * (jt * S.nk + k)] +
                                m.rhok[2 * (it * S.nk + k) + 1] * m.rhok[2 * (jt * S.nk + k) + 1]);
      aux = block_sum(aux, m.red);
      double c = aux + __ldg(vk + S.tab_nkew[iv]) * S.npnorm;
      pot_t[it] += c;
      pot0 += c;
    }
  pot0 = (pot0 + S.v0) / S.npnorm;
  efp = S.ntheta != 0 ? efp / S.npnorm : 0.0;
  if (tid == 0) {
    const int J7 = 7;
    props[QMC2D_JLTF] = ltf;
    props[QMC2D_JACC] = 0.0;
    props[QMC2D_JPOT0] = pot0;
    props[QMC2D_JKIN0] = kin0;
    props[QMC2D_JGG] = S.adrift != 0.0 ? ggsum / ngg : 1.0;
    for (int t = 0; t < nt; t++) {
      props[J7 + t] = pot_t[t] / S.np[t];
      props[J7 + nt + t] = kin_t[t];
      props[J7 + 2 * nt + t] = un_t[t];
    }
    props[J7 + 3 * nt] = efp;
    double et = pot0 + kin0 + efp;
    props[QMC2D_JETOT] = et;
    props[QMC2D_JE2] = et * et;
    *sign = 1.0;
  }
  // rho_k properties (compute_properties, reptation.f:2672-2683)
  {
    int cnt = 0;
    for (int it = 0; it < nt; it++) {
      if (S.irhok[it] == 0) continue;
      for (int e = tid; e < 2 * S.nk; e += kThreads)
        props[S.jrhok + cnt + e] = (it < S.nrhok) ? m.rhok[2 * it * S.nk + e] : 0.0;
      cnt += 2 * S.nk;
    }
  }
  __syncthreads();
  double et = props[QMC2D_JETOT];
  if (!isfinite(et) || !isfinite(ltf)) status |= ST_NONFINITE;
  __syncthreads();
  return status;
}

}  // namespace q2d
