// single.cu - VMC with single-electron moves for Slater-Jastrow decks without
// backflow displacement (the reference's only move is all-electron: move,
// reptation.f:4617-4680; this is the single-particle form of the same
// importance-sampled Metropolis step).
//
// One warp per walker, the walker's inverse Slater matrices resident in
// shared memory for the whole launch:
//   * electron i of spin s (column c of that spin's determinant) moves by
//     drift-diffusion from -grad_i ln|psi| to r'; the determinant ratio is
//     R = sum_k W(c,k) phi_k(r') and grad_i ln D(r') = sum_k W(c,k)
//     grad phi_k(r') / R, with W = D^-1 (rows: electrons, columns: orbitals
//     phi_k(r) = exp(i g_k.r)); the two-body Jastrow change is a sum over
//     the N-1 partners;
//   * Metropolis with the reference's acceptance (metropolis_test,
//     reptation.f:2622-2659: p = exp(min(0, max(-50, 2 ln|psi'/psi| +
//     (w_new - w_old)/2))));
//   * an accepted move updates W by Sherman-Morrison (the column of D
//     changes): t = W v, W(c,:) <- W(c,:)/R, W(j,:) <- W(j,:) - t_j W(c,:)
//     for j != c, and ln|det| += ln|R|;
//   * every `refresh` moves both spins' D are rebuilt from the positions and
//     inverted from scratch (Gauss-Jordan with partial pivoting by the warp,
//     in FP64); before that the drift max |W D - I| of the updated inverse
//     is recorded (the reference's zcheck idea, reptation.f:3841);
//   * after each sweep over all N electrons the walker's properties (the
//     reference's p_new vector: -ln psi, energies per type, efp, rho_k) are
//     measured from W in O(n^2 + N^2 + N K) and added to the block sums.
// Limits: no u3, every backflow table identically zero (checked by the
// handle), at most 162 electrons.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"
#include "handle.h"
#include "single.cuh"
#include "walker_eval.cuh"

namespace q2d {

namespace {

constexpr uint32_t kTagSingle = 0x5100u;  // Philox c3 of the single-electron streams
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Two uniforms in (0,1) with 53-bit mantissas from one Philox block (the
// conversion of the other device streams and of the oracle).
__device__ __forceinline__ double2 uni2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
                                        uint32_t c3) {
  uint4 o = philox10(make_uint4(c0, c1, c2, c3),
                     make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  auto cv = [](uint32_t a, uint32_t b) {
    unsigned long long k = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
    return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
  };
  return make_double2(cv(o.x, o.y), cv(o.z, o.w));
}

// Butterfly sum: every lane ends with the same bits.
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// Per-warp shared memory (doubles, each part 16-byte aligned).
struct Sweep {
  double *x;        // 2N positions
  double2 *W[2];    // per spin n_s x n_s, W[j * n + k]
  double2 *Dc[2];   // per spin n_s x n_s, Dc[j * n + k] = phi_k(r_j): the current orbitals
  double2 *Dsc;     // nmax x nmax: D of a refresh
  double2 *v, *t;   // nmax: new orbitals, W v (also the pivot column)
  int *perm;        // nmax row interchanges of a refresh
  double *g, *lap, *vp, *ph2, *ltf;  // 2N, N, N, N, N: the measurement's per-electron sums
  double *rhok;     // 2 * nk * 2
  double *props;    // nprops
};

__host__ __device__ inline size_t al2(size_t n) { return (n + 1) & ~size_t(1); }

__host__ __device__ inline size_t sweep_doubles(const DevSys &s) {
  const size_t N = s.N, nm = s.nmax;
  size_t d = al2(2 * N);
  for (int t = 0; t < s.nt; t++) d += 4 * (size_t)s.np[t] * s.np[t];
  d += 2 * nm * nm + 4 * nm + al2((nm + 1) / 2);
  d += al2(2 * N) + 4 * al2(N) + al2(4 * (size_t)s.nk) + al2(s.nprops);
  return d;
}

__device__ inline Sweep sweep_carve(const DevSys &s, double *p) {
  Sweep m;
  const size_t N = s.N, nm = s.nmax;
  m.x = p;
  p += al2(2 * N);
  for (int t = 0; t < 2; t++) {
    m.W[t] = reinterpret_cast<double2 *>(p);
    if (t < s.nt) p += 2 * (size_t)s.np[t] * s.np[t];
  }
  for (int t = 0; t < 2; t++) {
    m.Dc[t] = reinterpret_cast<double2 *>(p);
    if (t < s.nt) p += 2 * (size_t)s.np[t] * s.np[t];
  }
  m.Dsc = reinterpret_cast<double2 *>(p);
  p += 2 * nm * nm;
  m.v = reinterpret_cast<double2 *>(p);
  p += 2 * nm;
  m.t = reinterpret_cast<double2 *>(p);
  p += 2 * nm;
  m.perm = reinterpret_cast<int *>(p);
  p += al2((nm + 1) / 2);
  m.g = p;
  p += al2(2 * N);
  m.lap = p;
  p += al2(N);
  m.vp = p;
  p += al2(N);
  m.ph2 = p;
  p += al2(N);
  m.ltf = p;
  p += al2(N);
  m.rhok = p;
  p += al2(4 * (size_t)s.nk);
  m.props = p;
  return m;
}

// The first n wave vectors of the determinant (gvec order).
__device__ __forceinline__ double2 gv(const DevSys &S, int k) {
  return make_double2(__ldg(S.gvec + 2 * k), __ldg(S.gvec + 2 * k + 1));
}

// Electron i's first particle index of its spin and the spin's size.
__device__ __forceinline__ void spin_of(const DevSys &S, int i, int &s, int &c, int &n) {
  s = type_of(S, i);
  c = i - S.ipfrst[s];
  n = S.np[s];
}

// In-place Gauss-Jordan inversion of the n x n matrix A (row-major) with
// partial pivoting (the row of largest |re|+|im| in the column, ties to the
// lowest row, as izamax/dcabs1, reptation.f:9079, 9219); row interchanges
// are undone as column interchanges at the end. Returns ln|det A|; sets
// *sing on a zero pivot. The whole warp takes part.
__device__ double warp_invert(double2 *A, int n, double2 *col, int *perm, int lane, int *sing) {
  double logdet = 0.0;
  for (int p = 0; p < n; p++) {
    double best = -1.0;
    int bi = n;
    for (int i = p + lane; i < n; i += 32) {
      const double v = fabs(A[i * n + p].x) + fabs(A[i * n + p].y);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(kFull, best, o);
      const int oi = __shfl_xor_sync(kFull, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (!(best > 0.0)) *sing = 1;
    const int r = bi < n ? bi : p;
    if (lane == 0) perm[p] = r;
    if (r != p)
      for (int c = lane; c < n; c += 32) {
        const double2 a = A[p * n + c];
        A[p * n + c] = A[r * n + c];
        A[r * n + c] = a;
      }
    __syncwarp();
    const double2 piv = A[p * n + p];
    const double d = piv.x * piv.x + piv.y * piv.y;
    logdet += 0.5 * log(d);
    const double2 inv = make_double2(piv.x / d, -piv.y / d);
    for (int i = lane; i < n; i += 32) col[i] = A[i * n + p];
    __syncwarp();
    for (int c = lane; c < n; c += 32) A[p * n + c] = c == p ? inv : cmul(A[p * n + c], inv);
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) {
      const int i = e / n, c = e - i * n;
      if (i == p) continue;
      const double2 f = col[i];
      if (c == p) {
        const double2 q = cmul(f, inv);
        A[e] = make_double2(-q.x, -q.y);
      } else {
        const double2 a = A[p * n + c], w = A[e];
        A[e] = make_double2(w.x - (f.x * a.x - f.y * a.y), w.y - (f.x * a.y + f.y * a.x));
      }
    }
    __syncwarp();
  }
  for (int p = n - 1; p >= 0; p--) {
    const int r = perm[p];
    if (r != p)
      for (int i = lane; i < n; i += 32) {
        const double2 a = A[i * n + p];
        A[i * n + p] = A[i * n + r];
        A[i * n + r] = a;
      }
    __syncwarp();
  }
  return logdet;
}

// D(k, j) = exp(i g_k.r_j) of spin s into m.Dsc; with measure, the largest
// |W D - I| of the current W; then W = D^-1 from scratch. Returns ln|det D|.
__device__ double refresh_spin(const DevSys &S, const Sweep &m, int s, bool measure,
                               double *drift, int lane, int *sing) {
  const int n = S.np[s], f = S.ipfrst[s];
  for (int e = lane; e < n * n; e += 32) {
    const int k = e / n, j = e - k * n;
    const double2 g = gv(S, k);
    double sv, cv;
    sincos(g.x * m.x[2 * (f + j)] + g.y * m.x[2 * (f + j) + 1], &sv, &cv);
    m.Dsc[e] = make_double2(cv, sv);
    m.Dc[s][j * n + k] = make_double2(cv, sv);
  }
  __syncwarp();
  double2 *W = m.W[s];
  if (measure) {
    double e_max = 0.0;
    for (int e = lane; e < n * n; e += 32) {
      const int j = e / n, c = e - j * n;
      double re = 0.0, im = 0.0;
      for (int k = 0; k < n; k++) {
        const double2 w = W[j * n + k], d = m.Dsc[k * n + c];
        re += w.x * d.x - w.y * d.y;
        im += w.x * d.y + w.y * d.x;
      }
      if (j == c) re -= 1.0;
      e_max = fmax(e_max, fabs(re) + fabs(im));
    }
    *drift = fmax(*drift, wmax(e_max));
  }
  for (int e = lane; e < n * n; e += 32) W[e] = m.Dsc[e];
  __syncwarp();
  return warp_invert(W, n, m.t, m.perm, lane, sing);
}

// The drift cutoff of kinetic (reptation.f:2748-2763) on one electron's g.
__device__ __forceinline__ void cutoff(const DevSys &S, int ti, double &gx, double &gy) {
  if (S.adrift == 0.0) return;
  const double x2 = gx * gx + gy * gy;
  const double vari = 1.0 / (2.0 * S.hbs2m[ti] * S.delta);
  double gg = x2 * S.adrift * S.delta * S.delta * vari;
  gg = (-1.0 + sqrt(1.0 + 2.0 * gg)) / gg;
  gx *= gg;
  gy *= gg;
}

// The properties of the walker's current configuration from W (the
// assembly of compute_properties, reptation.f:2661-2727, kinetic :2729,
// potential :3986). Returns status bits.
__device__ int measure(const DevSys &S, const Sweep &m, const double logdet[2], int lane,
                       double *hl_out) {
  const int N = S.N, nt = S.nt;
  // pair sums per electron: u2 drift, Laplacian and half -ln psi_J, half
  // the pair potential
  for (int i = lane; i < N; i += 32) {
    const int ti = type_of(S, i);
    double gx = 0, gy = 0, lp = 0, lt = 0, v = 0;
    for (int j = 0; j < N; j++) {
      if (j == i) continue;
      const int tj = type_of(S, j);
      double rx, ry, r, byr, rem;
      int ind;
      pair_geom(S, m.x, i, j, rx, ry, r, byr, ind, rem);
      const double *row = pair_row(S, ti, tj, ind);
      if (S.has_u2) {
        double f, df, ddf;
        spline3(S, row + PR_U2, rem, f, df, ddf);
        lt += 0.5 * f;
        const double dtr = df * byr;
        gx += dtr * rx;
        gy += dtr * ry;
        lp += ddf + dtr;
      }
      if (S.has_v2) v += 0.5 * spline0(S, row + PR_V2, S.tab_iexp[S.iv2[ti][tj]], rem, byr);
    }
    m.g[2 * i] = gx;
    m.g[2 * i + 1] = gy;
    m.lap[i] = lp;
    m.ltf[i] = lt;
    m.vp[i] = v;
  }
  // rho_k per type slot
  for (int e = lane; e < nt * S.nk; e += 32) {
    const int ty = e / S.nk, k = e - ty * S.nk;
    if (S.irhok[ty] == 0) continue;
    const double kx = __ldg(S.kvec + 2 * k), ky = __ldg(S.kvec + 2 * k + 1);
    double c = 0.0, sn = 0.0;
    for (int i = S.ipfrst[ty]; i < S.ipfrst[ty] + S.np[ty]; i++) {
      double sv, cv;
      sincos(kx * m.x[2 * i] + ky * m.x[2 * i + 1], &sv, &cv);
      c += cv;
      sn += sv;
    }
    const int slot = S.irhok[ty] - 1;
    m.rhok[2 * (slot * S.nk + k)] = c;
    m.rhok[2 * (slot * S.nk + k) + 1] = sn;
  }
  __syncwarp();
  double lt = 0.0;
  for (int i = lane; i < N; i += 32) lt += m.ltf[i];
  const double ltf = wsum(lt) - (logdet[0] + (nt > 1 ? logdet[1] : 0.0));
  int status = 0;
  const bool underflow = S.has_bf && S.ref_underflow && exp(-ltf * 2.0) <= 0.0;
  if (underflow) status |= ST_UNDERFLOW;
  // determinant drift, Laplacian and phase gradient per electron
  double sums[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = lane; i < N; i += 32) {
    int s, c, n;
    spin_of(S, i, s, c, n);
    double gx = m.g[2 * i], gy = m.g[2 * i + 1], lp = m.lap[i], ph = 0.0;
    if (S.has_bf && !underflow) {
      const double2 *W = m.W[s];
      double2 Gx = make_double2(0, 0), Gy = Gx, L = Gx;
      const double2 *Dc = m.Dc[s];
      for (int k = 0; k < n; k++) {
        const double2 g = gv(S, k);
        const double2 wp = cmul(W[c * n + k], Dc[c * n + k]);
        Gx.x -= g.x * wp.y;
        Gx.y += g.x * wp.x;
        Gy.x -= g.y * wp.y;
        Gy.y += g.y * wp.x;
        const double gg = g.x * g.x + g.y * g.y;
        L.x -= gg * wp.x;
        L.y -= gg * wp.y;
      }
      gx -= Gx.x;
      gy -= Gy.x;
      lp -= L.x - (Gx.x * Gx.x - Gx.y * Gx.y + Gy.x * Gy.x - Gy.y * Gy.y);
      ph = Gx.y * Gx.y + Gy.y * Gy.y;
    }
    const double x2 = gx * gx + gy * gy;
    if (S.adrift != 0.0) {
      const int ti = type_of(S, i);
      const double vari = 1.0 / (2.0 * S.hbs2m[ti] * S.delta);
      double gg = x2 * S.adrift * S.delta * S.delta * vari;
      gg = (-1.0 + sqrt(1.0 + 2.0 * gg)) / gg;
      sums[8] += gg;
      gx *= gg;
      gy *= gg;
    }
    m.g[2 * i] = gx;
    m.g[2 * i + 1] = gy;
    const bool t1 = s == 1;  // compile-time indices: the sums stay in registers
    sums[0] += t1 ? 0.0 : lp;
    sums[1] += t1 ? 0.0 : x2;
    sums[2] += t1 ? 0.0 : m.vp[i];
    sums[3] += t1 ? 0.0 : ph;
    sums[4] += t1 ? lp : 0.0;
    sums[5] += t1 ? x2 : 0.0;
    sums[6] += t1 ? m.vp[i] : 0.0;
    sums[7] += t1 ? ph : 0.0;
  }
#pragma unroll
  for (int q = 0; q < 9; q++) sums[q] = wsum(sums[q]);
  double kin0 = 0.0, pot0 = 0.0, efp = 0.0;
  double kin_t[2] = {0, 0}, un_t[2] = {0, 0}, pot_t[2] = {0, 0};
#pragma unroll
  for (int t = 0; t < 2; t++) {
    if (t < nt) {
      const double hs = sums[4 * t], g2 = sums[4 * t + 1];
      hl_out[t] = hs;
      kin_t[t] = S.hbs2m[t] * (hs - g2);
      kin0 += kin_t[t];
      kin_t[t] /= S.np[t];
      un_t[t] = 1.0 / sqrt(g2);
      pot_t[t] = sums[4 * t + 2];
      efp += S.hbs2m[t] * sums[4 * t + 3];
    }
  }
  kin0 /= S.npnorm;
#pragma unroll
  for (int it = 0; it < 2; it++) {
    if (it >= nt) continue;
    int iv = S.iv2[it][it];
    if (iv >= 0) pot_t[it] += S.np[it] * (S.np[it] - 1) * 0.5 * S.tab_tail[iv];
    if (it == 0 && nt > 1) {
      iv = S.iv2[0][1];
      if (iv >= 0) {
        const double aux = S.np[0] * S.np[1] * S.tab_tail[iv];
        pot_t[0] += 0.5 * aux;
        pot_t[1] += 0.5 * aux;
      }
    }
  }
  pot0 = pot_t[0] + pot_t[1];
#pragma unroll
  for (int it = 0; it < 2; it++)
#pragma unroll
    for (int jt = 0; jt < 2; jt++) {
      if (it >= nt || jt >= nt) continue;
      const int iv = S.iv2[it][jt];
      if (iv < 0 || S.tab_nkew[iv] == 0) continue;
      const double *vk = S.coef + S.tab_vkoff[iv];
      double ks = 0.0;
      for (int k = lane; k < S.tab_nkew[iv]; k += 32)
        ks += __ldg(vk + k) * (m.rhok[2 * (it * S.nk + k)] * m.rhok[2 * (jt * S.nk + k)] +
                               m.rhok[2 * (it * S.nk + k) + 1] * m.rhok[2 * (jt * S.nk + k) + 1]);
      const double c = wsum(ks) + S.tab_kself[iv] * S.npnorm;
      pot_t[it] += c;
      pot0 += c;
    }
  pot0 = (pot0 + S.v0) / S.npnorm;
  efp = S.ntheta != 0 ? efp / S.npnorm : 0.0;
  double *props = m.props;
  if (lane == 0) {
    props[QMC2D_JLTF] = ltf;
    props[QMC2D_JPOT0] = pot0;
    props[QMC2D_JKIN0] = kin0;
    props[QMC2D_JGG] = S.adrift != 0.0 ? sums[8] / N : 1.0;
#pragma unroll
    for (int t = 0; t < 2; t++) {
      if (t >= nt) continue;
      props[7 + t] = pot_t[t] / S.np[t];
      props[7 + nt + t] = kin_t[t];
      props[7 + 2 * nt + t] = un_t[t];
    }
    props[7 + 3 * nt] = efp;
    const double et = pot0 + kin0 + efp;
    props[QMC2D_JETOT] = et;
    props[QMC2D_JE2] = et * et;
  }
  int cnt = 0;
  for (int it = 0; it < nt; it++) {
    if (S.irhok[it] == 0) continue;
    for (int e = lane; e < 2 * S.nk; e += 32)
      props[S.jrhok + cnt + e] = (it < S.nrhok) ? m.rhok[2 * it * S.nk + e] : 0.0;
    cnt += 2 * S.nk;
  }
  __syncwarp();
  if (!isfinite(props[QMC2D_JETOT]) || !isfinite(ltf)) status |= ST_NONFINITE;
  return status;
}

__global__ void __launch_bounds__(128, 1) single_kernel(const DevSys *sp, SingleArgs a,
                                                     size_t per_warp) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) double sm_single[];
  {
    const int *src = reinterpret_cast<const int *>(sp);
    int *dst = reinterpret_cast<int *>(&S);
    for (int q = threadIdx.x; q < (int)(sizeof(DevSys) / sizeof(int)); q += blockDim.x)
      dst[q] = src[q];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w = blockIdx.x * (blockDim.x >> 5) + warp;
  if (w >= a.nw) return;  // whole warps leave; no CTA barrier follows
  const Sweep m = sweep_carve(S, sm_single + warp * per_warp);
  const int N = S.N, N2 = 2 * N;
  for (int k = lane; k < N2; k += 32) m.x[k] = a.pop.x[(size_t)w * N2 + k];
  __syncwarp();
  int sing = 0, status = 0;
  double drift = 0.0, logdet[2] = {0.0, 0.0};
  for (int s = 0; s < S.nt; s++) logdet[s] = refresh_spin(S, m, s, false, &drift, lane, &sing);
  double nacc = 0.0, hl[2] = {0.0, 0.0};
  int since = 0;
  double *blk = a.blk + (size_t)w * S.nprops;
  for (int sw = 0; sw < a.nsweep; sw++) {
    const uint32_t t = a.sweep0 + (uint32_t)sw;
    double psum = 0.0;
    long long tph = clock64();
    const bool lead = lane == 0;
    for (int i = 0; i < N; i++) {
      int s, c, n;
      spin_of(S, i, s, c, n);
      const double var = 2.0 * S.hbs2m[s] * a.delta, vari = 1.0 / var;
      const double xi = m.x[2 * i], yi = m.x[2 * i + 1];
      // the draws first: they depend on nothing else
      const double2 u0 = uni2(a.seed, (uint32_t)(2 * i), (uint32_t)w, t, kTagSingle);
      const double2 u1 = uni2(a.seed, (uint32_t)(2 * i + 1), (uint32_t)w, t, kTagSingle);
      const double ua = uni2(a.seed, 0x80000000u | (uint32_t)i, (uint32_t)w, t, kTagSingle).x;
      const double2 *Wc = m.W[s] + c * n;
      const double2 *Dcc = m.Dc[s] + c * n;
      const int ti = s;
      // the Gaussian step (move, reptation.f:4633) is issued before the old
      // position's sums, so its transcendental latency overlaps them
      const double pi = 3.141592653589793;
      const double cx = cos(pi * u0.x) * sqrt(-2.0 * var * log(u0.y));
      const double cy = cos(pi * u1.x) * sqrt(-2.0 * var * log(u1.y));
      // -grad_i ln|psi| at the old position and sum_m u(r_im): the orbitals
      // from the cache, the partners' splines, one butterfly for both
      double o[5] = {0, 0, 0, 0, 0};  // Re G_x, Re G_y, J_x, J_y, u
      for (int q = lane; q < (n > N ? n : N); q += 32) {
        if (q < n) {
          const double2 g = gv(S, q), wp = cmul(Wc[q], Dcc[q]);
          o[0] -= g.x * wp.y;
          o[1] -= g.y * wp.y;
        }
        if (q < N && q != i && S.has_u2) {
          double rx = xi - m.x[2 * q], ry = yi - m.x[2 * q + 1];
          rx = rx - S.el[0] * round(S.eli[0] * rx);
          ry = ry - S.el[1] * round(S.eli[1] * ry);
          const double r2 = rx * rx + ry * ry, byr = rsqrt(r2), r = r2 * byr;
          const int ind = (int)(r * S.drti);
          const double rem = r - ind * S.drt;
          double f, df, ddf;
          spline3(S, pair_row(S, ti, type_of(S, q), ind) + PR_U2, rem, f, df, ddf);
          const double dtr = df * byr;
          o[2] += dtr * rx;
          o[3] += dtr * ry;
          o[4] += f;
        }
      }
#pragma unroll
      for (int q = 0; q < 5; q++) o[q] = wsum(o[q]);
      double gx = o[2] - o[0], gy = o[3] - o[1];
      const double uold = o[4];
      cutoff(S, s, gx, gy);
      // the proposal (move, reptation.f:4631-4646, for one electron)
      const double nx = xi - var * gx + cx, ny = yi - var * gy + cy;
      const double wold = -(cx * cx + cy * cy) * vari;
      phase_mark(S, PH_PROPOSE, tph, lead);
      // the ratio, grad ln D and the Jastrow at the new position
      double e9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // R, N_x, N_y (complex), J_x, J_y, u
      for (int q = lane; q < (n > N ? n : N); q += 32) {
        if (q < n) {
          const double2 g = gv(S, q);
          double sv, cv;
          sincos(g.x * nx + g.y * ny, &sv, &cv);
          m.v[q] = make_double2(cv, sv);
          const double2 wp = cmul(Wc[q], make_double2(cv, sv));
          e9[0] += wp.x;
          e9[1] += wp.y;
          e9[2] -= g.x * wp.y;
          e9[3] += g.x * wp.x;
          e9[4] -= g.y * wp.y;
          e9[5] += g.y * wp.x;
        }
        if (q < N && q != i && S.has_u2) {
          double rx = nx - m.x[2 * q], ry = ny - m.x[2 * q + 1];
          rx = rx - S.el[0] * round(S.eli[0] * rx);
          ry = ry - S.el[1] * round(S.eli[1] * ry);
          const double r2 = rx * rx + ry * ry, byr = rsqrt(r2), r = r2 * byr;
          const int ind = (int)(r * S.drti);
          const double rem = r - ind * S.drt;
          double f, df, ddf;
          spline3(S, pair_row(S, ti, type_of(S, q), ind) + PR_U2, rem, f, df, ddf);
          const double dtr = df * byr;
          e9[6] += dtr * rx;
          e9[7] += dtr * ry;
          e9[8] += f;
        }
      }
#pragma unroll
      for (int q = 0; q < 9; q++) e9[q] = wsum(e9[q]);
      const double2 R = make_double2(e9[0], e9[1]);
      const double2 dgx = cdiv(make_double2(e9[2], e9[3]), R);
      const double2 dgy = cdiv(make_double2(e9[4], e9[5]), R);
      const double unew = e9[8];
      double hx = e9[6] - dgx.x, hy = e9[7] - dgy.x;
      cutoff(S, s, hx, hy);
      const double bx = xi - nx + var * hx, by = yi - ny + var * hy;
      const double wnew = -(bx * bx + by * by) * vari;
      const double lnr = 0.5 * log(R.x * R.x + R.y * R.y) - (unew - uold);
      double p = 2.0 * lnr + 0.5 * (wnew - wold);
      p = exp(fmin(0.0, fmax(-50.0, p)));
      if (!(R.x * R.x + R.y * R.y > 0.0)) p = 0.0;
      psum += p;
      phase_mark(S, PH_PAIRS, tph, lead);
      if (p >= ua) {
        // Sherman-Morrison: column c of D becomes v
        double2 *W = m.W[s];
        for (int j = lane; j < n; j += 32) {
          double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
          int k = 0;
          for (; k + 1 < n; k += 2) {
            const double2 a0 = W[j * n + k], b0 = m.v[k];
            const double2 a1 = W[j * n + k + 1], b1 = m.v[k + 1];
            re0 += a0.x * b0.x - a0.y * b0.y;
            im0 += a0.x * b0.y + a0.y * b0.x;
            re1 += a1.x * b1.x - a1.y * b1.y;
            im1 += a1.x * b1.y + a1.y * b1.x;
          }
          if (k < n) {
            const double2 a0 = W[j * n + k], b0 = m.v[k];
            re0 += a0.x * b0.x - a0.y * b0.y;
            im0 += a0.x * b0.y + a0.y * b0.x;
          }
          m.t[j] = make_double2(re0 + re1, im0 + im1);
        }
        __syncwarp();
        const double2 Rc = m.t[c];
        const double rd = 1.0 / (Rc.x * Rc.x + Rc.y * Rc.y);
        const double2 rinv = make_double2(Rc.x * rd, -Rc.y * rd);
        for (int k = lane; k < n; k += 32) {
          W[c * n + k] = cmul(W[c * n + k], rinv);
          m.Dc[s][c * n + k] = m.v[k];
        }
        __syncwarp();
        for (int e = lane; e < n * n; e += 32) {
          const int j = e / n, k = e - j * n;
          if (j == c) continue;
          const double2 q = cmul(m.t[j], W[c * n + k]);
          W[e] = make_double2(W[e].x - q.x, W[e].y - q.y);
        }
        if (lane == 0) {
          m.x[2 * i] = nx;
          m.x[2 * i + 1] = ny;
        }
        __syncwarp();
        logdet[s] += 0.5 * log(Rc.x * Rc.x + Rc.y * Rc.y);
        nacc += 1.0;
      }
      phase_mark(S, PH_ACCEPT, tph, lead);
      if (a.refresh > 0 && ++since >= a.refresh) {
        for (int q = 0; q < S.nt; q++) logdet[q] = refresh_spin(S, m, q, true, &drift, lane, &sing);
        since = 0;
        phase_mark(S, PH_INVERT, tph, lead);
      }
    }
    status |= measure(S, m, logdet, lane, hl);
    phase_mark(S, PH_ASSEMBLE, tph, lead);
    if (lane == 0) m.props[QMC2D_JACC] = psum / N;
    __syncwarp();
    for (int ip = lane; ip < S.nprops; ip += 32) blk[ip] += m.props[ip];
  }
  if (sing) status |= ST_SINGULAR;
  for (int k = lane; k < N2; k += 32) {
    a.pop.x[(size_t)w * N2 + k] = m.x[k];
    a.pop.g[(size_t)w * N2 + k] = m.g[k];
  }
  if (a.nsweep > 0)
    for (int ip = lane; ip < S.nprops; ip += 32) a.pop.p[(size_t)w * S.nprops + ip] = m.props[ip];
  if (lane == 0) {
    if (a.nsweep > 0) {
      for (int t = 0; t < S.nt; t++) a.pop.h[(size_t)w * S.nt + t] = hl[t];
      a.pop.s[w] = 1.0;
      a.pop.age[w] = 0.0;
    }
    a.blk_norm[w] += a.nsweep;
    a.cnt[4 * w] += nacc;
    a.cnt[4 * w + 1] += (double)N * a.nsweep;
    a.drift[w] = fmax(a.drift[w], drift);
    if (status & (ST_SINGULAR | ST_NONFINITE)) atomicOr(&a.status[w], status);
  }
}

}  // namespace

size_t single_smem_per_walker(const DevSys &s) { return sizeof(double) * sweep_doubles(s); }

cudaError_t launch_single(const DevSys &hs, const DevSys *ds, const SingleArgs &a,
                          cudaStream_t st) {
  if (a.nw <= 0) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
      cudaSuccess)
    return e;
  const size_t per = sweep_doubles(hs);
  const size_t room = (size_t)optin - sizeof(DevSys) - 64;
  int nsm = 0;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return e;
  // spread small populations over the SMs (one walker per CTA), pack up to
  // four per CTA when there are walkers enough to fill them
  int wpb = a.nw >= 4 * 2 * nsm ? 4 : (a.nw >= 2 * 2 * nsm ? 2 : 1);
  while (wpb > 1 && wpb * per * sizeof(double) > room) wpb--;
  if (per * sizeof(double) > room) return cudaErrorInvalidConfiguration;
  const size_t sm = wpb * per * sizeof(double);
  if ((e = raise_smem_limit((const void *)single_kernel, sm)) != cudaSuccess) return e;
  const int grid = (a.nw + wpb - 1) / wpb;
  single_kernel<<<grid, 32 * wpb, sm, st>>>(ds, a, per);
  return cudaGetLastError();
}

}  // namespace q2d

// ------------------------------------------------------------------ C-ABI
extern "C" int qmc2d_vmc_single(qmc2d_handle *h, int nsweep, double delta, int refresh) {
  if (!h || nsweep < 0 || refresh < 0 || !(delta > 0.0)) {
    q2d::set_error("qmc2d_vmc_single: bad argument");
    return QMC2D_ERR_ARG;
  }
  if (h->nw <= 0) {
    q2d::set_error("qmc2d_vmc_single: empty population");
    return QMC2D_ERR_STACK;
  }
  if (h->hs.has_u3 || (h->hs.has_bf && !h->bf_zero)) {
    q2d::set_error("qmc2d_vmc_single: single-electron moves need a deck without u3 and "
                   "without backflow displacement (backflow tables identically zero)");
    return QMC2D_ERR_UNSUPPORTED;
  }
  cudaError_t e;
  auto fail = [](cudaError_t err, const char *what) {
    q2d::set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return QMC2D_ERR_CUDA;
  };
  if ((e = cudaSetDevice(h->device)) != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = join_side(h)) != cudaSuccess) return fail(e, "cudaStreamWaitEvent");
  if (h->hs.delta != delta && h->hs.adrift != 0.0) {
    h->hs.delta = delta;
    if ((e = cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess)
      return fail(e, "cudaMemcpyAsync");
  }
  if ((e = cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->d_sdrift, 0, sizeof(double) * h->nw, h->stream)) != cudaSuccess)
    return fail(e, "cudaMemsetAsync");
  q2d::SingleArgs a{};
  a.nw = h->nw;
  a.nsweep = nsweep;
  a.refresh = refresh;
  a.delta = delta;
  a.seed = h->seed;
  a.sweep0 = h->sweep_counter;
  a.pop = h->pop[h->cur];
  a.blk = h->d_blk;
  a.blk_norm = h->d_norm;
  a.cnt = h->d_cnt;
  a.drift = h->d_sdrift;
  a.status = h->d_status;
  {
    ProfScope ps(h, QMC2D_KERNEL_SINGLE, h->stream);
    if ((e = q2d::launch_single(h->hs, h->ds, a, h->stream)) != cudaSuccess) {
      if (e == cudaErrorInvalidConfiguration) {
        q2d::set_error("qmc2d_vmc_single: one walker's inverse does not fit shared memory");
        return QMC2D_ERR_LIMIT;
      }
      return fail(e, "single-electron sweep kernel");
    }
  }
  h->sweep_counter += (uint32_t)nsweep;
  return q2d_sync_status(h, h->nw);
}

extern "C" int qmc2d_single_drift(qmc2d_handle *h, double *max_err) {
  if (!h || !max_err) return QMC2D_ERR_ARG;
  cudaError_t e;
  if ((e = cudaSetDevice(h->device)) != cudaSuccess || (e = join_side(h)) != cudaSuccess ||
      (e = cudaStreamSynchronize(h->stream)) != cudaSuccess) {
    q2d::set_error(std::string("qmc2d_single_drift: ") + cudaGetErrorString(e));
    return QMC2D_ERR_CUDA;
  }
  std::vector<double> d(h->nw > 0 ? h->nw : 1, 0.0);
  if (h->nw > 0 &&
      (e = cudaMemcpy(d.data(), h->d_sdrift, sizeof(double) * h->nw, cudaMemcpyDeviceToHost)) !=
          cudaSuccess) {
    q2d::set_error(std::string("qmc2d_single_drift: ") + cudaGetErrorString(e));
    return QMC2D_ERR_CUDA;
  }
  double mx = 0.0;
  for (int i = 0; i < h->nw; i++) mx = d[i] > mx ? d[i] : mx;
  *max_err = mx;
  return QMC2D_OK;
}
