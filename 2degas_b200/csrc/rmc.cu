// rmc.cu - reptation QMC on the device: one CTA per reptile, the path ring
// in HBM. Restates read_path (reptation.f:1775), get_w_stack (:1804), fgg
// (:1853), reptation_metropolis_test (:1865), reptation_move (:1897) and
// the scalar part of path_props (:1567-1577). Random draws follow the
// Philox stream layout documented in include/qmc2d.h's RMC section.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/qmc2d.h"
#include "common.h"
#include "kernels.cuh"
#include "rmc.cuh"
#include "walker_eval.cuh"

namespace q2d {

namespace {

enum { JBRA = 0, JDTP = 1, JITP = 2, JLNG = 3, JNDS = 4 };

__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
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

__device__ __forceinline__ double2 u2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
                                      uint32_t c3) {
  uint4 o = philox(make_uint4(c0, c1, c2, c3), make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  auto cv = [](uint32_t a, uint32_t b) {
    unsigned long long k = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
    return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
  };
  return make_double2(cv(o.x, o.y), cv(o.z, o.w));
}

struct RmcArgs {
  int nrep, ntau, ntauskip, mdelta, nbuf, nstp;
  double delta, etrial, mage, mage_r;
  uint64_t seed;
  uint32_t step0;
  int ecut, rejection, wpiu, gstorto, nodalaction;
  double value_ecut;
  double *x, *g, *p, *h, *s, *age_stack, *w, *pp_old, *age;
  double *psum;  // nrep * nprops: raw window sums of the accepted paths
  int *ends;
  double *blk, *blk_norm, *cnt;
  int *status;
};

__device__ __forceinline__ void load_sys(DevSys &S, const DevSys *sp) {
  const int *src = reinterpret_cast<const int *>(sp);
  int *dst = reinterpret_cast<int *>(&S);
  for (int i = threadIdx.x; i < (int)(sizeof(DevSys) / sizeof(int)); i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
}

__device__ __forceinline__ double fgg(const RmcArgs &a, double e, double gg) {
  return a.ecut == 0 ? e : a.value_ecut + (e - a.value_ecut) * gg;
}

// Direction and number of bead growths of reptile r's move t
// (reptation_move, reptation.f:1915-1925): the same draw in every launch
// of the move.
__device__ __forceinline__ void rmc_dir(const RmcArgs &a, int r, uint32_t t, int &idir,
                                        int &ndelta) {
  const double2 dl = u2(a.seed, 0xFFFFFFF0u, (uint32_t)r, t, 2u);
  idir = (dl.x - 0.5) >= 0.0 ? 1 : -1;
  ndelta = 1 + (int)(dl.y * a.mdelta);
}

// Bead pointers of reptile r, ring slot j.
struct Bead {
  double *x, *g, *p, *h, *s, *age, *w;
};
__device__ __forceinline__ Bead bead(const DevSys &S, const RmcArgs &a, int r, int j) {
  size_t b = (size_t)r * a.nbuf + j;
  Bead o;
  o.x = a.x + b * 2 * S.N;
  o.g = a.g + b * 2 * S.N;
  o.p = a.p + b * S.nprops;
  o.h = a.h + b * S.nt;
  o.s = a.s + b;
  o.age = a.age_stack + b;
  o.w = a.w + b * 5;
  return o;
}

// path_props scalar part: mean over beads 1+ntauskip..ntau-ntauskip from
// kfirst; E_L is the mixed estimator of the two ends. raw (when given)
// receives the window sums before the division.
__device__ void path_props(const DevSys &S, const RmcArgs &a, int r, int kfirst, int klast,
                           double *pp, double *raw = nullptr) {
  for (int ip = threadIdx.x; ip < S.nprops; ip += blockDim.x) {
    double t = 0.0;
    for (int i = 1 + a.ntauskip; i <= a.ntau - a.ntauskip; i++) {
      int j = (kfirst + i - 1) % a.nbuf;
      t += bead(S, a, r, j).p[ip];
    }
    if (raw) raw[ip] = t;
    pp[ip] = t / (a.ntau - 2 * a.ntauskip);
  }
  __syncthreads();
  if (threadIdx.x == 0)
    pp[QMC2D_JETOT] =
        0.5 * (bead(S, a, r, klast).p[QMC2D_JETOT] + bead(S, a, r, kfirst).p[QMC2D_JETOT]);
  __syncthreads();
}

// The proposed path's window sums (the sums of path_props) from the
// accepted path's, psum: the window of beads ntauskip .. ntau-ntauskip-1
// after the first shifts by d = idir * ndelta ring slots, so |d| beads leave
// at one end and |d| enter at the other; every bead of the old window is
// still in its slot (the grown beads go to the spare slots beyond the ends).
// A full rescan when the windows do not overlap or `full` (every 256th
// step, so round-off of the running sums cannot build up).
__device__ void path_sums(const DevSys &S, const RmcArgs &a, int r, int jfirst, int d,
                          const double *psum, double *out, bool full) {
  const int cnt = a.ntau - 2 * a.ntauskip, nb = a.nbuf;
  const int e = d < 0 ? -d : d;
  const int kf = (jfirst + d + nb) % nb;
  for (int ip = threadIdx.x; ip < S.nprops; ip += blockDim.x) {
    double t;
    if (full || e >= cnt) {
      t = 0.0;
      for (int i = 0; i < cnt; i++) t += bead(S, a, r, (kf + a.ntauskip + i) % nb).p[ip];
    } else {
      t = psum[ip];
      for (int q = 0; q < e; q++) {
        const int out_slot = d > 0 ? jfirst + a.ntauskip + q : jfirst + a.ntauskip + cnt - 1 - q;
        const int in_slot = d > 0 ? jfirst + a.ntauskip + cnt + q : kf + a.ntauskip + q;
        t += bead(S, a, r, in_slot % nb).p[ip] - bead(S, a, r, out_slot % nb).p[ip];
      }
    }
    out[ip] = t;
  }
  __syncthreads();
}

// get_w_stack (reptation.f:1804-1851) for beads j -> jn; returns wnew/wold.
__device__ void get_w_stack(const DevSys &S, const RmcArgs &a, int r, int j, int jn, double *red,
                            double *wnew_out, double *wold_out) {
  Bead bj = bead(S, a, r, j), bn = bead(S, a, r, jn);
  double wf = 0, wb = 0, wg = 0;
  for (int k = threadIdx.x; k < 2 * S.N; k += blockDim.x) {
    int t = type_of(S, k >> 1);
    double var = 2.0 * S.hbs2m[t] * a.delta, vari = 1.0 / var;
    double d0 = bj.x[k] - bn.x[k];
    wg -= d0 * d0 * vari;
    double df = -var * bj.g[k];
    double d1 = bj.x[k] + df - bn.x[k];
    wf -= d1 * d1 * vari;
    double db = -var * bn.g[k];
    double d2 = bj.x[k] - db - bn.x[k];
    wb -= d2 * d2 * vari;
  }
  double wnew = block_sum(wb, red), wold = block_sum(wf, red), lng = block_sum(wg, red);
  if (threadIdx.x == 0) {
    lng += a.delta * S.npnorm * (bj.p[QMC2D_JKIN0] + bn.p[QMC2D_JKIN0]);
    bj.w[JLNG] = 0.5 * lng;
    bj.w[JDTP] = 0.5 * wold;
    bj.w[JBRA] = -.5 * a.delta * S.npnorm *
                 (fgg(a, bj.p[QMC2D_JETOT], bj.p[QMC2D_JGG]) +
                  fgg(a, bn.p[QMC2D_JETOT], bn.p[QMC2D_JGG]) - 2.0 * a.etrial);
    bn.w[JITP] = 0.5 * wnew;
    double nds = 0.0;
    for (int t = 0; t < S.nt; t++) {
      int ju = QMC2D_JUN(S.nt, t);
      double var = 2.0 * S.hbs2m[t] * a.delta;
      nds -= log(1.0 - exp(-bj.p[ju] * bn.p[ju] / (0.5 * var)));
    }
    bj.w[JNDS] = nds;
  }
  __syncthreads();
  *wnew_out = wnew;
  *wold_out = wold;
}

// read_path after the beads are evaluated: w_stack, bead acceptances,
// path properties, ends.
__global__ void rmc_init_kernel(const DevSys *sp, RmcArgs a) {
  __shared__ DevSys S;
  __shared__ double red[32];
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  double *pp = reinterpret_cast<double *>(smem);
  const int r = blockIdx.x;
  if (r >= a.nrep) return;
  for (int i = 0; i < a.ntau; i++) {
    Bead b = bead(S, a, r, i);
    if (threadIdx.x == 0) {
      b.p[QMC2D_JACC] = 1.0;
      *b.age = 0.0;
    }
  }
  __syncthreads();
  path_props(S, a, r, 0, a.ntau - 1, pp);
  for (int i = 1; i <= a.ntau - 1; i++) {
    int j = i - 1, jn = i;
    double wnew, wold;
    get_w_stack(S, a, r, j, jn, red, &wnew, &wold);
    if (threadIdx.x == 0) {
      Bead bj = bead(S, a, r, j), bn = bead(S, a, r, jn);
      double p = 2 * (bj.p[QMC2D_JLTF] - bn.p[QMC2D_JLTF]) + 0.5 * (wnew - wold);
      p = fmin(0.0, fmax(-50.0, p));
      bn.p[QMC2D_JACC] = exp(p);
    }
    __syncthreads();
  }
  for (int ip = threadIdx.x; ip < S.nprops; ip += blockDim.x)
    a.pp_old[(size_t)r * S.nprops + ip] = pp[ip];
  // the window sums the moves update, with the bead acceptances just set
  path_sums(S, a, r, 0, 0, nullptr, a.psum + (size_t)r * S.nprops, true);
  if (threadIdx.x == 0) {
    a.ends[2 * r] = 0;
    a.ends[2 * r + 1] = a.ntau - 1;
    a.age[r] = 0.0;
  }
}

// Evaluate beads b0 .. b0 + gridDim.x - 1 (reptile-major). With kGmat the
// CTA's determinant matrices take walker block blockIdx.x of the handle's
// device memory, so a launch covers at most the handle's capacity.
template <bool kGmat>
__global__ void __launch_bounds__(kThreads, 2) rmc_eval_beads_kernel(const DevSys *sp, RmcArgs a,
                                                                  const double *x, int b0) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  EvalSmem m;
  size_t off = eval_carve<kGmat>(S, smem, &m, kGmat ? gmat_block(S, blockIdx.x) : nullptr);
  double *pn = reinterpret_cast<double *>(smem + off);
  double *hn = pn + S.nprops;
  double *sn = hn + 2;
  const int bead_id = b0 + blockIdx.x;
  const int r = bead_id / a.ntau, i = bead_id % a.ntau;
  const int N2 = 2 * S.N;
  Bead b = bead(S, a, r, i);
  for (int k = threadIdx.x; k < N2; k += blockDim.x) {
    double v = x[((size_t)r * a.ntau + i) * N2 + k];
    m.x[k] = v;
    b.x[k] = v;
  }
  __syncthreads();
  long long tph = clock64();
  int st = eval_walker<double, kGmat>(S, m, hn, pn, sn, tph);
  for (int k = threadIdx.x; k < N2; k += blockDim.x) b.g[k] = m.g[k];
  for (int k = threadIdx.x; k < S.nprops; k += blockDim.x) b.p[k] = pn[k];
  if (threadIdx.x == 0) {
    for (int t = 0; t < S.nt; t++) b.h[t] = hn[t];
    *b.s = *sn;
    if (st) atomicOr(&a.status[r], st);
  }
}

// The bead growth after its evaluation (reptation_move, reptation.f:1961-2104):
// the reverse move, the bead's Langevin test (reptation_metropolis_test's
// per-bead part), the w_stack entries of the link and the new bead jn (a
// copy of bead j when rejected). m holds the proposal's positions and drift,
// pn / hn / sc[0] its properties, -lap per type and sign. Every thread of
// the CTA calls it.
__device__ void bead_tail(const DevSys &S, const RmcArgs &a, const EvalSmem &m, int r,
                          uint32_t t, int idir, int idelta, int j, int jn, double wold,
                          double dold, double lng, const double *pn, const double *hn,
                          const double *sc) {
  const int tid = threadIdx.x, N2 = 2 * S.N, nt = S.nt;
  const uint32_t c3 = 3u + (uint32_t)(idelta - 1);
  Bead bj = bead(S, a, r, j), bn = bead(S, a, r, jn);
  double sn = sc[0];
  double wn = 0.0;
  for (int k = tid; k < N2; k += blockDim.x) {
    int ti = type_of(S, k >> 1);
    double var = 2.0 * S.hbs2m[ti] * a.delta, vari = 1.0 / var;
    double chi = bj.x[k] - m.x[k] - (-var * m.g[k]);
    wn -= chi * chi * vari;
  }
  double wnew = block_sum(wn, m.red);
  double p = 2 * (bj.p[QMC2D_JLTF] - pn[QMC2D_JLTF]) + 0.5 * (wnew - wold);
  p = exp(fmin(0.0, fmax(-50.0, p)));
  if (a.rejection == 0) p = 1.0;
  else if (*bj.age == a.mage) p = 1.0;
  if (*bj.s * sn < 0.0) p = 0.0;
  double wg2 = a.delta * S.npnorm * (bj.p[QMC2D_JKIN0] + pn[QMC2D_JKIN0]);
  double ua = u2(a.seed, 0xFFFFFFFEu, (uint32_t)r, t, c3).x;
  bool rej = p < ua;
  __syncthreads();
  Bead ba = idir == 1 ? bj : bn, bb = idir == 1 ? bn : bj;
  if (rej) {
    if (tid == 0) {
      ba.w[JDTP] = 0.5 * dold;
      ba.w[JBRA] = -a.delta * S.npnorm * (fgg(a, bj.p[QMC2D_JETOT], bj.p[QMC2D_JGG]) - a.etrial);
      bb.w[JITP] = 0.5 * dold;
      ba.w[JLNG] = 0.5 * wg2;
      double nds = 0.0;
      for (int tt = 0; tt < nt; tt++) {
        int ju = QMC2D_JUN(nt, tt);
        double var = 2.0 * S.hbs2m[tt] * a.delta;
        nds -= log(1.0 - exp(-bj.p[ju] * bj.p[ju] / (0.5 * var)));
      }
      ba.w[JNDS] = nds;
      *bn.age = *bj.age + 1.0;
      *bn.s = *bj.s;
      for (int tt = 0; tt < nt; tt++) bn.h[tt] = bj.h[tt];
    }
    for (int k = tid; k < N2; k += blockDim.x) {
      bn.x[k] = bj.x[k];
      bn.g[k] = bj.g[k];
    }
    for (int k = tid; k < S.nprops; k += blockDim.x) bn.p[k] = bj.p[k];
  } else {
    lng += wg2;
    if (tid == 0) {
      ba.w[JDTP] = idir == 1 ? 0.5 * wold : 0.5 * wnew;
      ba.w[JBRA] = -0.5 * a.delta * S.npnorm *
                   ((fgg(a, bj.p[QMC2D_JETOT], bj.p[QMC2D_JGG]) +
                     fgg(a, pn[QMC2D_JETOT], pn[QMC2D_JGG])) -
                    2.0 * a.etrial);
      bb.w[JITP] = idir == 1 ? 0.5 * wnew : 0.5 * wold;
      ba.w[JLNG] = 0.5 * lng;
      double nds = 0.0;
      for (int tt = 0; tt < nt; tt++) {
        int ju = QMC2D_JUN(nt, tt);
        double var = 2.0 * S.hbs2m[tt] * a.delta;
        nds -= log(1.0 - exp(-bj.p[ju] * pn[ju] / (0.5 * var)));
      }
      ba.w[JNDS] = nds;
      *bn.age = 0.0;
      *bn.s = sn;
      for (int tt = 0; tt < nt; tt++) bn.h[tt] = hn[tt];
    }
    for (int k = tid; k < N2; k += blockDim.x) {
      bn.x[k] = m.x[k];
      bn.g[k] = m.g[k];
    }
    for (int k = tid; k < S.nprops; k += blockDim.x) bn.p[k] = pn[k];
  }
  __syncthreads();
  if (tid == 0) bn.p[QMC2D_JACC] = p;
  __syncthreads();
}

// What a reptation move does after its bead growths (reptation_move's path
// part, reptation.f:2105-2160, and reptation_metropolis_test :1865-1895):
// the proposed path's window sums, the action difference, the global test,
// and the block accumulators. pp is scratch; ppo, blk, psum the reptile's
// accepted-path averages, block sums and window sums; sc[1] scratch.
struct PathState {
  int jfirst, jlast;
  double age, norm, nacc;
};
__device__ void path_tail(const DevSys &S, const RmcArgs &a, int r, uint32_t t, int idir,
                          int ndelta, PathState &st, double *pp, double *ppo, double *blk,
                          double *psum, double *sc) {
  const int tid = threadIdx.x, nb = a.nbuf;
  double half = 0.5, one = 0.0, one_nds = 0.0, mezzo = 0.0;
  if (a.wpiu != 0) {
    mezzo = 0.5;
  } else if (a.gstorto != 0) {
    half = 0.0;
    one = 1.0;
    if (a.nodalaction != 0) one_nds = 1.0;
  }
  int &jfirst = st.jfirst, &jlast = st.jlast;
  double &age = st.age, &norm = st.norm, &nacc = st.nacc;
  int kfirst = (jfirst + idir * ndelta + nb) % nb;
  int klast = (jlast + idir * ndelta + nb) % nb;
  path_sums(S, a, r, jfirst, idir * ndelta, psum, pp, (t & 255u) == 0u);
  double wnew = 0.0;
  if (tid == 0) {
    auto P = [&](int j) { return bead(S, a, r, j); };
    wnew = (-P(kfirst).p[QMC2D_JLTF] * (1 + 2 * mezzo) - P(klast).p[QMC2D_JLTF] * (1 - 2 * mezzo) +
            P(jfirst).p[QMC2D_JLTF] * (1 + 2 * mezzo) + P(jlast).p[QMC2D_JLTF] * (1 - 2 * mezzo));
    if (idir == 1) {
      for (int idelta = 1; idelta <= ndelta; idelta++) {
        int j = (jfirst + idir * (idelta - 1) + nb) % nb;
        int jn = (jfirst + idir * idelta + nb) % nb;
        double *wj = P(j).w, *wn = P(jn).w;
        wnew = wnew - wj[JBRA] - wj[JDTP] * (half + mezzo) + wn[JITP] * (one + half + mezzo) -
               wj[JLNG] * one + wj[JNDS] * one_nds;
      }
      for (int idelta = 1; idelta <= ndelta; idelta++) {
        int j = (jlast + idir * (idelta - 1) + nb) % nb;
        int jn = (jlast + idir * idelta + nb) % nb;
        double *wj = P(j).w, *wn = P(jn).w;
        wnew = wnew + wj[JBRA] - wj[JDTP] * (one + half - mezzo) + wn[JITP] * (half - mezzo) +
               wj[JLNG] * one - wj[JNDS] * one_nds;
      }
    } else {
      for (int idelta = 1; idelta <= ndelta; idelta++) {
        int j = (jlast + idir * (idelta - 1) + nb) % nb;
        int jn = (jlast + idir * idelta + nb) % nb;
        double *wj = P(j).w, *wn = P(jn).w;
        wnew = wnew - wn[JBRA] + wn[JDTP] * (one + half - mezzo) - wj[JITP] * (half - mezzo) -
               wn[JLNG] * one + wn[JNDS] * one_nds;
      }
      for (int idelta = 1; idelta <= ndelta; idelta++) {
        int j = (jfirst + idir * (idelta - 1) + nb) % nb;
        int jn = (jfirst + idir * idelta + nb) % nb;
        double *wj = P(j).w, *wn = P(jn).w;
        wnew = wnew + wn[JBRA] + wn[JDTP] * (half + mezzo) - wj[JITP] * (one + half + mezzo) +
               wn[JLNG] * one - wn[JNDS] * one_nds;
      }
    }
    sc[1] = wnew;
  }
  __syncthreads();
  wnew = sc[1];
  // reptation_metropolis_test (reptation.f:1865-1895)
  double p = (age == a.mage_r) ? 1.0 : exp(fmin(0.0, fmax(-50.0, wnew)));
  double ua = u2(a.seed, 0xFFFFFFFDu, (uint32_t)r, t, 2u).x;
  if (p >= ua) {
    const double rc = 1.0 / (a.ntau - 2 * a.ntauskip);
    const double emix =
        0.5 * (bead(S, a, r, klast).p[QMC2D_JETOT] + bead(S, a, r, kfirst).p[QMC2D_JETOT]);
    jfirst = kfirst;
    jlast = klast;
    for (int ip = tid; ip < S.nprops; ip += blockDim.x) {
      psum[ip] = pp[ip];
      ppo[ip] = ip == QMC2D_JETOT ? emix : pp[ip] * rc;
    }
    age = 0.0;
    nacc += 1.0;
  } else {
    age += 1.0;
  }
  __syncthreads();
  for (int ip = tid; ip < S.nprops; ip += blockDim.x) blk[ip] += ppo[ip];
  norm += 1.0;
  __syncthreads();
}

// One CTA per reptile; with kGmat reptile r's determinant matrices take
// walker block r of the handle's device memory (nrep <= capacity).
template <bool kGmat>
__global__ void __launch_bounds__(kThreads, 2) rmc_move_kernel(const DevSys *sp, RmcArgs a) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  EvalSmem m;
  size_t off = eval_carve<kGmat>(S, smem, &m, kGmat ? gmat_block(S, blockIdx.x) : nullptr);
  double *pn = reinterpret_cast<double *>(smem + off);
  double *pp = pn + S.nprops;   // p_p_new
  double *ppo = pp + S.nprops;  // p_p_old
  double *blk = ppo + S.nprops;
  double *psum = blk + S.nprops;  // window sums of the accepted path
  double *hn = psum + S.nprops;
  double *sc = hn + 2;
  const int r = blockIdx.x, tid = threadIdx.x;
  if (r >= a.nrep) return;
  const int N2 = 2 * S.N, nb = a.nbuf;
  for (int ip = tid; ip < S.nprops; ip += blockDim.x) {
    ppo[ip] = a.pp_old[(size_t)r * S.nprops + ip];
    blk[ip] = a.blk[(size_t)r * S.nprops + ip];
    psum[ip] = a.psum[(size_t)r * S.nprops + ip];
  }
  PathState ps{a.ends[2 * r], a.ends[2 * r + 1], a.age[r], a.blk_norm[r], 0.0};
  int status = 0;
  const double pi = 3.141592653589793;
  __syncthreads();
  for (int istp = 0; istp < a.nstp; istp++) {
    const uint32_t t = a.step0 + (uint32_t)istp;
    int idir, ndelta;
    rmc_dir(a, r, t, idir, ndelta);
    const int jstart = idir == 1 ? ps.jlast : ps.jfirst;
    for (int idelta = 1; idelta <= ndelta; idelta++) {
      const int j = (jstart + idir * (idelta - 1) + nb) % nb;
      const int jn = (jstart + idir * idelta + nb) % nb;
      const uint32_t c3 = 3u + (uint32_t)(idelta - 1);
      long long tph = clock64();
      Bead bj = bead(S, a, r, j);
      double ww = 0, wg = 0, dd = 0;
      for (int k = tid; k < N2; k += blockDim.x) {
        int ti = type_of(S, k >> 1);
        double var = 2.0 * S.hbs2m[ti] * a.delta, vari = 1.0 / var;
        double drift = -var * bj.g[k];
        dd += drift * drift * vari;
        double2 u = u2(a.seed, (uint32_t)k, (uint32_t)r, t, c3);
        double chi = cos(pi * u.x) * sqrt(-2.0 * var * log(u.y));
        ww -= chi * chi * vari;
        m.x[k] = chi + drift + bj.x[k];
        wg -= (chi + drift) * (chi + drift) * vari;
      }
      double wold = block_sum(ww, m.red), dold = block_sum(dd, m.red);
      double lng = block_sum(wg, m.red);
      phase_mark(S, PH_PROPOSE, tph);
      status |= eval_walker<double, kGmat>(S, m, hn, pn, sc, tph);
      bead_tail(S, a, m, r, t, idir, idelta, j, jn, wold, dold, lng, pn, hn, sc);
      phase_mark(S, PH_ACCEPT, tph);
    }
    long long tpp = clock64();
    path_tail(S, a, r, t, idir, ndelta, ps, pp, ppo, blk, psum, sc);
    phase_mark(S, PH_PATH, tpp);
  }
  for (int ip = tid; ip < S.nprops; ip += blockDim.x) {
    a.pp_old[(size_t)r * S.nprops + ip] = ppo[ip];
    a.blk[(size_t)r * S.nprops + ip] = blk[ip];
    a.psum[(size_t)r * S.nprops + ip] = psum[ip];
  }
  if (tid == 0) {
    a.ends[2 * r] = ps.jfirst;
    a.ends[2 * r + 1] = ps.jlast;
    a.age[r] = ps.age;
    a.blk_norm[r] = ps.norm;
    a.cnt[4 * r] += ps.nacc;
    a.cnt[4 * r + 1] += a.nstp;
    a.status[r] |= status;
  }
}

// ------------------------------------------------ split bead growth
// The same move as rmc_move_kernel in two launches per bead growth, as a
// VMC/DMC move is: rmc_pairs_kernel draws the growing end's new bead and
// runs the pair passes (u2, u3, backflow, v2) and rho_k into the reptile's
// move scratch, with the pair rows staged in shared memory and G reptiles
// per CTA; rmc_det_kernel evaluates the determinants from the scratch (the
// backflow pair values stored by the pair passes), runs the bead's tail
// and, after the reptile's last growth of the move, the path tail. A move
// of mdelta > 1 takes mdelta launch pairs; a reptile whose move has fewer
// growths skips the later ones.
template <class R, int G, int LG>
__global__ void __launch_bounds__(G * kThreads, 2 / G) rmc_pairs_kernel(const DevSys *sp,
                                                                        RmcArgs a, double *scr,
                                                                        int idelta,
                                                                        int stage_rows) {
  constexpr int kPairThreads = G * kThreads;
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  const size_t carve = (pair_carve(S, nullptr, nullptr, kThreads) + 127) & ~size_t(127);
  const int grp = threadIdx.x / kThreads, tid = threadIdx.x - grp * kThreads;
  EvalSmem m;
  pair_carve(S, smem + grp * carve, &m, kThreads);
  const R *rows_g = pair_rows<R>(S);
  R *rows_s = reinterpret_cast<R *>(smem + G * carve);
  if (stage_rows) {  // the first copy16 16-byte parts of each global row
    using Lay = RowLayout<R>;
    constexpr int V = Lay::copy16, VG = Lay::gstride * (int)sizeof(R) / 16;
    const int nrow = S.cmb_nblk * (S.cmb_ng + 1);
    const float4 *src = reinterpret_cast<const float4 *>(rows_g);
    for (int e = threadIdx.x; e < nrow * V; e += kPairThreads) {
      const int rr = e / V, q = e - rr * V;
      reinterpret_cast<float4 *>(rows_s + (size_t)rr * Lay::sstride)[q] =
          __ldg(src + (size_t)rr * VG + q);
    }
  }
  __syncthreads();
  const GroupSync sync{1 + grp, kThreads};
  const int N = S.N, N2 = 2 * N, nb = a.nbuf;
  const uint32_t t = a.step0;
  const double pi = 3.141592653589793;
  const MoveScratch L = move_scratch(S, false);
  for (int r = blockIdx.x * G + grp; r < a.nrep; r += gridDim.x * G) {
    int idir, ndelta;
    rmc_dir(a, r, t, idir, ndelta);
    if (idelta > ndelta) continue;  // the whole group: r is the group's
    long long tph = clock64();
    const int jstart = idir == 1 ? a.ends[2 * r + 1] : a.ends[2 * r];
    const int j = (jstart + idir * (idelta - 1) + nb) % nb;
    const uint32_t c3 = 3u + (uint32_t)(idelta - 1);
    Bead bj = bead(S, a, r, j);
    double ww = 0, wg = 0, dd = 0;
    for (int k = tid; k < N2; k += kThreads) {
      int ti = type_of(S, k >> 1);
      double var = 2.0 * S.hbs2m[ti] * a.delta, vari = 1.0 / var;
      double drift = -var * bj.g[k];
      dd += drift * drift * vari;
      double2 u = u2(a.seed, (uint32_t)k, (uint32_t)r, t, c3);
      double chi = cos(pi * u.x) * sqrt(-2.0 * var * log(u.y));
      ww -= chi * chi * vari;
      m.x[k] = chi + drift + bj.x[k];
      wg -= (chi + drift) * (chi + drift) * vari;
    }
    const double wold = block_sum_t<kThreads>(ww, m.red, sync, tid);
    const double dold = block_sum_t<kThreads>(dd, m.red, sync, tid);
    const double lng = block_sum_t<kThreads>(wg, m.red, sync, tid);
    phase_mark(S, PH_PROPOSE, tph, tid == 0);
    double *o = scr + (size_t)r * L.stride;
    double *pout = (S.has_bf && !S.bf_zero) ? o + L.pair : nullptr;
    if (stage_rows)
      eval_pairs<kThreads, true, R, GroupSync, LG>(S, m, tph, pout, (const R *)rows_s, sync,
                                                   tid);
    else
      eval_pairs<kThreads, false, R, GroupSync, LG>(S, m, tph, pout, rows_g, sync, tid);
    pair_rhok<LG>(S, m, tid, kThreads, sync);
    sync();
    for (int e = tid; e < 4 * S.nk; e += kThreads) o[L.rhok + e] = m.rhok[e];
    for (int e = tid; e < N2; e += kThreads) {
      o[L.x + e] = m.x[e];
      o[L.g + e] = m.g[e];
      o[L.q + e] = m.q[e];
      o[L.qbd + e] = m.qbd[e];
    }
    for (int e = tid; e < 3 * N; e += kThreads) o[L.sb + e] = m.Sb[e];
    for (int e = tid; e < N; e += kThreads) {
      o[L.lap + e] = m.lap[e];
      o[L.ltf + e] = m.ltf[e];
      o[L.vp + e] = m.vp[e];
    }
    if (tid == 0) {
      o[L.wold] = wold;
      o[L.dold] = dold;
      o[L.lng] = lng;
    }
    sync();  // m is reused by the group's next reptile
  }
}

template <bool kGmat>
__global__ void __launch_bounds__(kThreads, 2) rmc_det_kernel(const DevSys *sp, RmcArgs a,
                                                              const double *scr, int idelta) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  EvalSmem m;
  size_t off = eval_carve<kGmat>(S, smem, &m, kGmat ? gmat_block(S, blockIdx.x) : nullptr);
  double *pn = reinterpret_cast<double *>(smem + off);
  double *pp = pn + S.nprops;
  double *ppo = pp + S.nprops;
  double *blk = ppo + S.nprops;
  double *psum = blk + S.nprops;
  double *hn = psum + S.nprops;
  double *sc = hn + 2;
  const int r = blockIdx.x, tid = threadIdx.x;
  if (r >= a.nrep) return;
  const uint32_t t = a.step0;
  int idir, ndelta;
  rmc_dir(a, r, t, idir, ndelta);
  if (idelta > ndelta) return;  // the whole CTA
  const int N = S.N, N2 = 2 * N, nb = a.nbuf;
  const MoveScratch L = move_scratch(S, false);
  const double *o = scr + (size_t)r * L.stride;
  const bool pairs_stored = S.has_bf && !S.bf_zero;
  if (pairs_stored) {
    // bring the stored pair values back into L2 before the Jacobian build
    const size_t bytes = (sizeof(double) * 3 * pair_count(N)) & ~size_t(15);
    const char *base = reinterpret_cast<const char *>(o + L.pair);
    for (size_t b0 = (size_t)tid * 32768; b0 < bytes; b0 += (size_t)kThreads * 32768) {
      const unsigned sz = (unsigned)(bytes - b0 < 32768 ? bytes - b0 : 32768);
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + b0), "r"(sz)
                   : "memory");
    }
  }
  for (int e = tid; e < N2; e += kThreads) {
    m.x[e] = o[L.x + e];
    m.g[e] = o[L.g + e];
    m.q[e] = o[L.q + e];
    m.qbd[e] = o[L.qbd + e];
    m.gd[e] = 0.0;
  }
  for (int e = tid; e < 3 * N; e += kThreads) m.Sb[e] = o[L.sb + e];
  for (int e = tid; e < N; e += kThreads) {
    m.lap[e] = o[L.lap + e];
    m.ltf[e] = o[L.ltf + e];
    m.vp[e] = o[L.vp + e];
    m.lapd[e] = 0.0;
    m.ph2[e] = 0.0;
    m.ph2d[e] = 0.0;
  }
  const double wold = o[L.wold], dold = o[L.dold], lng = o[L.lng];
  __syncthreads();
  long long tph = clock64();
  const int status = eval_det<kGmat>(S, m, hn, pn, sc, tph, pairs_stored ? o + L.pair : nullptr,
                                     o + L.rhok);
  const int jstart = idir == 1 ? a.ends[2 * r + 1] : a.ends[2 * r];
  const int j = (jstart + idir * (idelta - 1) + nb) % nb;
  const int jn = (jstart + idir * idelta + nb) % nb;
  bead_tail(S, a, m, r, t, idir, idelta, j, jn, wold, dold, lng, pn, hn, sc);
  phase_mark(S, PH_ACCEPT, tph);
  if (tid == 0 && status) atomicOr(&a.status[r], status);
  if (idelta < ndelta) return;  // the whole CTA
  // the move's end, with the reptile's state from and back to device memory
  long long tpp = clock64();
  for (int ip = tid; ip < S.nprops; ip += blockDim.x) {
    ppo[ip] = a.pp_old[(size_t)r * S.nprops + ip];
    blk[ip] = a.blk[(size_t)r * S.nprops + ip];
    psum[ip] = a.psum[(size_t)r * S.nprops + ip];
  }
  PathState ps{a.ends[2 * r], a.ends[2 * r + 1], a.age[r], a.blk_norm[r], 0.0};
  __syncthreads();
  path_tail(S, a, r, t, idir, ndelta, ps, pp, ppo, blk, psum, sc);
  for (int ip = tid; ip < S.nprops; ip += blockDim.x) {
    a.pp_old[(size_t)r * S.nprops + ip] = ppo[ip];
    a.blk[(size_t)r * S.nprops + ip] = blk[ip];
    a.psum[(size_t)r * S.nprops + ip] = psum[ip];
  }
  if (tid == 0) {
    a.ends[2 * r] = ps.jfirst;
    a.ends[2 * r + 1] = ps.jlast;
    a.age[r] = ps.age;
    a.blk_norm[r] = ps.norm;
    a.cnt[4 * r] += ps.nacc;
    a.cnt[4 * r + 1] += 1.0;
  }
  phase_mark(S, PH_PATH, tpp);
}

// The path estimators of path_props (reptation.f:1578-1737) of reptile r's
// current path into rows[r * e.nvalues ..]: one CTA per reptile; every
// output bin is summed by one thread in the reference's order (bead itau
// ascending, then particles, then dimensions), so the result does not
// depend on the thread count. cm: ncmass * ntau * 2 doubles of shared
// memory, the centre of mass of each record's type in every bead (the
// cmass_p properties of compute_properties, reptation.f:2696-2707).
__global__ void __launch_bounds__(kThreads) rmc_estimators_kernel(const DevSys *sp, RmcArgs a,
                                                                  qmc2d_rmc_estimators e,
                                                                  double *rows) {
  __shared__ DevSys S;
  extern __shared__ double cm[];
  load_sys(S, sp);
  const int r = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
  if (r >= a.nrep) return;
  const int kfirst = a.ends[2 * r], ntau = a.ntau, nb = ntau - 2 * a.ntauskip;
  double *row = rows + (size_t)r * e.nvalues;
  auto xb = [&](int itau) { return bead(S, a, r, (kfirst + itau - 1) % a.nbuf).x; };
  auto pb = [&](int itau) { return bead(S, a, r, (kfirst + itau - 1) % a.nbuf).p; };
  const double pi = 3.141592653589793;
  for (int item = tid; item < e.ncmass * ntau * 2; item += nth) {
    const int c = item / (ntau * 2), itau = (item % (ntau * 2)) / 2 + 1, d = item & 1;
    const int t = e.cmass_type[c];
    const double *x = xb(itau);
    double sum = 0.0;
    for (int ip = S.ipfrst[t]; ip < S.ipfrst[t] + S.np[t]; ip++) sum += x[2 * ip + d];
    cm[item] = sum / S.np[t];
  }
  __syncthreads();
  // cmass z: the middle bead (itau = ntau/2 + 1)
  for (int item = tid; item < e.ncmass * 2; item += nth) {
    const int c = item / 2, d = item & 1, t = e.cmass_type[c];
    const double v = cm[(c * ntau + ntau / 2) * 2 + d] * (2.0 * pi * S.eli[d]) * S.np[t];
    row[e.jcmass_z + 4 * c + 2 * d] = cos(v);
    row[e.jcmass_z + 4 * c + 2 * d + 1] = sin(v);
  }
  // cmass diffusion
  int off = e.jcmass_d;
  for (int c = 0; c < e.ncmass; c++)
    for (int k = 0; k < e.cmass_nskip; k++) {
      const int skip = e.cmass_ntauskip[c][k], ts = e.cmass_tau_skip[c];
      const int nij = (ntau - 2 * skip) / ts;
      for (int ij = tid; ij < nij; ij += nth) {
        double re = 0.0, nrm = 0.0;
        for (int itau = 1 + skip; itau + ij * ts <= ntau - skip; itau++) {
          const int jtau = itau + ij * ts;
          for (int d = 0; d < 2; d++) {
            const double df = cm[(c * ntau + itau - 1) * 2 + d] - cm[(c * ntau + jtau - 1) * 2 + d];
            re += df * df;
          }
          nrm += 1.0;
        }
        row[off + ij] = re / nrm;
      }
      off += nij;
    }
  // mstar
  off = e.jmstar;
  for (int i = 0; i < e.nmstar; i++) {
    const int t = e.mstar_type[i], ts = e.mstar_tau_skip[i], nij = nb / ts;
    for (int ij = tid; ij < nij; ij += nth) {
      double re = 0.0, nrm = 0.0;
      for (int itau = 1 + a.ntauskip; itau + ij * ts <= ntau - a.ntauskip; itau++) {
        const double *xi = xb(itau), *xj = xb(itau + ij * ts);
        for (int ip = S.ipfrst[t]; ip < S.ipfrst[t] + S.np[t]; ip++) {
          for (int d = 0; d < 2; d++) {
            const double df = xi[2 * ip + d] - xj[2 * ip + d];
            re += df * df;
          }
          nrm += 1.0;
        }
      }
      row[off + ij] = re / nrm;
    }
    off += nij;
  }
  // itc
  off = e.jitc;
  for (int i = 0; i < e.nitc; i++) {
    const int ts = e.itc_tau_skip[i], nij = nb / ts, cplx = e.itc_complex[i] != 0;
    const int nc = cplx ? e.itc_count[i] / 2 : e.itc_count[i];
    for (int item = tid; item < nc * nij; item += nth) {
      const int q = item / nij, ij = item - q * nij;
      const int ic = cplx ? 2 * q : q;  // 0-based icount
      double re = 0.0, im = 0.0, nrm = 0.0;
      for (int itau = 1 + a.ntauskip; itau + ij * ts <= ntau - a.ntauskip; itau++) {
        const double *p1 = pb(itau), *p2 = pb(itau + ij * ts);
        double ri = 0.0, ii = 0.0, rj = 0.0, ij2 = 0.0;
        for (int s2 = 0; s2 < e.itc_add[i]; s2++) {
          ri += p1[e.itc_start[i][s2] + ic];
          if (cplx) ii += p1[e.itc_start[i][s2] + ic + 1];
        }
        for (int s2 = 0; s2 < e.jtc_add[i]; s2++) {
          rj += p2[e.jtc_start[i][s2] + ic];
          if (cplx) ij2 += p2[e.jtc_start[i][s2] + ic + 1];
        }
        if (cplx) {
          ii *= e.itc_complex[i];
          ij2 *= e.jtc_complex[i];
          re += ri * rj - ii * ij2;
          im += ri * ij2 + ii * rj;
        } else {
          re += ri * rj;
        }
        nrm += 1.0;
      }
      if (cplx) {
        row[off + 2 * q * nij + ij] = re / nrm;
        row[off + 2 * q * nij + nij + ij] = im / nrm;
      } else {
        row[off + q * nij + ij] = re / nrm;
      }
    }
    off += nij * e.itc_count[i];
  }
}

// out[v] = the mean over reptiles of rows[r * nv + v], summed in reptile order.
__global__ void rmc_estimators_mean_kernel(const double *rows, int nrep, int nv, double *out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double s = 0.0;
  for (int r = 0; r < nrep; r++) s += rows[(size_t)r * nv + v];
  out[v] = s / nrep;
}

}  // namespace

void rmc_free(RmcState *r) {
  void *b[] = {r->x,    r->g,      r->p,    r->h,   r->s,   r->age_stack, r->w,
               r->ends, r->pp_old, r->psum, r->age, r->est};
  for (void *p : b) cudaFree(p);
  *r = RmcState{};
}

}  // namespace q2d

// ----------------------------------------------------------------- C-ABI
#include <string>
#include <vector>

#include "handle.h"

namespace {

int rfail(cudaError_t e, const char *what) {
  q2d::set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return QMC2D_ERR_CUDA;
}

#define RCK(call)                                   \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return rfail(e_, #call); \
  } while (0)

q2d::RmcArgs rmc_args(qmc2d_handle *h, int nstp) {
  q2d::RmcState &r = h->rmc;
  q2d::RmcArgs a{};
  a.nrep = r.nrep;
  a.ntau = r.ntau;
  a.ntauskip = r.ntauskip;
  a.mdelta = r.mdelta;
  a.nbuf = r.nbuf;
  a.nstp = nstp;
  a.delta = r.delta;
  a.etrial = r.etrial;
  a.mage = r.mage;
  a.mage_r = r.mage_r;
  a.seed = h->seed;
  a.step0 = r.step;
  a.ecut = h->hs.ecut;
  a.value_ecut = h->hs.value_ecut;
  a.rejection = h->hs.rejection;
  a.wpiu = h->hs.wpiu;
  a.gstorto = h->hs.gstorto;
  a.nodalaction = h->hs.nodalaction;
  a.x = r.x;
  a.g = r.g;
  a.p = r.p;
  a.h = r.h;
  a.s = r.s;
  a.age_stack = r.age_stack;
  a.w = r.w;
  a.pp_old = r.pp_old;
  a.psum = r.psum;
  a.age = r.age;
  a.ends = r.ends;
  a.blk = h->d_blk;
  a.blk_norm = h->d_norm;
  a.cnt = h->d_cnt;
  a.status = h->d_status;
  return a;
}

size_t rmc_move_smem(const q2d::DevSys &s) {
  return q2d::eval_carve(s, nullptr, nullptr) + sizeof(double) * (5 * (size_t)s.nprops + 16);
}

}  // namespace

extern "C" int qmc2d_rmc_init(qmc2d_handle *h, int nrep, const qmc2d_rmc_params *prm,
                              const double *x) {
  if (!h || !prm || !x || nrep <= 0 || nrep > h->cap || prm->ntau < 2 || prm->mdelta < 1 ||
      prm->ntau - 2 * prm->ntauskip < 1 || !(prm->delta > 0.0)) {
    q2d::set_error("qmc2d_rmc_init: bad argument");
    return QMC2D_ERR_ARG;
  }
  RCK(cudaSetDevice(h->device));
  RCK(join_side(h));
  RCK(cudaStreamSynchronize(h->stream));
  const int split = h->rmc.split;  // a launch choice: kept across set-ups
  q2d::rmc_free(&h->rmc);
  q2d::RmcState &r = h->rmc;
  r.split = split;
  r.nrep = nrep;
  r.ntau = prm->ntau;
  r.ntauskip = prm->ntauskip;
  r.mdelta = prm->mdelta;
  r.nbuf = prm->ntau + prm->mdelta;
  r.delta = prm->delta;
  r.etrial = prm->etrial;
  r.mage = prm->mage;
  r.mage_r = prm->mage_r;
  r.step = 0;
  size_t nb = (size_t)nrep * r.nbuf;
  int N = h->N, nt = h->nt, np = h->nprops;
  RCK(cudaMalloc(&r.x, sizeof(double) * nb * 2 * N));
  RCK(cudaMalloc(&r.g, sizeof(double) * nb * 2 * N));
  RCK(cudaMalloc(&r.p, sizeof(double) * nb * np));
  RCK(cudaMalloc(&r.h, sizeof(double) * nb * nt));
  RCK(cudaMalloc(&r.s, sizeof(double) * nb));
  RCK(cudaMalloc(&r.age_stack, sizeof(double) * nb));
  RCK(cudaMalloc(&r.w, sizeof(double) * nb * 5));
  RCK(cudaMalloc(&r.ends, sizeof(int) * 2 * nrep));
  RCK(cudaMalloc(&r.pp_old, sizeof(double) * nrep * np));
  RCK(cudaMalloc(&r.psum, sizeof(double) * nrep * np));
  RCK(cudaMalloc(&r.age, sizeof(double) * nrep));
  RCK(cudaMemsetAsync(r.w, 0, sizeof(double) * nb * 5, h->stream));
  RCK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->cap, h->stream));
  double *dx = nullptr;
  size_t nx = (size_t)nrep * r.ntau * 2 * N;
  RCK(cudaMalloc(&dx, sizeof(double) * nx));
  RCK(cudaMemcpyAsync(dx, x, sizeof(double) * nx, cudaMemcpyHostToDevice, h->stream));
  q2d::RmcArgs a = rmc_args(h, 0);
  size_t sm = q2d::eval_smem_bytes(h->hs);
  const void *kb = h->hs.gmat ? (const void *)q2d::rmc_eval_beads_kernel<true>
                              : (const void *)q2d::rmc_eval_beads_kernel<false>;
  RCK(q2d::raise_smem_limit(kb, sm));
  // with determinants in device memory a launch covers at most `capacity`
  // beads, one walker block each
  const int total = nrep * r.ntau, chunk = h->hs.gmat ? h->cap : total;
  for (int b0 = 0; b0 < total; b0 += chunk) {
    const int nb = total - b0 < chunk ? total - b0 : chunk;
    if (h->hs.gmat)
      q2d::rmc_eval_beads_kernel<true><<<nb, q2d::kThreads, sm, h->stream>>>(h->ds, a, dx, b0);
    else
      q2d::rmc_eval_beads_kernel<false><<<nb, q2d::kThreads, sm, h->stream>>>(h->ds, a, dx, b0);
    RCK(cudaGetLastError());
  }
  q2d::rmc_init_kernel<<<nrep, q2d::kThreads, sizeof(double) * np, h->stream>>>(h->ds, a);
  RCK(cudaGetLastError());
  RCK(cudaStreamSynchronize(h->stream));
  cudaFree(dx);
  h->nw = 0;
  return q2d_sync_status(h, nrep);
}

template <int G, int LG>
static cudaError_t launch_rmc_pairs_t(const q2d::DevSys &hs, const q2d::DevSys *ds,
                                      const q2d::RmcArgs &a, double *scr, int idelta,
                                      cudaStream_t st) {
  int dev = 0, nsm = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
      cudaSuccess)
    return e;
  const void *k = (const void *)q2d::rmc_pairs_kernel<double, G, LG>;
  const size_t carve =
      G * ((q2d::pair_carve(hs, nullptr, nullptr, q2d::kThreads) + 127) & ~size_t(127));
  const size_t rows = sizeof(double) * q2d::RowLayout<double>::sstride * (size_t)hs.cmb_nblk *
                      (hs.cmb_ng + 1);
  const int stage =
      hs.tune_stage != 1 && carve + rows + sizeof(q2d::DevSys) <= (size_t)optin ? 1 : 0;
  const size_t sm = carve + (stage ? rows : 0);
  if ((e = q2d::raise_smem_limit(k, sm)) != cudaSuccess) return e;
  int per_sm = 1;
  if (G == 1 && (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G * q2d::kThreads,
                                                                   sm)) != cudaSuccess)
    return e;
  const int need = (a.nrep + G - 1) / G, cap = nsm * (per_sm > 0 ? per_sm : 1);
  q2d::rmc_pairs_kernel<double, G, LG>
      <<<need < cap ? need : cap, G * q2d::kThreads, sm, st>>>(ds, a, scr, idelta, stage);
  return cudaGetLastError();
}

// the lanes per particle in force (DevSys::tune_lanes, as the DMC pair kernel)
template <int G>
static cudaError_t launch_rmc_pairs(const q2d::DevSys &hs, const q2d::DevSys *ds,
                                    const q2d::RmcArgs &a, double *scr, int idelta,
                                    cudaStream_t st) {
  switch (hs.tune_lanes) {
    case 4: return launch_rmc_pairs_t<G, 4>(hs, ds, a, scr, idelta, st);
    case 16: return launch_rmc_pairs_t<G, 16>(hs, ds, a, scr, idelta, st);
    default: return launch_rmc_pairs_t<G, 8>(hs, ds, a, scr, idelta, st);
  }
}

extern "C" int qmc2d_rmc(qmc2d_handle *h, int nstp) {
  if (!h || nstp < 0) return QMC2D_ERR_ARG;
  if (h->rmc.nrep <= 0) {
    q2d::set_error("qmc2d_rmc: no reptiles (call qmc2d_rmc_init)");
    return QMC2D_ERR_STACK;
  }
  if (nstp == 0) return QMC2D_OK;
  RCK(cudaSetDevice(h->device));
  RCK(join_side(h));
  RCK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->rmc.nrep, h->stream));
  q2d::RmcArgs a = rmc_args(h, nstp);
  size_t sm = rmc_move_smem(h->hs);
  if (!h->rmc.split) {
    const void *km = h->hs.gmat ? (const void *)q2d::rmc_move_kernel<true>
                                : (const void *)q2d::rmc_move_kernel<false>;
    RCK(q2d::raise_smem_limit(km, sm));
    ProfScope ps(h, QMC2D_KERNEL_RMC, h->stream);
    if (h->hs.gmat)
      q2d::rmc_move_kernel<true><<<h->rmc.nrep, q2d::kThreads, sm, h->stream>>>(h->ds, a);
    else
      q2d::rmc_move_kernel<false><<<h->rmc.nrep, q2d::kThreads, sm, h->stream>>>(h->ds, a);
    RCK(cudaGetLastError());
  } else {
    // per move and bead growth: the pair passes, then the rest
    const void *kd = h->hs.gmat ? (const void *)q2d::rmc_det_kernel<true>
                                : (const void *)q2d::rmc_det_kernel<false>;
    RCK(q2d::raise_smem_limit(kd, sm));
    for (int istp = 0; istp < nstp; istp++) {
      a.step0 = h->rmc.step + (uint32_t)istp;
      for (int idelta = 1; idelta <= h->rmc.mdelta; idelta++) {
        {
          ProfScope ps(h, QMC2D_KERNEL_PAIRS, h->stream);
          RCK(h->hs.tune_groups == 1
                  ? launch_rmc_pairs<1>(h->hs, h->ds, a, h->d_mscr, idelta, h->stream)
                  : launch_rmc_pairs<2>(h->hs, h->ds, a, h->d_mscr, idelta, h->stream));
        }
        ProfScope ps(h, QMC2D_KERNEL_RMC, h->stream);
        if (h->hs.gmat)
          q2d::rmc_det_kernel<true>
              <<<h->rmc.nrep, q2d::kThreads, sm, h->stream>>>(h->ds, a, h->d_mscr, idelta);
        else
          q2d::rmc_det_kernel<false>
              <<<h->rmc.nrep, q2d::kThreads, sm, h->stream>>>(h->ds, a, h->d_mscr, idelta);
        RCK(cudaGetLastError());
      }
    }
  }
  h->rmc.step += (uint32_t)nstp;
  return q2d_sync_status(h, h->rmc.nrep);
}

extern "C" int qmc2d_rmc_set_launch(qmc2d_handle *h, int split) {
  if (!h || split < 0 || split > 1) {
    q2d::set_error("qmc2d_rmc_set_launch: bad argument");
    return QMC2D_ERR_ARG;
  }
  h->rmc.split = split;
  return QMC2D_OK;
}

extern "C" int qmc2d_rmc_get_path(qmc2d_handle *h, int rep, double *x, double *props) {
  if (!h || rep < 0 || rep >= h->rmc.nrep) return QMC2D_ERR_ARG;
  RCK(cudaSetDevice(h->device));
  RCK(join_side(h));
  RCK(cudaStreamSynchronize(h->stream));
  q2d::RmcState &r = h->rmc;
  int ends[2];
  RCK(cudaMemcpy(ends, r.ends + 2 * rep, sizeof(int) * 2, cudaMemcpyDeviceToHost));
  size_t N2 = 2 * (size_t)h->N, np = h->nprops;
  for (int i = 0; i < r.ntau; i++) {
    size_t b = (size_t)rep * r.nbuf + (ends[0] + i) % r.nbuf;
    if (x) RCK(cudaMemcpy(x + i * N2, r.x + b * N2, sizeof(double) * N2, cudaMemcpyDeviceToHost));
    if (props)
      RCK(cudaMemcpy(props + i * np, r.p + b * np, sizeof(double) * np, cudaMemcpyDeviceToHost));
  }
  return QMC2D_OK;
}

extern "C" int qmc2d_rmc_path_estimators(qmc2d_handle *h, const qmc2d_rmc_estimators *est,
                                         double *out) {
  if (!h || !est || !out || est->nvalues < 0) return QMC2D_ERR_ARG;
  q2d::RmcState &r = h->rmc;
  if (r.nrep <= 0) {
    q2d::set_error("qmc2d_rmc_path_estimators: no reptiles (call qmc2d_rmc_init)");
    return QMC2D_ERR_STACK;
  }
  if (est->ntau != r.ntau || est->ntauskip != r.ntauskip || est->ncmass > QMC2D_MAX_EST ||
      est->nmstar > QMC2D_MAX_EST || est->nitc > QMC2D_MAX_EST) {
    q2d::set_error("qmc2d_rmc_path_estimators: set up for another path length");
    return QMC2D_ERR_ARG;
  }
  if (est->nvalues == 0) return QMC2D_OK;
  RCK(cudaSetDevice(h->device));
  RCK(join_side(h));
  const size_t need = ((size_t)r.nrep + 1) * est->nvalues;
  if (need > r.est_cap) {
    RCK(cudaStreamSynchronize(h->stream));
    cudaFree(r.est);
    r.est = nullptr;
    r.est_cap = 0;
    RCK(cudaMalloc(&r.est, sizeof(double) * need));
    r.est_cap = need;
  }
  q2d::RmcArgs a = rmc_args(h, 0);
  const size_t sm = sizeof(double) * 2 * (size_t)r.ntau * est->ncmass;
  RCK(q2d::raise_smem_limit((const void *)q2d::rmc_estimators_kernel, sm));
  q2d::rmc_estimators_kernel<<<r.nrep, q2d::kThreads, sm, h->stream>>>(h->ds, a, *est, r.est);
  RCK(cudaGetLastError());
  double *mean = r.est + (size_t)r.nrep * est->nvalues;
  q2d::rmc_estimators_mean_kernel<<<(est->nvalues + 255) / 256, 256, 0, h->stream>>>(
      r.est, r.nrep, est->nvalues, mean);
  RCK(cudaGetLastError());
  RCK(cudaMemcpyAsync(out, mean, sizeof(double) * est->nvalues, cudaMemcpyDeviceToHost,
                      h->stream));
  RCK(cudaStreamSynchronize(h->stream));
  return QMC2D_OK;
}
