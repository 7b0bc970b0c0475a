// kernels.cu - walker kernels for sm_100a: batched evaluation
// (compute_properties), the VMC/DMC move in two launches (move + the pair
// passes of compute_properties; the rest of compute_properties +
// metropolis_test + averages(2), reptation.f:4617, 2661, 2622, 4275), the
// fixed-population comb of branch2 (reptation.f:2162) and the slot gather
// that replaces its send/receive/prov_dest copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"
#include "walker_eval.cuh"

namespace q2d {

// ------------------------------------------------------------------ Philox
// Philox4x32-10 (Salmon et al., SC'11): 10 rounds, Weyl key schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
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

// 53 random bits, offset by half an ulp: u in (0,1).
__device__ __forceinline__ double open01(uint32_t a, uint32_t b) {
  unsigned long long k = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
  return ((double)k + 0.5) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double2 uniform2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
                                            uint32_t c3) {
  uint4 o = philox4x32_10(make_uint4(c0, c1, c2, c3),
                          make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  return make_double2(open01(o.x, o.y), open01(o.z, o.w));
}

__device__ __forceinline__ void load_sys(DevSys &S, const DevSys *sp) {
  const int *src = reinterpret_cast<const int *>(sp);
  int *dst = reinterpret_cast<int *>(&S);
  for (int i = threadIdx.x; i < (int)(sizeof(DevSys) / sizeof(int)); i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
}

// ---------------------------------------------------------------- eval
template <class R, bool kGmat>
__global__ void __launch_bounds__(kThreads, 2) eval_kernel(const DevSys *sp, int nw,
                                                        const double *__restrict__ x, double *g,
                                                        double *hl, double *props, double *s,
                                                        int *status) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  EvalSmem m;
  size_t off = eval_carve<kGmat>(S, smem, &m, kGmat ? gmat_block(S, blockIdx.x) : nullptr);
  double *pn = reinterpret_cast<double *>(smem + off);
  double *hn = pn + S.nprops;
  double *sn = hn + 2;
  const int w = blockIdx.x;
  if (w >= nw) return;
  const int N2 = 2 * S.N;
  for (int j = threadIdx.x; j < N2; j += blockDim.x) m.x[j] = x[(size_t)w * N2 + j];
  __syncthreads();
  long long tph = clock64();
  int st = eval_walker<R, kGmat>(S, m, hn, pn, sn, tph);
  for (int j = threadIdx.x; j < N2; j += blockDim.x) g[(size_t)w * N2 + j] = m.g[j];
  for (int j = threadIdx.x; j < S.nprops; j += blockDim.x)
    props[(size_t)w * S.nprops + j] = pn[j];
  if (threadIdx.x == 0) {
    for (int t = 0; t < S.nt; t++) hl[(size_t)w * S.nt + t] = hn[t];
    s[w] = *sn;
    status[w] = st;
  }
}

size_t eval_smem_bytes(const DevSys &s) {
  return eval_carve(s, nullptr, nullptr) + align16(sizeof(double) * (s.nprops + 3));
}

size_t gmat_doubles(const DevSys &s) {
  if (!s.gmat) return 0;
  size_t g = 0;
  eval_carve(s, nullptr, nullptr, nullptr, &g);
  return ((g + 7) / 8 + 31) & ~size_t(31);
}

// ------------------------------------------------------------- the move
// Walker state kept in shared memory across the CTA's steps.
struct MoveSmem {
  double *xo, *go, *po, *pn, *blk, *ho, *hn, *sc;
};

// props_in_buf (the one-buffer move kernel): the new properties pn go to the
// orbital buffer, which is free once the determinants are done
// (props_buf_fits); the old ones and the block sums stay in HBM.
__host__ __device__ inline size_t move_carve(const DevSys &s, char *base, MoveSmem *m,
                                             bool props_in_buf = false) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base ? base + off : nullptr;
    off += align16(bytes);
    return p;
  };
  MoveSmem t;
  t.xo = (double *)take(sizeof(double) * 2 * s.N);
  t.go = (double *)take(sizeof(double) * 2 * s.N);
  t.po = t.pn = t.blk = nullptr;
  if (!props_in_buf) {
    t.po = (double *)take(sizeof(double) * s.nprops);
    t.pn = (double *)take(sizeof(double) * s.nprops);
    t.blk = (double *)take(sizeof(double) * s.nprops);
  }
  t.ho = (double *)take(sizeof(double) * 2);
  t.hn = (double *)take(sizeof(double) * 2);
  t.sc = (double *)take(sizeof(double) * 8);
  if (m) *m = t;
  return off;
}

size_t move_smem_bytes(const DevSys &s) {
  return eval_carve(s, nullptr, nullptr) + move_carve(s, nullptr, nullptr);
}

// The one-buffer move kernel (move_kernel<false, true>): both spins'
// orbitals and inverses come from orb_inv_kernel and take one shared
// buffer in turn, the new properties use that buffer after the
// determinants, and the old properties and block sums are read from HBM at
// the write-back, so three CTAs fit an SM.
inline bool props_buf_fits(const DevSys &s) {
  const int n = s.nmax > 0 ? s.nmax : 1;
  const size_t awbytes = sizeof(double2) * (n * n + n * ws_ld(n));
  const size_t mbytes = sizeof(double) * 2 * n * xt_ldm(2 * n);
  return sizeof(double) * (size_t)s.nprops <= std::max(awbytes, mbytes);
}
size_t move_smem_bytes_seq(const DevSys &s) {
  return eval_carve(s, nullptr, nullptr, nullptr, nullptr, true) +
         move_carve(s, nullptr, nullptr, true);
}

// One move of one walker is two launches. pairs_kernel: the proposal
// (move, reptation.f:4631-4646) and the pair passes, written to the
// walker's MoveScratch block. move_kernel: the rest of the evaluation, the
// reverse move, metropolis_test and the averages, with the walker's state
// in shared memory.
//
// pairs_kernel is persistent: its CTAs walk over the population with G
// independent groups of kThreads threads each, every group on its own
// walker and its own named barrier, so one group's latency overlaps the
// other's. Its random spline-row lookups (three per pair) go to a
// shared-memory copy of the pair rows when they fit and are wanted
// (stage_rows), made once per launch and shared by the groups; random rows
// in global memory cost an L1 tag lookup per lane, shared memory a few bank
// wavefronts per warp. G and the staging are the launch choices that
// qmc2d_autotune times (DevSys::tune_groups, tune_stage); by default G = 2
// with the rows staged. Both caps keep 128 registers a thread (G = 2: one
// 512-thread CTA per SM; G = 1: up to two 256-thread CTAs).

//
// R is the precision of the u2 and v2 pair terms (qmc2d_set_precision), LG
// the lanes per particle of the pair passes (4, 8 or 16: a launch choice,
// DevSys::tune_lanes).
template <class R, int G, int LG>
__global__ void __launch_bounds__(G * kThreads, 2 / G) pairs_kernel(const DevSys *sp, DevPop pop,
                                                                    MoveArgs a, int stage_rows) {
  constexpr int kPairGroups = G, kPairThreads = G * kThreads;
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  const size_t carve = (pair_carve(S, nullptr, nullptr, kThreads) + 127) & ~size_t(127);
  const int grp = threadIdx.x / kThreads, tid = threadIdx.x - grp * kThreads;
  EvalSmem m;
  pair_carve(S, smem + grp * carve, &m, kThreads);
  const R *rows_g = pair_rows<R>(S);
  R *rows_s = reinterpret_cast<R *>(smem + kPairGroups * carve);
  if (stage_rows) {  // the first copy16 16-byte parts of each global row
    using Lay = RowLayout<R>;
    constexpr int V = Lay::copy16, VG = Lay::gstride * (int)sizeof(R) / 16;
    const int nrow = S.cmb_nblk * (S.cmb_ng + 1);
    const float4 *src = reinterpret_cast<const float4 *>(rows_g);
    for (int e = threadIdx.x; e < nrow * V; e += kPairThreads) {
      const int r = e / V, q = e - r * V;
      cp_async16(reinterpret_cast<float4 *>(rows_s + (size_t)r * Lay::sstride) + q,
                 src + (size_t)r * VG + q);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  const GroupSync sync{1 + grp, kThreads};
  const int N = S.N, N2 = 2 * N;
  const uint32_t step = a.step0 + (a.ctr ? a.ctr[0] : 0u);
  const double pi = 3.141592653589793;
  const MoveScratch L = move_scratch(S);
  for (int w = blockIdx.x * kPairGroups + grp; w < a.nw; w += gridDim.x * kPairGroups) {
    long long tph = clock64();
    double wo = 0.0;
    for (int j = tid; j < N2; j += kThreads) {
      int ti = type_of(S, j >> 1);
      double var = 2.0 * S.hbs2m[ti] * a.delta, vari = 1.0 / var;
      double2 u = uniform2(a.seed, (uint32_t)j, (uint32_t)w, step, 0u);
      double chi = cos(pi * u.x) * sqrt(-2.0 * var * log(u.y));
      wo -= chi * chi * vari;
      m.x[j] = chi + (-var * pop.g[(size_t)w * N2 + j]) + pop.x[(size_t)w * N2 + j];
    }
    const double wold = block_sum_t<kThreads>(wo, m.red, sync, tid);
    phase_mark(S, PH_PROPOSE, tph, tid == 0);
    double *o = a.scr + (size_t)w * L.stride;
    double *pout = S.has_bf ? o + L.pair : nullptr;
    if (stage_rows)
      eval_pairs<kThreads, true, R, GroupSync, LG>(S, m, tph, pout, (const R *)rows_s, sync,
                                                   tid);
    else
      eval_pairs<kThreads, false, R, GroupSync, LG>(S, m, tph, pout, rows_g, sync, tid);
    pair_rhok<LG>(S, m, tid, kThreads, sync);
    sync();
    for (int j = tid; j < 4 * S.nk; j += kThreads) o[L.rhok + j] = m.rhok[j];
    for (int j = tid; j < N2; j += kThreads) {
      o[L.x + j] = m.x[j];
      o[L.g + j] = m.g[j];
      o[L.q + j] = m.q[j];
      o[L.qbd + j] = m.qbd[j];
    }
    for (int j = tid; j < 3 * N; j += kThreads) o[L.sb + j] = m.Sb[j];
    for (int j = tid; j < N; j += kThreads) {
      o[L.lap + j] = m.lap[j];
      o[L.ltf + j] = m.ltf[j];
      o[L.vp + j] = m.vp[j];
    }
    if (tid == 0) o[L.wold] = wold;
    sync();  // m is reused by the group's next walker
  }
}

size_t move_scratch_doubles(const DevSys &hs) { return move_scratch(hs).stride; }

// ------------------------------------------------- orbitals and inversion
// orb_inv_kernel: for every (walker, spin) of a move, one warp forms the
// plane-wave orbital matrix A(k, j) = exp(i g_k . q_j) of the proposed
// backflow coordinates (paho_orbitals, reptation.f:10298-10315) and inverts
// it by Gauss-Jordan with partial pivoting (zgefa/zgedi, reptation.f:9227,
// 9338), lane k holding row k in registers: the pivot key is the top word
// of |re|+|im| with 255 - row in its low byte (one redux per step), the
// pivot row reaches the other lanes through shared memory, and every lane
// updates its row. The row is held rotated: at step k register j holds
// column (k + j) mod NM, so the pivot column is always register 0, each
// update writes its result one register down (no moves) and the eliminated
// column enters at register NM - 1; after NM steps the columns are back in
// place. The step loop is therefore not unrolled and its code stays in the
// instruction cache. A spin with n < NM orbitals is padded to NM with
// identity rows, whose steps k >= n pivot on row k and leave rows < n
// unchanged. Outputs, as gj_invert_reg: W(pi(k), c) = A^-1(k, pi(c)) with
// the pivot rows unscaled until the end, perm, |pivot|^2 and the singular
// flag, into the walker's move scratch, where move_kernel reads them
// instead of inverting. No block barrier after the DevSys load: each warp
// works alone, many per scheduler, so one matrix's pivot chain hides
// behind the others' updates.
constexpr int kOrbWarps = 4;  // warps (spin matrices) per CTA

__host__ __device__ inline size_t orb_inv_warp_doubles(int n) {
  // the warp's tile of W (n x ws_ld(n) complex), q of its electrons, two pivot rows
  return (size_t)2 * n * ws_ld(n) + 2 * (size_t)n + 4 * 32;
}

template <int NM>
__global__ void __launch_bounds__(32 * kOrbWarps) orb_inv_kernel(const DevSys *sp, MoveArgs a) {
  static_assert(NM <= 32, "one lane per row");
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5, nt = S.nt;
  const int item = blockIdx.x * kOrbWarps + wl, w = item / nt, spn = item - w * nt;
  if (w >= a.nw) return;  // whole warps; nothing below waits on other warps
  const int n = S.np[spn], f0 = S.ipfrst[spn], ld = ws_ld(n), r = lane;
  size_t wd = 0;
  for (int t = 0; t < nt; t++) wd = max(wd, orb_inv_warp_doubles(S.np[t]));
  double *base = reinterpret_cast<double *>(smem) + (size_t)wl * wd;
  double2 *tile = reinterpret_cast<double2 *>(base);
  double *qs = base + 2 * (size_t)n * ld;
  double2 *prow = reinterpret_cast<double2 *>(qs + 2 * n);  // 2 x 32, double-buffered
  const MoveScratch L = move_scratch(S);
  double *o = a.scr + (size_t)w * L.stride;
  size_t off = L.inv;
  for (int t = 0; t < spn; t++) off += inv_spin_doubles(S.np[t]);
  double2 *outA = reinterpret_cast<double2 *>(o + off);
  double2 *outW = outA + (size_t)n * n;
  double *outD = reinterpret_cast<double *>(outW + (size_t)n * ld);
  double *outP = outD + n;
  double *outS = outP + n;
  for (int e = lane; e < 2 * n; e += 32) qs[e] = o[L.q + 2 * f0 + e];
  __syncwarp();
  // orbitals: lane r is orbital r; rows n .. NM-1 are identity rows
  const double gx = r < n ? __ldg(S.gvec + 2 * r) : 0.0, gy = r < n ? __ldg(S.gvec + 2 * r + 1) : 0.0;
  double2 v[NM];
#pragma unroll
  for (int j = 0; j < NM; j++) {
    const bool on = r < n && j < n;
    const double kr = on ? qs[2 * j] * gx + qs[2 * j + 1] * gy : 0.0;
    double sv, cv;
    sincos(kr, &sv, &cv);
    v[j] = on ? make_double2(cv, sv) : make_double2(r == j ? 1.0 : 0.0, 0.0);
  }
  // A, column-major (A[k + j n]): for each j the lanes write consecutive k
  if (r < n)
#pragma unroll
    for (int j = 0; j < NM; j++)
      if (j < n) outA[r + (size_t)j * n] = v[j];
  bool used = r >= n;
  double2 my_inv = make_double2(1.0, 0.0);
  int my_perm = 0, sing = 0;
  double my_dk = 0.0;
#pragma unroll 1
  for (int k = 0; k < NM; k++) {
    int p = k;  // an identity row's own step
    if (k < n) {
      const double av = fabs(v[0].x) + fabs(v[0].y);
      const unsigned key =
          used ? 0u : ((unsigned)__double2hiint(av) & ~0xFFu) | (unsigned)(255 - r);
      const unsigned best = __reduce_max_sync(0xffffffffu, key);
      // Every unused row's key has 255 - r in its low byte, so p is an
      // unused row < n at every step, an exactly zero or NaN column included.
      p = 255 - (int)(best & 0xFFu);
      sing |= (best >> 8) == 0u;  // every candidate zero (or subnormal)
    }
    double2 *pr = prow + (k & 1) * 32;
    if (r == p)
#pragma unroll
      for (int c = 0; c < NM; c++) pr[c] = v[c];
    __syncwarp();
    const double2 piv = pr[0];
    const double d = piv.x * piv.x + piv.y * piv.y;
    const double rd = rcp_newton(d);
    const double2 inv = make_double2(piv.x * rd, -piv.y * rd);
    if (lane == k && k < n) {
      my_perm = p;
      my_dk = d;
    }
    const bool isp = r == p;
    used = used || isp;
    if (isp) my_inv = inv;
    double2 fac = cmul(v[0], inv);
    if (isp || r >= n) fac = make_double2(0.0, 0.0);
    // register j - 1 <- column (k + j) mod NM, the next pivot column first
#pragma unroll
    for (int j = 1; j < NM; j++) {
      const double2 b = pr[j];
      v[j - 1].x = fma(-fac.x, b.x, fma(fac.y, b.y, v[j].x));
      v[j - 1].y = fma(-fac.x, b.y, fma(-fac.y, b.x, v[j].y));
    }
    v[NM - 1] = isp ? make_double2(1.0, 0.0) : make_double2(-fac.x, -fac.y);
  }
  // rows normalised by their own pivot, out through shared memory so the
  // scratch writes are consecutive
  if (r < n)
#pragma unroll
    for (int c = 0; c < NM; c++)
      if (c < n) tile[(size_t)r * ld + c] = cmul(v[c], my_inv);
  __syncwarp();
  for (int e = lane; e < n * ld; e += 32) outW[e] = tile[e];
  if (lane < n) {
    outD[lane] = my_dk;
    outP[lane] = (double)my_perm;
  }
  if (lane == 0) outS[0] = (double)sing;
}


// kSeq: the one-buffer form for moves whose orbitals and inverses come from
// orb_inv_kernel (smaller shared memory, 80 registers: three CTAs per SM).
template <bool kGmat, bool kSeq>
__global__ void __launch_bounds__(kThreads, kSeq ? 3 : 2) move_kernel(const DevSys *sp, DevPop pop,
                                                                      MoveArgs a) {
  __shared__ DevSys S;
  extern __shared__ __align__(16) char smem[];
  load_sys(S, sp);
  EvalSmem m;
  size_t off = eval_carve<kGmat>(S, smem, &m, kGmat ? gmat_block(S, blockIdx.x) : nullptr,
                                 nullptr, kSeq);
  MoveSmem v;
  move_carve(S, smem + off, &v, kSeq);
  if (kSeq) v.pn = reinterpret_cast<double *>(m.A[0]);  // po and blk stay in HBM
  const int w = blockIdx.x, tid = threadIdx.x;
  if (w >= a.nw) return;
  const int N = S.N, N2 = 2 * N, np = S.nprops, nt = S.nt;
  const MoveScratch L = move_scratch(S);
  const double *o = a.scr + (size_t)w * L.stride;
  // the pair values are read by the Jacobian build long after this point,
  // the orbitals and inverse of orb_inv_kernel at the start of the
  // determinant section; by now the earlier kernels' writes for this walker
  // have left L2, so bring them back (bulk L2 prefetch, 32 KB per request;
  // both blocks start 16-byte aligned and are whole doubles long: round down
  // to 16 bytes and let the tail come with the loads)
  auto prefetch_l2 = [&](const double *p, size_t doubles) {
    const size_t bytes = (sizeof(double) * doubles) & ~size_t(15);
    const char *base = reinterpret_cast<const char *>(p);
    for (size_t b0 = (size_t)tid * 32768; b0 < bytes; b0 += (size_t)kThreads * 32768) {
      const unsigned sz = (unsigned)(bytes - b0 < 32768 ? bytes - b0 : 32768);
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + b0), "r"(sz)
                   : "memory");
    }
  };
  if (!kGmat && a.orb_inv && L.inv) {
    size_t nd = 0;
    for (int t = 0; t < nt; t++) nd += inv_spin_doubles(S.np[t]);
    prefetch_l2(o + L.inv, nd);
  }
  if (S.has_bf && !S.bf_zero) prefetch_l2(o + L.pair, 3 * pair_count(N));
  if (kSeq) {  // read at the write-back (from a 16-byte boundary)
    const size_t e0 = (size_t)w * np, e1 = (e0 + 1) & ~size_t(1);
    prefetch_l2(pop.p + e1, np - (e1 - e0));
    prefetch_l2(a.blk + e1, np - (e1 - e0));
  }
  // the walker's state into shared memory: asynchronous 8-byte copies, all
  // in flight at once (plain loads in the HBM-determinant instance, whose
  // register budget they would push into spills)
  auto ld8 = [&](double *dst, const double *src) {
    if (kGmat)
      *dst = *src;
    else
      cp_async8(dst, src);
  };
  for (int j = tid; j < N2; j += kThreads) {
    ld8(v.xo + j, pop.x + (size_t)w * N2 + j);
    ld8(v.go + j, pop.g + (size_t)w * N2 + j);
    ld8(m.x + j, o + L.x + j);
    ld8(m.g + j, o + L.g + j);
    ld8(m.q + j, o + L.q + j);
    ld8(m.qbd + j, o + L.qbd + j);
    m.gd[j] = 0.0;
  }
  for (int j = tid; j < 3 * N; j += kThreads) ld8(m.Sb + j, o + L.sb + j);
  for (int j = tid; j < N; j += kThreads) {
    ld8(m.lap + j, o + L.lap + j);
    ld8(m.ltf + j, o + L.ltf + j);
    ld8(m.vp + j, o + L.vp + j);
    m.lapd[j] = 0.0;
    m.ph2[j] = 0.0;
    m.ph2d[j] = 0.0;
  }
  if (!kSeq)
    for (int j = tid; j < np; j += kThreads) {
      ld8(v.po + j, pop.p + (size_t)w * np + j);
      ld8(v.blk + j, a.blk + (size_t)w * np + j);
    }
  if (tid < nt) ld8(v.ho + tid, pop.h + (size_t)w * nt + tid);
  const double wold = o[L.wold];
  // kSeq: of the old properties only these two before the write-back
  const double po_ltf = kSeq ? pop.p[(size_t)w * np + QMC2D_JLTF] : 0.0;
  const double po_et = kSeq ? pop.p[(size_t)w * np + QMC2D_JETOT] : 0.0;
  if (!kGmat) cp_async_wait_all();
  __syncthreads();
  double so = pop.s[w];
  double age = pop.age[w];
  double norm = a.blk_norm[w];
  double wate = (a.dmc && !a.first) ? a.wate[w] : 1.0;
  double nacc = 0.0, nforced = 0.0;
  int status = 0;
  const uint32_t step = a.step0 + (a.ctr ? a.ctr[0] : 0u);
  long long tph = clock64();
  double sn = 1.0;
  status |= eval_det<kGmat, kSeq>(S, m, v.hn, v.pn, &v.sc[0], tph,
                                  S.has_bf ? o + L.pair : nullptr, o + L.rhok,
                                  !kGmat && a.orb_inv && L.inv ? o + L.inv : nullptr);
  sn = v.sc[0];
  // reverse move (reptation.f:4660-4674)
  double wn = 0.0;
  for (int j = tid; j < N2; j += kThreads) {
    int ti = type_of(S, j >> 1);
    double var = 2.0 * S.hbs2m[ti] * a.delta, vari = 1.0 / var;
    double chi = v.xo[j] - m.x[j] - (-var * m.g[j]);
    wn -= chi * chi * vari;
  }
  double wnew = block_sum(wn, m.red);
  double p;
  if (age == a.mage) {
    p = 1.0;
    nforced += 1.0;
  } else {
    p = ((kSeq ? po_ltf : v.po[QMC2D_JLTF]) - v.pn[QMC2D_JLTF]) * 2.0 + 0.5 * (wnew - wold);
    p = fmin(0.0, fmax(-50.0, p));
    p = exp(p);
  }
  // metropolis_test (reptation.f:2622-2659)
  double xr = 1.0;
  if (p < 1.0) xr = uniform2(a.seed, 0xFFFFFFFEu, (uint32_t)w, step, 0u).x;
  bool acc = p >= xr;
  const double et_old = kSeq ? po_et : v.po[QMC2D_JETOT];
  double elocal = acc ? 0.5 * (v.pn[QMC2D_JETOT] + et_old) : et_old;
  // the old properties read above before the copy below overwrites them;
  // kSeq reads them from registers, and block_sum's last barrier already
  // follows every read of xo and go
  if (!kSeq) __syncthreads();
  if (acc) {
    for (int j = tid; j < N2; j += kThreads) {
      v.xo[j] = m.x[j];
      v.go[j] = m.g[j];
    }
    if (!kSeq)
      for (int j = tid; j < np; j += kThreads) v.po[j] = v.pn[j];
    if (tid < nt) v.ho[tid] = v.hn[tid];
    so = sn;
    age = 0.0;
    nacc += 1.0;
  } else {
    age += 1.0;
  }
  if (!kSeq) __syncthreads();  // po's copy before its acceptance entry
  if (tid == 0 && !kSeq) v.po[QMC2D_JACC] = p;
  double wgt = 1.0;
  if (a.dmc) {
    // dmc weight (reptation.f:898-903), multiplied over the generation's moves;
    // with ecut > 0 (qmc2d_set_dmc_ecut, not in the reference) the local
    // energy in the weight is first clamped to etrial +- ecut
    double el = elocal;
    if (a.ecut > 0.0) el = fmin(fmax(el, a.etrial - a.ecut), a.etrial + a.ecut);
    double peso = exp(-S.npnorm * (el - a.etrial) * a.delta);
    if (peso > a.mmult) peso = a.mmult;
    wate *= peso;
    wgt = wate;
  }
  if (!kSeq) {
    __syncthreads();  // the acceptance entry before the sums
    for (int j = tid; j < np; j += kThreads) v.blk[j] += v.po[j] * wgt;
  }
  norm += wgt;
  phase_mark(S, PH_ACCEPT, tph);
  __syncthreads();
  for (int j = tid; j < N2; j += kThreads) {
    pop.x[(size_t)w * N2 + j] = v.xo[j];
    pop.g[(size_t)w * N2 + j] = v.go[j];
  }
  if (kSeq) {
    // the walker's properties: the new ones if accepted, else the old ones
    // in HBM, with the acceptance probability; the block sums in HBM
    for (int j = tid; j < np; j += kThreads) {
      const size_t i = (size_t)w * np + j;
      double val = acc ? v.pn[j] : pop.p[i];
      if (j == QMC2D_JACC) val = p;
      double b = a.blk[i];
      b += val * wgt;
      a.blk[i] = b;
      if (acc || j == QMC2D_JACC) pop.p[i] = val;
    }
  } else {
    for (int j = tid; j < np; j += kThreads) {
      pop.p[(size_t)w * np + j] = v.po[j];
      a.blk[(size_t)w * np + j] = v.blk[j];
    }
  }
  if (tid < nt) pop.h[(size_t)w * nt + tid] = v.ho[tid];
  if (tid == 0) {
    pop.s[w] = so;
    pop.age[w] = age;
    a.blk_norm[w] = norm;
    a.cnt[4 * w + 0] += nacc;
    a.cnt[4 * w + 1] += 1.0;
    a.cnt[4 * w + 2] += nforced;
    if (status) a.cnt[4 * w + 3] += 1.0;
    if (a.wate) a.wate[w] = wate;
    a.status[w] |= status;
  }
}

// ------------------------------------------------------------- branch2
// One block. Population-wide steps of branch2 (reptation.f:2174-2212) and
// prov_dest's in-rank assignment (reptation.f:2260-2271) on global scratch.
// Exclusive scan of one value per thread over the block (warp shuffles,
// then the warp totals by warp 0); ws holds 33 values, ws[32] the total.
template <class T>
__device__ T block_exclusive_scan(T v, T *ws) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  T ex = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) ex = T(0);
  __syncthreads();  // ws may still be read by a previous scan
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    T t = lane < nwarp ? ws[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    T e = __shfl_up_sync(0xffffffffu, t, 1);
    if (lane == 0) e = T(0);
    if (lane < nwarp) ws[lane] = e;
    if (lane == 31) ws[32] = t;
  }
  __syncthreads();
  return ws[w] + ex;
}

constexpr int kBranchThreads = 1024;

__global__ void __launch_bounds__(kBranchThreads) branch_kernel(int nw, double *wate,
                                                                uint64_t seed, uint32_t gen0,
                                                                const uint32_t *ctr,
                                                                BranchScratch b) {
  const uint32_t gen = gen0 + (ctr ? ctr[1] : 0u);
  __shared__ double dws[33];
  __shared__ int iws[33];
  __shared__ double red[32];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int seg = (nw + nt - 1) / nt;
  const int lo = min(nw, tid * seg), hi = min(nw, lo + seg);
  // cap at wmult = 10 (reptation.f:2174-2181)
  int ncap = 0;
  double loc = 0.0;
  for (int i = lo; i < hi; i++) {
    double v = wate[i];
    if (v > 10.0) {
      v = 10.0;
      wate[i] = v;
      ncap++;
    }
    loc += v;
  }
  if (ncap) atomicAdd(b.ncapped, ncap);
  // somma
  for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
  if ((tid & 31) == 0) red[tid >> 5] = loc;
  __syncthreads();
  double somma = 0.0;
  for (int k = 0; k < nt / 32; k++) somma += red[k];
  // multiplicities and fractional parts, inclusive scan of the fractions
  double part = 0.0;
  for (int i = lo; i < hi; i++) {
    double ww = nw * wate[i] / somma;
    int tm = (int)ww;
    b.mult[i] = tm;
    b.delt[i] = ww - tm;
    part += ww - tm;
  }
  double run = block_exclusive_scan(part, dws);
  for (int i = lo; i < hi; i++) {
    run += b.delt[i];
    b.csum[i] = run;
  }
  __syncthreads();
  double k0 = b.csum[nw - 1];
  int ncomb = (int)llround(k0);
  // systematic comb: copy c lands on the first walker whose cumulative
  // fraction reaches c + r_c (r_c from the shared stream, as rannyu2), the
  // last walker when none does. csum is non-decreasing, so copy c lands in
  // this thread's walkers [lo, hi) exactly when csum[lo-1] < c + r_c <=
  // csum[hi-1] (or beyond csum[nw-1] for the last segment): each thread
  // draws only the few copies whose c is in that range and finds the walker
  // among its own.
  if (lo < hi) {
    const double cprev = lo > 0 ? b.csum[lo - 1] : -1.0, clast = b.csum[hi - 1];
    const int cmin = lo > 0 ? max(0, (int)floor(cprev) - 1) : 0;
    const int cmax = hi == nw ? ncomb - 1 : min(ncomb - 1, (int)floor(clast));
    for (int c = cmin; c <= cmax; c++) {
      const double target = c + uniform2(seed, (uint32_t)c, 0xFFFFFFFFu, gen, 1u).x;
      if (lo > 0 && !(cprev < target)) continue;
      int i = lo;
      while (i < hi && b.csum[i] < target) i++;
      if (i == hi) {
        if (hi != nw) continue;
        i = nw - 1;
      }
      b.mult[i] += 1;
    }
  }
  __syncthreads();
  // slots left empty take the surplus copies in order of source slot
  int zc = 0, ec = 0;
  for (int i = lo; i < hi; i++) {
    int mu = b.mult[i];
    zc += mu == 0;
    ec += mu > 1 ? mu - 1 : 0;
  }
  int zr = block_exclusive_scan(zc, iws);
  int er = block_exclusive_scan(ec, iws);
  const int etot = iws[32];  // every thread's extras
  for (int i = lo; i < hi; i++) {
    int mu = b.mult[i];
    b.zrank[i] = zr;
    b.ecum[i] = er;
    zr += mu == 0;
    er += mu > 1 ? mu - 1 : 0;
  }
  __syncthreads();
  for (int j = lo; j < hi; j++) {
    int src = j;
    if (b.mult[j] == 0) {
      int z = b.zrank[j];
      if (z < etot) {
        int a0 = 0, a1 = nw;  // upper_bound(ecum, z) - 1
        while (a0 < a1) {
          int mid = (a0 + a1) >> 1;
          if (b.ecum[mid] <= z) a0 = mid + 1;
          else a1 = mid;
        }
        src = a0 - 1;
      }
    }
    b.src[j] = src;
  }
}

__global__ void gather_kernel(DevPop from, DevPop to, const int *src, int N2, int nt, int np) {
  const int j = blockIdx.x, i = src[j];
  for (int e = threadIdx.x; e < N2; e += blockDim.x) {
    to.x[(size_t)j * N2 + e] = from.x[(size_t)i * N2 + e];
    to.g[(size_t)j * N2 + e] = from.g[(size_t)i * N2 + e];
  }
  for (int e = threadIdx.x; e < np; e += blockDim.x)
    to.p[(size_t)j * np + e] = from.p[(size_t)i * np + e];
  if (threadIdx.x < nt) to.h[(size_t)j * nt + threadIdx.x] = from.h[(size_t)i * nt + threadIdx.x];
  if (threadIdx.x == 0) {
    to.s[j] = from.s[i];
    to.age[j] = from.age[i];
  }
}

// Walker records [x(2N), g(2N), h(nt), p(np), s, age] of slots[k] to or
// from row k of a contiguous buffer (one CTA per record).
__global__ void records_kernel(DevPop pop, const int *slots, double *buf, int N2, int nt, int np,
                               int unpack) {
  const int k = blockIdx.x, j = slots[k];
  const size_t len = 2 * (size_t)N2 + nt + np + 2;
  double *r = buf + (size_t)k * len;
  double *f[6] = {pop.x + (size_t)j * N2, pop.g + (size_t)j * N2, pop.h + (size_t)j * nt,
                  pop.p + (size_t)j * np, pop.s + j, pop.age + j};
  const int n[6] = {N2, N2, nt, np, 1, 1};
  size_t off = 0;
  for (int q = 0; q < 6; q++) {
    for (int e = threadIdx.x; e < n[q]; e += blockDim.x) {
      if (unpack) f[q][e] = r[off + e];
      else r[off + e] = f[q][e];
    }
    off += n[q];
  }
}

__global__ void philox_probe_kernel(uint64_t seed, const uint32_t *ctr, uint32_t *out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint4 o = philox4x32_10(make_uint4(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]),
                          make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  out[4 * i] = o.x;
  out[4 * i + 1] = o.y;
  out[4 * i + 2] = o.z;
  out[4 * i + 3] = o.w;
}

// ------------------------------------------------- block sums over walkers
// out[j] = sum_w blk[w*np + j] (j < np), out[np] = sum_w norm[w]: one CTA per
// output, a fixed strided split and tree, so the result is reproducible.
__global__ void __launch_bounds__(256) block_reduce_kernel(const double *blk, const double *norm,
                                                           int n, int np, double *out) {
  __shared__ double part[256];
  const int j = blockIdx.x, t = threadIdx.x;
  double s = 0.0;
  if (j < np)
    for (int w = t; w < n; w += 256) s += blk[(size_t)w * np + j];
  else
    for (int w = t; w < n; w += 256) s += norm[w];
  part[t] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) part[t] += part[t + o];
    __syncthreads();
  }
  if (t == 0) out[j] = part[0];
}

// ------------------------------------------------------------ launchers
// The dynamic shared-memory limit of kernel fn on the current device is only
// ever raised: handles of different systems driven from several host threads
// launch the same kernels with different sizes, and a lower limit set by one
// between another's set and launch would fail that launch.
cudaError_t raise_smem_limit(const void *fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> cur;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t &c = cur[{dev, fn}];
  if (bytes <= c) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) c = bytes;
  return e;
}
static cudaError_t set_smem(const void *fn, size_t bytes) { return raise_smem_limit(fn, bytes); }

cudaError_t launch_eval(const DevSys &hs, const DevSys *ds, int nw, const double *x, double *g,
                        double *hl, double *props, double *s, int *status, cudaStream_t st) {
  if (nw <= 0) return cudaSuccess;
  size_t sm = eval_smem_bytes(hs);
  auto k = hs.gmat ? (hs.pair_f32 ? eval_kernel<float, true> : eval_kernel<double, true>)
                   : (hs.pair_f32 ? eval_kernel<float, false> : eval_kernel<double, false>);
  cudaError_t e = set_smem((const void *)k, sm);
  if (e != cudaSuccess) return e;
  k<<<nw, kThreads, sm, st>>>(ds, nw, x, g, hl, props, s, status);
  return cudaGetLastError();
}

template <class R, int G, int LG>
static cudaError_t launch_pairs_t(const DevSys &hs, const DevSys *ds, DevPop pop,
                                  const MoveArgs &a, cudaStream_t st, int nsm, int optin) {
  const void *k = (const void *)pairs_kernel<R, G, LG>;
  const size_t carve = G * ((pair_carve(hs, nullptr, nullptr, kThreads) + 127) & ~size_t(127));
  const size_t rows =
      sizeof(R) * RowLayout<R>::sstride * (size_t)hs.cmb_nblk * (hs.cmb_ng + 1);
  const int stage =
      hs.tune_stage != 1 && carve + rows + sizeof(DevSys) <= (size_t)optin ? 1 : 0;
  const size_t sm = carve + (stage ? rows : 0);
  cudaError_t e;
  if ((e = set_smem(k, sm)) != cudaSuccess) return e;
  int per_sm = 1;
  if (G == 1 &&
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, G * kThreads, sm)) !=
          cudaSuccess)
    return e;
  const int need = (a.nw + G - 1) / G;
  const int cap = nsm * (per_sm > 0 ? per_sm : 1);
  const int grid = need < cap ? need : cap;
  pairs_kernel<R, G, LG><<<grid, G * kThreads, sm, st>>>(ds, pop, a, stage);
  return cudaGetLastError();
}

template <class R, int LG>
static cudaError_t launch_pairs_g(const DevSys &hs, const DevSys *ds, DevPop pop,
                                  const MoveArgs &a, cudaStream_t st, int nsm, int optin) {
  return hs.tune_groups == 1 ? launch_pairs_t<R, 1, LG>(hs, ds, pop, a, st, nsm, optin)
                             : launch_pairs_t<R, 2, LG>(hs, ds, pop, a, st, nsm, optin);
}

template <class R>
static cudaError_t launch_pairs_r(const DevSys &hs, const DevSys *ds, DevPop pop,
                                  const MoveArgs &a, cudaStream_t st, int nsm, int optin) {
  switch (hs.tune_lanes) {
    case 4: return launch_pairs_g<R, 4>(hs, ds, pop, a, st, nsm, optin);
    case 16: return launch_pairs_g<R, 16>(hs, ds, pop, a, st, nsm, optin);
    default: return launch_pairs_g<R, 8>(hs, ds, pop, a, st, nsm, optin);
  }
}

cudaError_t launch_pairs(const DevSys &hs, const DevSys *ds, DevPop pop, const MoveArgs &a,
                         cudaStream_t st) {
  if (a.nw <= 0) return cudaSuccess;
  int dev = 0, nsm = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
      cudaSuccess)
    return e;
  return hs.pair_f32 ? launch_pairs_r<float>(hs, ds, pop, a, st, nsm, optin)
                     : launch_pairs_r<double>(hs, ds, pop, a, st, nsm, optin);
}

bool orb_inv_applies(const DevSys &hs) { return hs.split_inv && orb_inv_fits(hs); }
bool orb_inv_pays(const DevSys &hs, int nw, int nsm, int min_per_sm) {
  return orb_inv_applies(hs) && (long)nw * hs.nt >= (long)nsm * min_per_sm;
}

cudaError_t launch_orb_inv(const DevSys &hs, const DevSys *ds, const MoveArgs &a,
                           cudaStream_t st) {
  if (a.nw <= 0 || !a.orb_inv || !orb_inv_applies(hs)) return cudaSuccess;
  size_t wd = 0;
  for (int t = 0; t < hs.nt; t++) wd = std::max(wd, orb_inv_warp_doubles(hs.np[t]));
  const size_t sm = sizeof(double) * wd * kOrbWarps;
  const int items = a.nw * hs.nt, grid = (items + kOrbWarps - 1) / kOrbWarps;
  // registers for the rows: the closed shells' sizes 13, 21, 25, 29 (N = 58,
  // the benchmark shell) exactly, others padded to 16 or 32 columns
  const int nm = hs.nmax;
  auto k = nm <= 13   ? orb_inv_kernel<13>
           : nm <= 16 ? orb_inv_kernel<16>
           : nm <= 21 ? orb_inv_kernel<21>
           : nm <= 25 ? orb_inv_kernel<25>
           : nm <= 29 ? orb_inv_kernel<29>
                      : orb_inv_kernel<32>;
  cudaError_t e = set_smem((const void *)k, sm);
  if (e != cudaSuccess) return e;
  k<<<grid, 32 * kOrbWarps, sm, st>>>(ds, a);
  return cudaGetLastError();
}

cudaError_t launch_move(const DevSys &hs, const DevSys *ds, DevPop pop, const MoveArgs &a,
                        cudaStream_t st) {
  if (a.nw <= 0) return cudaSuccess;
  const bool seq = !hs.gmat && a.orb_inv && orb_inv_applies(hs) && props_buf_fits(hs);
  size_t sm = seq ? move_smem_bytes_seq(hs) : move_smem_bytes(hs);
  auto k = hs.gmat ? move_kernel<true, false>
                   : (seq ? move_kernel<false, true> : move_kernel<false, false>);
  cudaError_t e = set_smem((const void *)k, sm);
  if (e != cudaSuccess) return e;
  k<<<a.nw, kThreads, sm, st>>>(ds, pop, a);
  return cudaGetLastError();
}

cudaError_t launch_block_reduce(const double *blk, const double *norm, int n, int np,
                                double *out, cudaStream_t st) {
  if (n <= 0 || np <= 0) return cudaSuccess;
  block_reduce_kernel<<<np + 1, 256, 0, st>>>(blk, norm, n, np, out);
  return cudaGetLastError();
}

cudaError_t launch_branch(int nw, double *wate, uint64_t seed, uint32_t gen, BranchScratch b,
                          cudaStream_t st, const uint32_t *ctr) {
  if (nw <= 0) return cudaSuccess;
  branch_kernel<<<1, kBranchThreads, 0, st>>>(nw, wate, seed, gen, ctr, b);
  return cudaGetLastError();
}

cudaError_t launch_gather(const DevSys &hs, DevPop from, DevPop to, const int *src, int nw,
                          cudaStream_t st) {
  if (nw <= 0) return cudaSuccess;
  gather_kernel<<<nw, 128, 0, st>>>(from, to, src, 2 * hs.N, hs.nt, hs.nprops);
  return cudaGetLastError();
}

__global__ void counters_add_kernel(uint32_t *ctr, uint32_t steps, uint32_t gens) {
  ctr[0] += steps;
  ctr[1] += gens;
}

cudaError_t launch_counters_add(uint32_t *ctr, uint32_t steps, uint32_t gens, cudaStream_t st) {
  counters_add_kernel<<<1, 1, 0, st>>>(ctr, steps, gens);
  return cudaGetLastError();
}

cudaError_t launch_records(const DevSys &hs, DevPop pop, const int *slots, double *buf, int n,
                           int unpack, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  records_kernel<<<n, 128, 0, st>>>(pop, slots, buf, 2 * hs.N, hs.nt, hs.nprops, unpack);
  return cudaGetLastError();
}

cudaError_t launch_philox_probe(uint64_t seed, const uint32_t *ctr, uint32_t *out, int n,
                                cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  philox_probe_kernel<<<(n + 127) / 128, 128, 0, st>>>(seed, ctr, out, n);
  return cudaGetLastError();
}

}  // namespace q2d
