// walker_eval.cuh - FP64 evaluation of one walker by one CTA: the
// reference's compute_properties (reptation.f:2661) = distances :4127,
// two_body :2981, three_body :2777, slater_excitations :9967, kinetic :2729,
// potential :3986, restated for a 256-thread CTA with every intermediate in
// shared memory.
//
// Layout and parallel decomposition
//   * pair sums: LG threads per particle i sweep j != i (each unordered pair
//     is visited from both ends, so per-particle sums need no atomics); the
//     LG partial sums meet by warp shuffles in a fixed order. LG is 8, or 4
//     or 16 as a launch choice of the pair kernel.
//   * u3 (l=1 factorised triplets): with G_i = -sum_j xi(r_ij) r_ij and
//     M_ij = xi I + (xi'/r) r r^T, the gradient of -1/2 sum|G|^2 on k is
//     sum_j M_kj (G_k - G_j) and its Laplacian is
//     sum_j (xi'' + 3 xi'/r) r_kj.(G_k - G_j) - tr(S_k^2) - sum_j tr(M_kj^2),
//     S_k = sum_j M_kj: the dense dg/ddg of makeg/dotg are never formed.
//   * determinants: A(k,j) = exp(i g_k.q_j) for both spins at once; each
//     spin's matrix is inverted by half the CTA (Gauss-Jordan with partial
//     pivoting, rows chosen in place instead of swapped, every row held in
//     registers, one group barrier per step), then rho_k on all warps.
//     Then, per spin, F_a = A^-1 diag(i g_a) A (register-tiled complex
//     GEMM) and the backflow cross term sum_{j,k} Re[(J_j.F(k,j))(J_k.F(j,k))]
//     as the quadratic form of the symmetric 2n x 2n matrix
//     M_ac(j,k) = Re[F_a(k,j) F_c(j,k)] against the Jacobian columns of every
//     electron (FP64 tensor-core GEMM, mma.m8n8k4); the drift and the first
//     two Laplacian terms are summed while the Jacobian columns are built.
#pragma once

#include <cuda_runtime.h>

#include "devsys.h"

namespace q2d {

struct EvalSmem {
  double *x, *g, *q, *G3, *S3, *Sb, *qbd, *lap, *ltf, *vp, *ph2;
  double *gd, *lapd, *ph2d;  // determinant contributions (added unless underflow)
  double *rhok;              // 2*nk per rhok slot
  double2 *A[2], *W[2];      // per spin: orbitals (column-major) and the inversion workspace
  double2 *F0, *F1;          // F_a of the spin being processed, column-major
  double *D2, *U, *part, *red, *gsh, *dk[2];
  double *fdg;  // F0(j,j), F1(j,j) of the spin being processed (4 doubles per j)
  int *perm[2], *used[2], *iscal, *gidx;
  double *gval;
  // register-resident inversion: per spin, double-buffered pivot-row slots
  // of every warp and the warps' pivot keys (inside the F0 region)
  double2 *gslot[2];
  unsigned *gkey[2];
  // inversion in global memory (gmat): each spin's panel, multipliers and
  // scaled pivot rows (gj_invert_gmem)
  double2 *fcol[2];
  // blocked inversion with one-warp panels (gj_invert_panel): each spin's
  // multipliers, scaled pivot rows, pivot reciprocals and rows (inside the
  // F0 region, like gslot/gkey)
  double2 *pscr[2];
  // lattice power tables of rho_k in the pair kernels (DevSys::rk_lat):
  // exp(2 pi i p x_i / Lx) at [p N + i], p <= rk_p1, then exp(2 pi i p y_i / Ly)
  double2 *rkt = nullptr;
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
// Row stride of the inversion workspace: odd, so the rows that the lanes of
// a warp own fall on distinct 16-byte bank groups.
__host__ __device__ inline int ws_ld(int n) { return n | 1; }

// Register-resident Gauss-Jordan: complex columns per thread, and the
// lanes per row L (a power of two) with kGjCols*L >= n and one row per
// thread of an nthr-thread group; 0 when n does not fit that layout.
constexpr int kGjCols = 8;
// Pivot steps per pass over a determinant held in HBM (gj_invert_gmem),
// and the shared memory that inversion takes per spin: the panel (later
// the scaled pivot rows), the multipliers, the pivots' reciprocals and rows.
constexpr int kGjBlock = 8;
__host__ __device__ inline size_t gj_gmem_scratch(int n) {
  return sizeof(double2) * (2 * (size_t)kGjBlock * n + kGjBlock) + sizeof(int) * kGjBlock;
}

// Per-spin scratch of gj_invert_panel (complex elements): multipliers and
// scaled pivot rows of a block (kGjBlock x n each), the block's pivot
// reciprocals and, in the last two elements, its pivot rows (ints).
__host__ __device__ inline size_t gj_panel_scratch(int n) {
  return 2 * (size_t)kGjBlock * n + kGjBlock + 2;
}

__host__ __device__ inline int gj_reg_lanes(int n, int nthr) {
  for (int L = 1; L <= 32; L *= 2)
    if (kGjCols * L >= n && nthr / L >= n) return L;
  return 0;
}
// Row slot of the register-resident inversion per warp (complex elements):
// the warp's candidate pivot row, lane s's kGjCols columns at s (kGjCols+1)
// (the odd stride keeps the lanes' 16-byte words on distinct banks), then
// the candidate's reciprocal and |pivot|^2.
__host__ __device__ inline int gj_reg_slot(int L) { return L * (kGjCols + 1) + 2; }

// Warps per spin for the register-resident inversion (all warps of the CTA).
__host__ __device__ inline int gj_reg_warps(int nt) { return (kThreads / 32) / (nt > 1 ? 2 : 1); }

// Cross-term GEMM Y = M U on the FP64 tensor cores (mma.m8n8k4): M is
// n2 x n2 row-major with row stride xt_ldm, the Jacobian block is stored
// transposed (UT, one row of xt_ldu per column of U). Both strides are
// 4 or 12 (mod 16) doubles, so the eight-byte fragment loads of a
// half-warp (4 rows x 4 consecutive columns) fall on 16 distinct banks.
__host__ __device__ inline int xt_row_tiles(int n2) { return (n2 + 7) / 8; }
__host__ __device__ inline int xt_ldm(int n2) {
  int l = (n2 + 3) & ~3;
  return (l % 8 == 0) ? l + 4 : l;
}
__host__ __device__ inline int xt_ldu(int n2) { return 8 * xt_row_tiles(n2) + 4; }

// Carve the dynamic shared memory; returns bytes used. With s.gmat the
// determinant matrices (A, W, F0 region) come from gbase instead, the
// walker's block of global memory, and *gbytes (when given) receives its
// size. kG fixes s.gmat at compile time in the kernels (0 off, 1 on); the
// host's sizing reads it (-1). one_buf: a single orbital/inverse/M buffer
// that the spins take in turn (the move kernel when orb_inv_kernel has
// formed both spins' orbitals and inverses: m.A[1] = m.A[0]).
template <int kG = -1>
__host__ __device__ inline size_t eval_carve(const DevSys &s, char *base, EvalSmem *m,
                                             char *gbase = nullptr, size_t *gbytes = nullptr,
                                             bool one_buf = false) {
  const bool gm = kG < 0 ? s.gmat != 0 : kG != 0;
  size_t off = 0, goff = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base ? base + off : nullptr;
    off += align16(bytes);
    return p;
  };
  // the large matrices: shared memory, or the global block with s.gmat
  auto mtake = [&](size_t bytes) -> char * {
    if (!gm) return take(bytes);
    char *p = gbase ? gbase + goff : nullptr;
    goff += (bytes + 255) & ~size_t(255);
    return p;
  };
  int N = s.N, n = s.nmax > 0 ? s.nmax : 1, ld = ws_ld(n);
  int nsp = s.nt;
  EvalSmem t;
  t.x = (double *)take(sizeof(double) * 2 * N);
  t.g = (double *)take(sizeof(double) * 2 * N);
  t.q = (double *)take(sizeof(double) * 2 * N);
  t.G3 = s.has_u3 ? (double *)take(sizeof(double) * 2 * N) : nullptr;  // u3 only
  t.S3 = s.has_u3 ? (double *)take(sizeof(double) * 3 * N) : nullptr;
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
  t.A[0] = t.A[1] = t.W[0] = t.W[1] = nullptr;
  t.F0 = t.F1 = nullptr;
  t.gslot[0] = t.gslot[1] = nullptr;
  t.gkey[0] = t.gkey[1] = nullptr;
  t.D2 = t.U = t.part = t.gsh = t.fdg = nullptr;
  t.dk[0] = t.dk[1] = nullptr;
  t.perm[0] = t.perm[1] = t.used[0] = t.used[1] = nullptr;
  t.fcol[0] = t.fcol[1] = nullptr;
  t.pscr[0] = t.pscr[1] = nullptr;
  if (s.has_bf) {
    // A[s] and W[s] are adjacent: the 2n x 2n real cross-term matrix of spin
    // s (row stride xt_ldm) overlays them once F0/F1 are formed.
    const size_t awbytes = sizeof(double2) * (n * n + n * ld);
    const size_t mbytes = sizeof(double) * 2 * n * xt_ldm(2 * n);
#pragma unroll
    for (int sp = 0; sp < 2; sp++) {
      if (sp >= nsp) continue;
      t.A[sp] = (one_buf && sp > 0) ? t.A[0] : (double2 *)mtake(awbytes > mbytes ? awbytes : mbytes);
      t.W[sp] = t.A[sp] ? t.A[sp] + n * n : nullptr;
      t.dk[sp] = (double *)take(sizeof(double) * n);
      t.perm[sp] = (int *)take(sizeof(int) * n);
      t.used[sp] = (int *)take(sizeof(int) * n);
      t.fcol[sp] = gm ? (double2 *)take(gj_gmem_scratch(n)) : nullptr;
    }
    // F0/F1 are dead once the cross-term matrix is built, so the cross
    // term's Jacobian columns U and partial sums share their space.
    // The inversion's pivot-row slots and keys are dead before F0/F1 are
    // formed, so they share the same space too.
    size_t fbytes = sizeof(double2) * 2 * n * n;
    const int ldu = xt_ldu(2 * n);
    size_t ubytes = sizeof(double) * ((size_t)kChunk * ldu + (size_t)xt_row_tiles(2 * n) * kChunk);
    const int gw = gj_reg_warps(nsp), gl = gj_reg_lanes(n, 32 * gw);
    const size_t slot_per_spin = (size_t)2 * gw * (gl > 0 ? gj_reg_slot(gl) : 0);  // double2
    size_t sbytes = sizeof(double2) * 2 * slot_per_spin + sizeof(unsigned) * 2 * 2 * gw;
    size_t rbytes = fbytes > ubytes ? fbytes : ubytes;
    if (sbytes > rbytes) rbytes = sbytes;
    const size_t pbytes = sizeof(double2) * 2 * gj_panel_scratch(n);
    if (!gm && pbytes > rbytes) rbytes = pbytes;
    t.F0 = (double2 *)mtake(rbytes);
    t.F1 = t.F0 ? t.F0 + n * n : nullptr;
    t.U = reinterpret_cast<double *>(t.F0);
    t.part = t.U ? t.U + (size_t)kChunk * ldu : nullptr;
    t.gslot[0] = t.F0;
    t.gslot[1] = t.F0 ? t.F0 + slot_per_spin : nullptr;
    t.gkey[0] = t.F0 ? reinterpret_cast<unsigned *>(t.F0 + 2 * slot_per_spin) : nullptr;
    t.gkey[1] = t.gkey[0] ? t.gkey[0] + 2 * gw : nullptr;
    t.pscr[0] = gm ? nullptr : t.F0;
    t.pscr[1] = (gm || !t.F0) ? nullptr : t.F0 + gj_panel_scratch(n);
    t.D2 = (double *)take(sizeof(double) * 3 * n);
    t.fdg = (double *)take(sizeof(double) * 4 * n);
    t.gsh = (double *)take(sizeof(double) * 2 * n);
  }
  t.red = (double *)take(sizeof(double) * kThreads);
  t.iscal = (int *)take(sizeof(int) * 8);
  t.gidx = (int *)take(sizeof(int) * 16);
  t.gval = (double *)take(sizeof(double) * 16);
  if (m) *m = t;
  if (gbytes) *gbytes = goff;
  return off;
}

// The walker's block of global memory for the determinant matrices of
// CTA b (gmat), or nullptr.
__device__ __forceinline__ char *gmat_block(const DevSys &S, int b) {
  return S.gmat ? reinterpret_cast<char *>(S.gmat_base + (size_t)b * S.gmat_stride) : nullptr;
}

// The pair passes alone (pairs_kernel): only the per-particle arrays they
// write and the reduction buffer; every other pointer is null.
__host__ __device__ inline size_t pair_carve(const DevSys &s, char *base, EvalSmem *m,
                                             int nthreads) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base ? base + off : nullptr;
    off += align16(bytes);
    return p;
  };
  const int N = s.N;
  EvalSmem t{};
  t.x = (double *)take(sizeof(double) * 2 * N);
  t.g = (double *)take(sizeof(double) * 2 * N);
  t.q = (double *)take(sizeof(double) * 2 * N);
  t.G3 = s.has_u3 ? (double *)take(sizeof(double) * 2 * N) : nullptr;  // u3 only
  t.S3 = s.has_u3 ? (double *)take(sizeof(double) * 3 * N) : nullptr;
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
  t.red = (double *)take(sizeof(double) * nthreads);
  t.rkt = s.rk_lat ? (double2 *)take(sizeof(double2) * (s.rk_p1 + s.rk_p2 + 2) * N) : nullptr;
  if (m) *m = t;
  return off;
}

// Per-walker move scratch in global memory (doubles), written by the pair
// kernel and read by the move kernel of the same step: the proposed
// configuration, the pair passes' per-particle sums, the proposal's log
// density, rho_k (both slots), and (backflow) the spline values of every
// pair i < j:
// eta(r_ij), eta'(r_ij)/r_ij and 3 eta'/r + eta'' at [k P + pair_tri(N, i, j)],
// P = N (N - 1) / 2 (the values are functions of r_ij alone, computed from
// the same bits for (i, j) and (j, i), so one triangle serves both orders).
// A reptile's bead growth also keeps its proposal's drift term (dold) and
// the free-propagator sum (lng) of get_w_stack (reptation.f:1804-1851).
__host__ __device__ inline size_t pair_count(int N) { return (size_t)N * (N - 1) / 2; }
// Row-major upper triangle without the diagonal: (a, b), a < b.
__host__ __device__ inline size_t pair_tri(int N, int a, int b) {
  return (size_t)a * (2 * N - a - 1) / 2 + (size_t)(b - a - 1);
}
struct MoveScratch {
  int x, g, q, sb, qbd, lap, ltf, vp, wold, dold, lng, rhok, pair;
  size_t inv;  // orb_inv_kernel's output per spin (0: no such region)
  size_t stride;
};
// Doubles of one spin's block of orb_inv_kernel output (n orbitals): the
// orbital matrix A (n x n complex, column-major as EvalSmem::A), the
// inverse W (n x ws_ld(n) complex, as EvalSmem::W), |pivot|^2, the pivot
// rows (as doubles) and the singular flag; even, so blocks stay 16-byte
// aligned.
__host__ __device__ inline size_t inv_spin_doubles(int n) {
  return ((size_t)2 * n * n + (size_t)2 * n * ws_ld(n) + 2 * (size_t)n + 2 + 1) & ~size_t(1);
}
// The batched orbital-and-inversion kernel applies: backflow determinants in
// shared memory, every spin at most 32 orbitals.
__host__ __device__ inline bool orb_inv_fits(const DevSys &s) {
  return s.has_bf && !s.gmat && s.nmax > 0 && s.nmax <= 32;
}
// with_inv: the layout of VMC/DMC moves, which may batch their inversion;
// reptation's kernels never do and lay their blocks out without that region
// (the same allocation holds them, closer together).
__host__ __device__ inline MoveScratch move_scratch(const DevSys &s, bool with_inv = true) {
  const int N = s.N;
  MoveScratch l;
  l.x = 0;
  l.g = 2 * N;
  l.q = 4 * N;
  l.sb = 6 * N;
  l.qbd = 9 * N;
  l.lap = 11 * N;
  l.ltf = 12 * N;
  l.vp = 13 * N;
  l.wold = 14 * N;
  l.dold = 14 * N + 1;
  l.lng = 14 * N + 2;
  l.rhok = 14 * N + 3;
  l.pair = (14 * N + 3 + 4 * (s.nk > 0 ? s.nk : 1) + 3) & ~3;
  size_t end = (size_t)l.pair + (s.has_bf ? 3 * pair_count(N) : 0);
  l.inv = 0;
  if (with_inv && orb_inv_fits(s)) {
    end = (end + 1) & ~size_t(1);
    l.inv = end;
    for (int sp = 0; sp < s.nt; sp++) end += inv_spin_doubles(s.np[sp]);
  }
  l.stride = (end + 31) & ~size_t(31);  // 256-byte aligned walker blocks
  return l;
}

// ----------------------------------------------------------------- helpers

__device__ __forceinline__ int type_of(const DevSys &S, int i) {
  return (S.nt > 1 && i >= S.ipfrst[1]) ? 1 : 0;
}

// Four doubles of the packed tables in a single 256-bit read-only load; p is
// 32-byte aligned (pair rows are 128-byte aligned, their parts 32 bytes).
__device__ __forceinline__ double4 knot_row(const double *p) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
      : "l"(p));
  return r;
}

// Pair-row parts: the four coefficients of each kind's table.
enum : int { PR_U2 = 0, PR_U3 = 4, PR_BF = 8, PR_V2 = 12 };

// The pair row of type pair (a, b) at knot min(cmb_ng, ind) in the rows at
// `rows` (the packed buffer's S.coef + S.cmb_off, or a shared-memory copy):
// part q holds the row min(ngrid, ind) of that pair's table of kind q, which
// is the knot getf/getf_0 clamp to (NaN/negative ind -> knot 0).
// Rows are 16 doubles apart in global memory and kPairRowSh apart in a
// shared-memory copy: 144 bytes, so consecutive knots start on different
// 16-byte bank groups and a warp's random rows spread over eight of them.
constexpr int kPairRowSh = 18;
template <int RS = 16>
__device__ __forceinline__ const double *pair_row(const DevSys &S, const double *rows, int a,
                                                  int b, int ind) {
  const int k = max(0, min(S.cmb_ng, ind));
  return rows + ((size_t)S.cmb_blk[a][b] * (S.cmb_ng + 1) + k) * RS;
}
__device__ __forceinline__ const double *pair_row(const DevSys &S, int a, int b, int ind) {
  return pair_row(S, S.coef + S.cmb_off, a, b, ind);
}

// Four doubles of a pair row in shared (kSh) or global memory.
template <bool kSh>
__device__ __forceinline__ double4 row_part(const double *p) {
  if (kSh) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const double2 b = reinterpret_cast<const double2 *>(p)[1];
    return make_double4(a.x, a.y, b.x, b.y);
  }
  return knot_row(p);
}

// getf (reptation.f:4114): the cubic of one knot row, f, f', f''.
template <bool kSh = false>
__device__ __forceinline__ void spline3(const DevSys &S, const double *part, double rem,
                                        double &f, double &df, double &ddf) {
  const double4 u = row_part<kSh>(part);
  double rm = rem * S.drti;
  f = u.x + rm * (u.y + rm * (u.z + rm * u.w));
  df = (u.y + rm * (2.0 * u.z + rm * (3.0 * u.w))) * S.drti;
  ddf = (u.z + rm * (3.0 * u.w)) * S.drti2;
}

// getf_0 (reptation.f:4103): f * (1/r)**iexp.
template <bool kSh = false>
__device__ __forceinline__ double spline0(const DevSys &S, const double *part, int iexp,
                                          double rem, double byr) {
  const double4 u = row_part<kSh>(part);
  double rm = rem * S.drti;
  double f = u.x + rm * (u.y + rm * (u.z + rm * u.w));
  for (int k = 0; k < iexp; k++) f *= byr;
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

// ---- the pair passes in either precision R of the two-body Jastrow and
// real-space Ewald terms (double, or float in the mixed-precision mode of
// qmc2d_set_precision); the u3 and backflow terms are FP64 in both.
//
// Row layouts per knot (units of R):
// - FP64 rows: u2 | u3 | backflow | v2, four doubles each (128 bytes), 16
//   apart in global memory and kPairRowSh (144 bytes) in shared memory;
// - mixed rows: the backflow and u3 rows in FP64, then the u2 and v2 rows
//   rounded to float (96 bytes), 32 floats (128 bytes, so the FP64 parts
//   stay 32-byte aligned for one 256-bit load) apart in global memory and
//   28 floats (112 bytes) in shared memory, which spreads a warp's random
//   rows over eight 16-byte bank groups as kPairRowSh does.
template <class R>
struct RowLayout;
template <>
struct RowLayout<double> {
  static constexpr int u2 = 0, u3 = 4, bf = 8, v2 = 12;
  static constexpr int gstride = 16, sstride = kPairRowSh, copy16 = 8;
};
template <>
struct RowLayout<float> {
  static constexpr int bf = 0, u3 = 8, u2 = 16, v2 = 20;
  static constexpr int gstride = 32, sstride = 28, copy16 = 6;
};

template <class R>
__device__ __forceinline__ const R *pair_rows(const DevSys &S);
template <>
__device__ __forceinline__ const double *pair_rows<double>(const DevSys &S) {
  return S.coef + S.cmb_off;
}
template <>
__device__ __forceinline__ const float *pair_rows<float>(const DevSys &S) {
  return reinterpret_cast<const float *>(S.coef + S.cmbm_off);
}

template <int RS>
__device__ __forceinline__ const float *pair_row(const DevSys &S, const float *rows, int a, int b,
                                                 int ind) {
  const int k = max(0, min(S.cmb_ng, ind));
  return rows + ((size_t)S.cmb_blk[a][b] * (S.cmb_ng + 1) + k) * RS;
}

// Four floats of a mixed row (one 128-bit load).
template <bool kSh>
__device__ __forceinline__ float4 row_part(const float *p) {
  return kSh ? *reinterpret_cast<const float4 *>(p) : __ldg(reinterpret_cast<const float4 *>(p));
}

// The knot spacing in precision R.
template <class R>
struct Knots {
  R drt, drti, drti2;
  __device__ explicit Knots(const DevSys &S) : drt((R)S.drt), drti((R)S.drti), drti2((R)S.drti2) {}
};

// getf / getf_0 in precision R (for R = double the same operations as
// spline3 / spline0 above).
template <bool kSh, class R>
__device__ __forceinline__ void spline3(const Knots<R> &K, const R *part, R rem, R &f, R &df,
                                        R &ddf) {
  const auto u = row_part<kSh>(part);
  const R rm = rem * K.drti;
  f = u.x + rm * (u.y + rm * (u.z + rm * u.w));
  df = (u.y + rm * ((R)2 * u.z + rm * ((R)3 * u.w))) * K.drti;
  ddf = (u.z + rm * ((R)3 * u.w)) * K.drti2;
}
template <bool kSh, class R>
__device__ __forceinline__ R spline0(const Knots<R> &K, const R *part, int iexp, R rem, R byr) {
  const auto u = row_part<kSh>(part);
  const R rm = rem * K.drti;
  R f = u.x + rm * (u.y + rm * (u.z + rm * u.w));
  for (int k = 0; k < iexp; k++) f *= byr;
  return f;
}

// Pair geometry. FP64: as pair_geom above. FP32: the minimum-image
// difference is formed in FP64 (walker coordinates are not wrapped into the
// cell and can lie many cells away) and rounded to float; r, 1/r, the knot
// and the remainder follow in FP32.
__device__ __forceinline__ void pair_geom(const DevSys &S, const Knots<double> &K,
                                          const double *x, int i, int j, double &rx, double &ry,
                                          double &r, double &byr, int &ind, double &rem) {
  rx = x[2 * i] - x[2 * j];
  ry = x[2 * i + 1] - x[2 * j + 1];
  rx = rx - S.el[0] * round(S.eli[0] * rx);
  ry = ry - S.el[1] * round(S.eli[1] * ry);
  r = sqrt(rx * rx + ry * ry);
  ind = (int)(r * K.drti);
  rem = r - ind * K.drt;
  byr = 1.0 / r;
}
__device__ __forceinline__ void pair_geom(const DevSys &S, const Knots<float> &K,
                                          const double *x, int i, int j, float &rx, float &ry,
                                          float &r, float &byr, int &ind, float &rem) {
  double dx = x[2 * i] - x[2 * j];
  double dy = x[2 * i + 1] - x[2 * j + 1];
  dx = dx - S.el[0] * round(S.eli[0] * dx);
  dy = dy - S.el[1] * round(S.eli[1] * dy);
  rx = (float)dx;
  ry = (float)dy;
  const float r2 = rx * rx + ry * ry;
  byr = rsqrtf(r2);
  r = r2 * byr;
  ind = (int)(r * K.drti);
  rem = r - (float)ind * K.drt;
}

// A lane's running sum of pair terms. FP64: a plain sum. FP32: Kahan's
// compensated sum (the rounding error of each addition is carried in c and
// subtracted from the next term), read out in FP64 as s - c.
template <class R>
struct PairSum;
template <>
struct PairSum<double> {
  double s = 0.0;
  __device__ __forceinline__ void add(double v) { s += v; }
  __device__ __forceinline__ double value() const { return s; }
};
template <>
struct PairSum<float> {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Backflow Jacobian dq_j/dx_i (2x2, symmetric) for j != i (qa of
// slater_excitations, reptation.f:10093-10168): -(eta I + eta'/r r r^T).
// ti, tj: the types of i and j.
__device__ __forceinline__ void bf_offdiag(const DevSys &S, const double *x, int i, int j,
                                           int ti, int tj, double &jxx, double &jxy,
                                           double &jyy, double &qbx, double &qby) {
  double rx, ry, r, byr, rem;
  int ind;
  pair_geom(S, x, i, j, rx, ry, r, byr, ind, rem);
  double t, dt, ddt;
  spline3(S, pair_row(S, ti, tj, ind) + PR_BF, rem, t, dt, ddt);
  double c = dt * byr;
  jxx = -(t + c * rx * rx);
  jxy = -(c * rx * ry);
  jyy = -(t + c * ry * ry);
  double w2 = c * 3.0 + ddt;  // div grad of eta(r) r, the qb term
  qbx = -w2 * rx;
  qby = -w2 * ry;
}

// d += a b for one 8x8x4 FP64 tensor-core tile (warp-wide).
__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Sum over an aligned group of L lanes (L a power of two) in a fixed
// order; every lane of the warp must call it.
template <int L>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double group8_sum(double v) { return group_sum<8>(v); }

// Deterministic block sum of K values at once; results valid in every
// thread. Uses red[0 .. K*8).
template <int K>
__device__ __forceinline__ void block_sum_n(double (&v)[K], double *red) {
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0)
#pragma unroll
    for (int k = 0; k < K; k++) red[k * 8 + w] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    double t = 0.0;
    for (int ww = 0; ww < kThreads / 32; ww++) t += red[k * 8 + ww];
    v[k] = t;
  }
  __syncthreads();
}

// Barriers of a group of threads: the whole CTA, or the `n` threads that use
// named barrier `id` (whole warps; a CTA running several walkers).
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct GroupSync {
  int id, n;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
  }
};

// Deterministic sum over a group of NT threads (NT/32 warps) with index tid
// in the group and barrier sync; red[0 .. NT/32).
template <int NT, class Sync = CtaSync>
__device__ __forceinline__ double block_sum_t(double v, double *red, Sync sync = Sync(),
                                              int tid = threadIdx.x) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = tid >> 5, l = tid & 31;
  sync();
  if (l == 0) red[w] = v;
  sync();
  double t = 0.0;
  for (int ww = 0; ww < NT / 32; ww++) t += red[ww];
  sync();
  return t;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  double a[1] = {v};
  block_sum_n<1>(a, red);
  return a[0];
}

// Adds the SM cycles since t to phase k (thread 0 only, when timers are on).
// (lead: the thread that records, thread 0 of its group.)
__device__ __forceinline__ void phase_mark(const DevSys &S, int k, long long &t, bool lead) {
  if (S.phase != nullptr && lead) {
    long long now = clock64();
    atomicAdd(&S.phase[k], (unsigned long long)(now - t));
    t = now;
  }
}
__device__ __forceinline__ void phase_mark(const DevSys &S, int k, long long &t) {
  phase_mark(S, k, t, threadIdx.x == 0);
}

// One 16-byte (cp.async.cg, through L2 only) or 8-byte global-to-shared
// copy without a register round trip, and the wait for every copy this
// thread issued.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(double *smem_dst, const double *gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// ------------------------------------------------- Gauss-Jordan inversion
//
// In-place inversion of the n x n complex matrix W (row-major, row stride
// ld) by a group of G warps (gt = 0 .. 32G-1 in the group). Step k pivots
// on column k at the unused row p of largest |re|+|im| (izamax/dcabs1,
// reptation.f:9079, 9219; ties go to the lowest row); the row is marked used
// instead of swapped. With pi(k) the pivot row of step k, the inverse is
//     A^-1(k, pi(c)) = W(pi(k), c),
// and |det A| = prod_k |pivot_k|. perm[k] = pi(k), dk[k] = |pivot_k|^2.
//
// Work split: L lanes share a row (L = largest power of two <= 32G/n, at
// most 8), each owning a contiguous slice of the columns; a thread owns at
// most 4 rows. The elimination of a slice goes in register chunks of 8 so
// the loads of a chunk are all in flight at once.
constexpr int kGjMaxRows = 4;

__device__ inline void gj_invert(double2 *W, int ld, int n, int *perm, double *dk, int *used,
                                 int *singular, int gt, int G, int bar_id, double *gval,
                                 int *gidx) {
  const int nthr = 32 * G, lane = gt & 31, wg = gt >> 5;
  int L = 1;
  while (L < 8 && 2 * L * n <= nthr) L *= 2;
  const int R = nthr / L;  // rows covered per pass
  const int my_s = gt % L, my_r0 = gt / L;
  const int h = (n + L - 1) / L;
  const int c_lo = my_s * h, c_hi = min(n, c_lo + h);
  auto gsync = [&]() {
    if (G == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
  };
  for (int r = gt; r < n; r += nthr) used[r] = 0;
  gsync();
  for (int k = 0; k < n; k++) {
    // pivot search over the unused rows (slice-0 lanes)
    double best = -1.0;
    int bi = n;
    if (my_s == 0)
#pragma unroll
      for (int i = 0; i < kGjMaxRows; i++) {
        int r = my_r0 + i * R;
        if (r < n && !used[r]) {
          double v = cabs1(W[r * ld + k]);
          if (v > best) {
            best = v;
            bi = r;
          }
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
    if (G > 1) {
      if (lane == 0) {
        gval[wg] = best;
        gidx[wg] = bi;
      }
      gsync();
      best = gval[0];
      bi = gidx[0];
      for (int w = 1; w < G; w++)
        if (gval[w] > best || (gval[w] == best && gidx[w] < bi)) {
          best = gval[w];
          bi = gidx[w];
        }
    }
    const int p = bi < n ? bi : k;  // bi == n only if every candidate is NaN
    const double2 piv = W[p * ld + k];
    const double d = piv.x * piv.x + piv.y * piv.y;
    const double rd = 1.0 / d;
    const double2 inv = make_double2(piv.x * rd, -piv.y * rd);
    // multipliers of my rows, read before anyone writes column k
    double2 f[kGjMaxRows];
#pragma unroll
    for (int i = 0; i < kGjMaxRows; i++) {
      int r = my_r0 + i * R;
      f[i] = (r < n && r != p) ? W[r * ld + k] : make_double2(0.0, 0.0);
    }
    gsync();
    if (gt == 0) {
      perm[k] = p;
      dk[k] = d;
      used[p] = 1;
      if (!(best > 0.0)) *singular = 1;
    }
    double2 *prow = W + p * ld;
    for (int c = gt; c < n; c += nthr) prow[c] = (c == k) ? inv : cmul(prow[c], inv);
    gsync();
#pragma unroll
    for (int i = 0; i < kGjMaxRows; i++) {
      const int r = my_r0 + i * R;
      if (r >= n || r == p) continue;
      double2 *__restrict__ row = W + r * ld;
      const double2 *__restrict__ pr = prow;
      const double2 fi = f[i];
      for (int c0 = c_lo; c0 < c_hi; c0 += 8) {
        double2 a[8], v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          int c = min(c0 + u, c_hi - 1);
          a[u] = pr[c];
          v[u] = row[c];
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          v[u].x -= fi.x * a[u].x - fi.y * a[u].y;
          v[u].y -= fi.x * a[u].y + fi.y * a[u].x;
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
          if (c0 + u < c_hi) row[c0 + u] = v[u];
      }
      if (k >= c_lo && k < c_hi) {
        double2 v = cmul(fi, inv);
        row[k] = make_double2(-v.x, -v.y);
      }
    }
    gsync();
  }
}

// The same inversion (same pivot rule, same outputs perm, dk, W and the
// singular flag, the same operations on every element in the same order)
// for W in global memory (determinants held in HBM), kGjBlock pivot steps
// per pass over the matrix, so that each element crosses L2 once per block
// instead of once per step. Per block of steps k0 .. k0+nb-1:
//   * panel: columns k0.. of every row are copied to shared memory (P) and
//     the nb steps run there alone: pivot search, the multipliers of every
//     row (F[j][r], the row's column-k entry before step k) and the
//     panel's own elimination; the panel then goes back to W;
//   * pivot rows: for every column c outside the panel, the pivot row of
//     step j as it is scaled at step j, Q[j][c] = (W(p_j, c) - sum over
//     earlier steps j' of F[j'][p_j] Q[j'][c]) / pivot_j (Q takes P's
//     place);
//   * every row, lanes on consecutive columns (coalesced) and four rows in
//     flight per warp: W(r, c) -= F[j][r] Q[j][c] for the block's steps in
//     order (a pivot row starts from its Q and takes the later steps only).
// scr: gj_gmem_scratch(n) bytes of shared memory.
// Gauss-Jordan in blocks of kGjBlock pivot steps for a spin of n <= 32
// orbitals in shared memory, by a group of G warps. Warp 0 factors each
// panel of kGjBlock columns in registers (lane r holds row r), with its pivot
// searches, broadcasts and eliminations warp-synchronous; then the group
// forms the block's pivot rows outside the panel, scaled as at their step
// (Q), and applies the block's steps to every row there, in step order. Three
// group barriers per block instead of one per pivot step. Pivot rule,
// outputs and per-element operations as gj_invert_gmem (the unused row of
// largest |re|+|im|, ties to the lowest row; A^-1(k, pi(c)) = W(pi(k), c)).
__device__ inline void gj_invert_panel(double2 *W, int ld, int n, int *perm, double *dk,
                                       int *singular, int gt, int G, int bar_id,
                                       double2 *scr) {
  constexpr int B = kGjBlock;
  const int nthr = 32 * G, lane = gt & 31, wg = gt >> 5;
  double2 *F = scr;              // F[j * n + r]: multiplier of row r at step j
  double2 *Q = scr + B * n;      // Q[j * n + c]: scaled pivot rows outside the panel
  double2 *I = scr + 2 * B * n;  // I[j]: 1 / pivot of step j
  int *PJ = reinterpret_cast<int *>(I + B);  // PJ[j]: pivot row of step j
  auto gsync = [&]() {
    if (G == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
  };
  auto sub = [](double2 &v, double2 f, double2 a) {
    v.x -= f.x * a.x - f.y * a.y;
    v.y -= f.x * a.y + f.y * a.x;
  };
  bool used = lane >= n;  // warp 0: row `lane` has been a pivot
  for (int k0 = 0; k0 < n; k0 += B) {
    const int nb = min(B, n - k0);
    if (wg == 0) {
      const int r = lane;
      const bool valid = r < n;
      double2 pv[B];
#pragma unroll
      for (int j = 0; j < B; j++)
        pv[j] = (valid && j < nb) ? W[r * ld + k0 + j] : make_double2(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < B; j++) {
        if (j >= nb) break;
        unsigned long long key = 0ull;
        if (!used) {
          const double a = fabs(pv[j].x) + fabs(pv[j].y);
          key = ((unsigned long long)__double_as_longlong(a) & ~0xFFull) | (unsigned)(255 - r);
        }
        {
          const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
          const unsigned hm = __reduce_max_sync(0xffffffffu, hi);
          const unsigned lm = __reduce_max_sync(0xffffffffu, hi == hm ? lo : 0u);
          key = ((unsigned long long)hm << 32) | lm;
        }
        // every unused row < n has 255 - r in its key's low byte, so p is
        // such a row at every step, an exactly zero or NaN column included
        const int p = 255 - (int)(key & 0xFFull);
        double2 pr[B];
#pragma unroll
        for (int jj = 0; jj < B; jj++) {
          pr[jj].x = __shfl_sync(0xffffffffu, pv[jj].x, p);
          pr[jj].y = __shfl_sync(0xffffffffu, pv[jj].y, p);
        }
        const double2 piv = pr[j];
        const double d = piv.x * piv.x + piv.y * piv.y;
        const double rd = 1.0 / d;
        const double2 inv = make_double2(piv.x * rd, -piv.y * rd);
        if (lane == 0) {
          perm[k0 + j] = p;
          dk[k0 + j] = d;
          I[j] = inv;
          PJ[j] = p;
          if ((key >> 8) == 0ull) *singular = 1;  // every candidate exactly zero
        }
        if (r == p) {
          used = true;
#pragma unroll
          for (int jj = 0; jj < B; jj++) pv[jj] = (jj == j) ? inv : cmul(pv[jj], inv);
        } else if (valid) {
          const double2 fi = pv[j];
          F[j * n + r] = fi;
#pragma unroll
          for (int jj = 0; jj < B; jj++)
            if (jj != j) sub(pv[jj], fi, cmul(pr[jj], inv));
          const double2 t = cmul(fi, inv);
          pv[j] = make_double2(-t.x, -t.y);
        }
      }
#pragma unroll
      for (int j = 0; j < B; j++)
        if (valid && j < nb) W[r * ld + k0 + j] = pv[j];
    }
    gsync();
    // the block's pivot rows outside the panel, as scaled at their step
    for (int c = gt; c < n; c += nthr) {
      if (c >= k0 && c < k0 + nb) continue;
      for (int j = 0; j < nb; j++) {
        const int prow = PJ[j];
        double2 x = W[prow * ld + c];
        for (int jj = 0; jj < j; jj++) sub(x, F[jj * n + prow], Q[jj * n + c]);
        Q[j * n + c] = cmul(x, I[j]);
      }
    }
    gsync();
    // every row, outside the panel: the block's steps in order
    for (int r0 = wg; r0 < n; r0 += 4 * G) {
      int role[4];  // -2: no row, -1: not a pivot of the block, j: pivot of step j
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = r0 + i * G;
        role[i] = r < n ? -1 : -2;
        for (int j = 0; j < nb; j++)
          if (PJ[j] == r) role[i] = j;
      }
      for (int c = lane; c < n; c += 32) {
        if (c >= k0 && c < k0 + nb) continue;
        double2 v[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
          v[i] = role[i] == -2  ? make_double2(0.0, 0.0)
                 : role[i] >= 0 ? Q[role[i] * n + c]
                                : W[(r0 + i * G) * ld + c];
        for (int j = 0; j < nb; j++) {
          const double2 a = Q[j * n + c];
#pragma unroll
          for (int i = 0; i < 4; i++)
            if (role[i] != -2 && j > role[i]) sub(v[i], F[j * n + r0 + i * G], a);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (role[i] != -2) W[(r0 + i * G) * ld + c] = v[i];
      }
    }
    gsync();
  }
}

__device__ inline void gj_invert_gmem(double2 *W, int ld, int n, int *perm, double *dk,
                                      int *used, int *singular, int gt, int G, int bar_id,
                                      double *gval, int *gidx, double2 *scr) {
  constexpr int B = kGjBlock;
  const int nthr = 32 * G, lane = gt & 31, wg = gt >> 5;
  double2 *P = scr;              // P[r * B + j]: panel
  double2 *Q = scr;              // Q[j * n + c]: scaled pivot rows (after the panel)
  double2 *F = scr + B * n;      // F[j * n + r]: multipliers
  double2 *I = scr + 2 * B * n;  // I[j]: 1 / pivot of step j
  int *PJ = reinterpret_cast<int *>(I + B);  // PJ[j]: pivot row of step j
  auto gsync = [&]() {
    if (G == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
  };
  auto sub = [](double2 &v, double2 f, double2 a) {
    v.x -= f.x * a.x - f.y * a.y;
    v.y -= f.x * a.y + f.y * a.x;
  };
  for (int r = gt; r < n; r += nthr) used[r] = 0;
  for (int k0 = 0; k0 < n; k0 += B) {
    const int nb = min(B, n - k0);
    for (int e = gt; e < n * nb; e += nthr) {
      const int r = e / nb, j = e - r * nb;
      P[r * B + j] = W[(size_t)r * ld + k0 + j];
    }
    gsync();
    for (int j = 0; j < nb; j++) {
      const int k = k0 + j;
      double best = -1.0;
      int bi = n;
      for (int r = gt; r < n; r += nthr)
        if (!used[r]) {
          const double a = cabs1(P[r * B + j]);
          if (a > best) {
            best = a;
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
      if (G > 1) {
        if (lane == 0) {
          gval[wg] = best;
          gidx[wg] = bi;
        }
        gsync();
        best = gval[0];
        bi = gidx[0];
        for (int w = 1; w < G; w++)
          if (gval[w] > best || (gval[w] == best && gidx[w] < bi)) {
            best = gval[w];
            bi = gidx[w];
          }
      }
      const int p = bi < n ? bi : k;  // bi == n only if every candidate is NaN
      const double2 piv = P[p * B + j];
      const double d = piv.x * piv.x + piv.y * piv.y;
      const double rd = 1.0 / d;
      const double2 inv = make_double2(piv.x * rd, -piv.y * rd);
      for (int r = gt; r < n; r += nthr) F[j * n + r] = P[r * B + j];
      gsync();  // F; gval and gidx are read
      if (gt == 0) {
        perm[k] = p;
        dk[k] = d;
        used[p] = 1;
        I[j] = inv;
        PJ[j] = p;
        if (!(best > 0.0)) *singular = 1;
      }
      if (gt < nb) P[p * B + gt] = (gt == j) ? inv : cmul(P[p * B + gt], inv);
      gsync();
      for (int e = gt; e < n * nb; e += nthr) {
        const int r = e / nb, jj = e - r * nb;
        if (r == p) continue;
        const double2 fi = F[j * n + r];
        double2 v;
        if (jj == j) {
          const double2 t = cmul(fi, inv);
          v = make_double2(-t.x, -t.y);
        } else {
          v = P[r * B + jj];
          sub(v, fi, P[p * B + jj]);
        }
        P[r * B + jj] = v;
      }
      gsync();
    }
    for (int e = gt; e < n * nb; e += nthr) {
      const int r = e / nb, j = e - r * nb;
      W[(size_t)r * ld + k0 + j] = P[r * B + j];
    }
    gsync();  // P is free: Q takes its place
    // the block's pivot rows outside the panel, as scaled at their step
    for (int c = gt; c < n; c += nthr) {
      if (c >= k0 && c < k0 + nb) continue;
      for (int j = 0; j < nb; j++) {
        const int pr = PJ[j];
        double2 x = W[(size_t)pr * ld + c];
        for (int jj = 0; jj < j; jj++) sub(x, F[jj * n + pr], Q[jj * n + c]);
        Q[j * n + c] = cmul(x, I[j]);
      }
    }
    gsync();
    // every row, outside the panel: the block's steps in order
    for (int r0 = wg; r0 < n; r0 += 4 * G) {
      int role[4];  // -2: no row, -1: not a pivot of the block, j: pivot of step j
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = r0 + i * G;
        role[i] = r < n ? -1 : -2;
        for (int j = 0; j < nb; j++)
          if (PJ[j] == r) role[i] = j;
      }
      for (int c = lane; c < n; c += 32) {
        if (c >= k0 && c < k0 + nb) continue;
        double2 v[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
          v[i] = role[i] == -2  ? make_double2(0.0, 0.0)
                 : role[i] >= 0 ? Q[role[i] * n + c]
                                : W[(size_t)(r0 + i * G) * ld + c];
        for (int j = 0; j < nb; j++) {
          const double2 a = Q[j * n + c];
#pragma unroll
          for (int i = 0; i < 4; i++)
            if (role[i] != -2 && j > role[i]) sub(v[i], F[j * n + r0 + i * G], a);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (role[i] != -2) W[(size_t)(r0 + i * G) * ld + c] = v[i];
      }
    }
    gsync();
  }
}

// 1/d by Newton-Raphson from the hardware estimate (rcp.approx.ftz.f64):
// each step y <- y + y (1 - d y) doubles the number of correct bits, and
// two steps bring the estimate to within a few units in the last place.
// Branch-free, unlike the correctly rounded division, so the scheduler can
// overlap it with independent work. d = 0 or subnormal gives NaN.
__device__ __forceinline__ double rcp_newton(double d) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
  double e = fma(-d, y, 1.0);
  y = fma(y, e, y);
  e = fma(-d, y, 1.0);
  return fma(y, e, y);
}

// The same inversion (same pivot rule up to ties, same outputs perm, dk, W
// and the singular flag) with every row held in registers: thread gt of
// the 32G-thread group (G = 4 or 8) owns row r = gt / L and the columns
// s kGjCols + j (s = gt % L, j < kGjCols) with L = gj_reg_lanes(n, 32G).
// Step k (column k, owned by lane k / kGjCols of each row, register
// k % kGjCols):
//   * the owner lane forms the row's pivot key, the top 32 bits of the
//     double |re|+|im| (non-negative doubles order as integers) with the
//     low byte replaced by 255 - r (ties within 2^-12 relative go to the
//     lowest row; rows already used give 0), and the reciprocal of its
//     candidate, 1 / pivot = conj(pivot) / |pivot|^2 (rcp_newton);
//   * one redux gives the warp's best row, which publishes its columns,
//     reciprocal and |pivot|^2 to the warp's slot, lane 0 the key;
//   * one group barrier; every thread takes the best of the G keys (one or
//     two 16-byte loads), the pivot row's slot, and updates its registers
//     v -= (f / pivot) pivot_row, column k becoming -f / pivot.
// The iteration is software-pipelined: after the barrier of step k a
// thread first updates the register of column k+1, then forms step k+1's
// key and reciprocal and starts its redux, then updates its other columns
// (their loads and FMAs hide the redux and the reciprocal), then publishes
// for step k+1. The pivot row is left unscaled (its column k set to 1) and
// every row is divided by its own pivot at the end, which gives the
// normalised Gauss-Jordan result. Slots and keys are double-buffered by
// the parity of k: the publications for step k+1 follow the barrier of
// step k, after every read of step k-1.
// slots: 2 G gj_reg_slot(L) double2; keys: 2 G unsigned, 16-byte aligned
// (G is 4 or 8: the keys of a step are one or two 16-byte words).
__device__ inline void gj_invert_reg(double2 *W, int ld, int n, int *perm, double *dk,
                                     int *singular, int gt, int G, int bar_id, double2 *slots,
                                     unsigned *keys) {
  constexpr int C = kGjCols;
  const int nthr = 32 * G, lane = gt & 31, wg = gt >> 5;
  const int L = gj_reg_lanes(n, nthr);
  const int r = gt / L, s = gt - (gt / L) * L;
  const int rpw_log = 5 - (31 - __clz(L));  // log2(32 / L): rows per warp
  const int SL = gj_reg_slot(L), HDR = L * (C + 1);
  auto gsync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory"); };
  double2 v[C];
#pragma unroll
  for (int j = 0; j < C; j++) {
    const int c = s * C + j;
    v[j] = (r < n && c < n) ? W[r * ld + c] : make_double2(0.0, 0.0);
  }
  bool used = r >= n;
  double2 my_inv = make_double2(1.0, 0.0);
  auto pivot_key = [&](double2 f, bool own) -> unsigned {
    const double a = fabs(f.x) + fabs(f.y);
    return (own && !used) ? ((unsigned)__double2hiint(a) & ~0xFFu) | (unsigned)(255 - r) : 0u;
  };
  // step k's candidates: the warp's best row, its reciprocal and |pivot|^2
  auto publish = [&](int k, unsigned wk, bool own, double2 f0, double cd, double crd) {
    const int buf = k & 1;
    double2 *mys = slots + (buf * G + wg) * SL;
    if (wk != 0u && r == 255 - (int)(wk & 0xFFu)) {
#pragma unroll
      for (int jj = 0; jj < C; jj++) mys[s * (C + 1) + jj] = v[jj];
      if (own) {
        mys[HDR] = make_double2(f0.x * crd, -f0.y * crd);
        mys[HDR + 1] = make_double2(cd, 0.0);
      }
    }
    if (lane == 0) keys[buf * G + wg] = wk;
  };
  double fx, fy;  // this row's entry in the pivot column (the multiplier source)
  {
    const bool own = s == 0;
    const double2 f0 = v[0];
    const double cd = f0.x * f0.x + f0.y * f0.y;
    const unsigned wk = __reduce_max_sync(0xffffffffu, pivot_key(f0, own));
    publish(0, wk, own, f0, cd, rcp_newton(cd));
    fx = __shfl_sync(0xffffffffu, f0.x, 0, L);
    fy = __shfl_sync(0xffffffffu, f0.y, 0, L);
  }
#pragma unroll 1
  for (int sb = 0; sb * C < n; sb++) {
    const bool own = s == sb;
#pragma unroll
    for (int j = 0; j < C; j++) {
      const int k = sb * C + j;
      const int buf = k & 1;
      gsync();
      unsigned best;
      {
        const uint4 k4 = *reinterpret_cast<const uint4 *>(keys + buf * G);
        best = max(max(k4.x, k4.y), max(k4.z, k4.w));
        if (G > 4) {
          const uint4 k8 = *reinterpret_cast<const uint4 *>(keys + buf * G + 4);
          best = max(best, max(max(k8.x, k8.y), max(k8.z, k8.w)));
        }
      }
      // Every unused row's key has 255 - r in its low byte, so p is an
      // unused row < n at every step, an exactly zero or NaN column included.
      const int p = 255 - (int)(best & 0xFFu);
      const double2 *ps = slots + (buf * G + (p >> rpw_log)) * SL;
      const double2 inv = ps[HDR];
      if (gt == 0) {
        perm[k] = p;
        dk[k] = ps[HDR + 1].x;
        if ((best >> 8) == 0u) *singular = 1;  // every candidate zero (or subnormal)
      }
      const bool piv = r == p;
      used = used || piv;
      my_inv = piv ? inv : my_inv;
      double2 fac = cmul(make_double2(fx, fy), inv);
      if (piv) fac = make_double2(0.0, 0.0);
      // column k+1 first: step k+1's key depends on it
      const int jn = (j + 1) % C;
      {
        const double2 b = ps[s * (C + 1) + jn];
        v[jn].x = fma(-fac.x, b.x, fma(fac.y, b.y, v[jn].x));
        v[jn].y = fma(-fac.x, b.y, fma(-fac.y, b.x, v[jn].y));
      }
      const int sbn = j + 1 == C ? sb + 1 : sb;
      const bool ownn = s == sbn;
      const double2 f0 = v[jn];
      const double cd = f0.x * f0.x + f0.y * f0.y;
      const unsigned wk = __reduce_max_sync(0xffffffffu, pivot_key(f0, ownn));
#pragma unroll
      for (int jj = 0; jj < C; jj++) {
        if (jj == jn) continue;
        const double2 b = ps[s * (C + 1) + jj];
        v[jj].x = fma(-fac.x, b.x, fma(fac.y, b.y, v[jj].x));
        v[jj].y = fma(-fac.x, b.y, fma(-fac.y, b.x, v[jj].y));
      }
      if (own) v[j] = piv ? make_double2(1.0, 0.0) : make_double2(-fac.x, -fac.y);
      const double crd = rcp_newton(cd);
      if (k + 1 >= n) break;
      publish(k + 1, wk, ownn, f0, cd, crd);
      fx = __shfl_sync(0xffffffffu, f0.x, sbn, L);
      fy = __shfl_sync(0xffffffffu, f0.y, sbn, L);
    }
  }
#pragma unroll
  for (int j = 0; j < C; j++) {
    const int c = s * C + j;
    if (r < n && c < n) W[r * ld + c] = cmul(v[j], my_inv);
  }
  gsync();
}

// rho_k per rhok slot (distances, reptation.f:4225-4243) by threads
// t0 .. t0+nthr-1.
// nthr is a multiple of 32 (whole warps): each (type, k) item is summed by
// a group of LG lanes (8, or the pair kernel's lanes per particle), lane l
// taking particles l, l+LG, ..., then a fixed shuffle tree.
template <int LG = kGroup>
__device__ inline void compute_rhok(const DevSys &S, const EvalSmem &m, int t, int nthr) {
  const int total = S.nt * S.nk, per_round = nthr / LG, l8 = t & (LG - 1);
  for (int e0 = 0; e0 < total; e0 += per_round) {
    const int e = e0 + t / LG;
    const int ty = e < total ? e / S.nk : 0, k = e - ty * S.nk;
    const bool on = e < total && S.irhok[ty] != 0;
    double c = 0.0, sn = 0.0;
    if (on) {
      const double kx = __ldg(S.kvec + 2 * k), ky = __ldg(S.kvec + 2 * k + 1);
      for (int i = S.ipfrst[ty] + l8; i < S.ipfrst[ty] + S.np[ty]; i += LG) {
        double kr = kx * m.x[2 * i] + ky * m.x[2 * i + 1];
        double sv, cv;
        sincos(kr, &sv, &cv);
        c += cv;
        sn += sv;
      }
    }
    c = group_sum<LG>(c);
    sn = group_sum<LG>(sn);
    if (on && l8 == 0) {
      const int slot = S.irhok[ty] - 1;
      m.rhok[2 * (slot * S.nk + k)] = c;
      m.rhok[2 * (slot * S.nk + k) + 1] = sn;
    }
  }
}

// rho_k of the pair kernels when every k vector is on the reciprocal lattice
// (DevSys::rk_lat): with k = 2 pi (n1 / Lx, n2 / Ly), exp(i k.x) =
// X_{n1}(x) Y_{n2}(y), X_p(x) = exp(2 pi i p x / Lx), and each particle's
// X_0 .. X_{rk_p1}, Y_0 .. Y_{rk_p2} are built once by repeated complex
// multiplication (conjugates for negative indices), so a (k, particle) term
// is one complex product instead of a sincos. Items, lanes and the shuffle
// tree as compute_rhok; each term agrees with its sincos to a few ulp.
// Threads t .. t+nthr-1 of the group whose barrier is sync.
template <int LG, class Sync>
__device__ inline void compute_rhok_lattice(const DevSys &S, const EvalSmem &m, int t, int nthr,
                                            Sync sync) {
  const int N = S.N, P1 = S.rk_p1, P2 = S.rk_p2;
  double2 *X = m.rkt, *Y = m.rkt + (size_t)(P1 + 1) * N;
  for (int i = t; i < N; i += nthr) {
    double sx, cx, sy, cy;
    sincospi(2.0 * (m.x[2 * i] * S.eli[0]), &sx, &cx);
    sincospi(2.0 * (m.x[2 * i + 1] * S.eli[1]), &sy, &cy);
    const double2 bx = make_double2(cx, sx), by = make_double2(cy, sy);
    double2 px = make_double2(1.0, 0.0), py = px;
    X[i] = px;
    Y[i] = py;
    for (int p = 1; p <= P1; p++) {
      px = cmul(px, bx);
      X[(size_t)p * N + i] = px;
    }
    for (int p = 1; p <= P2; p++) {
      py = cmul(py, by);
      Y[(size_t)p * N + i] = py;
    }
  }
  sync();
  const double c1 = S.el[0] * 0.15915494309189535, c2 = S.el[1] * 0.15915494309189535;
  const int total = S.nt * S.nk, per_round = nthr / LG, l8 = t & (LG - 1);
  for (int e0 = 0; e0 < total; e0 += per_round) {
    const int e = e0 + t / LG;
    const int ty = e < total ? e / S.nk : 0, k = e - ty * S.nk;
    const bool on = e < total && S.irhok[ty] != 0;
    double c = 0.0, sn = 0.0;
    if (on) {
      const int n1 = __double2int_rn(__ldg(S.kvec + 2 * k) * c1);
      const int n2 = __double2int_rn(__ldg(S.kvec + 2 * k + 1) * c2);
      const double2 *xp = X + (size_t)abs(n1) * N, *yp = Y + (size_t)abs(n2) * N;
      for (int i = S.ipfrst[ty] + l8; i < S.ipfrst[ty] + S.np[ty]; i += LG) {
        double2 xv = xp[i], yv = yp[i];
        if (n1 < 0) xv.y = -xv.y;
        if (n2 < 0) yv.y = -yv.y;
        c += xv.x * yv.x - xv.y * yv.y;
        sn += xv.x * yv.y + xv.y * yv.x;
      }
    }
    c = group_sum<LG>(c);
    sn = group_sum<LG>(sn);
    if (on && l8 == 0) {
      const int slot = S.irhok[ty] - 1;
      m.rhok[2 * (slot * S.nk + k)] = c;
      m.rhok[2 * (slot * S.nk + k) + 1] = sn;
    }
  }
}

// rho_k in a pair kernel: from the lattice tables when the group's shared
// memory has them, else one sincos per (k, particle).
template <int LG, class Sync>
__device__ inline void pair_rhok(const DevSys &S, const EvalSmem &m, int t, int nthr, Sync sync) {
  if (m.rkt)
    compute_rhok_lattice<LG>(S, m, t, nthr, sync);
  else
    compute_rhok<LG>(S, m, t, nthr);
}

// ---------------------------------------------------------- the evaluation
//
// Input: m.x holds the configuration. Output (in shared memory): m.g (drift
// -grad ln psi), hl[nt] (-lap ln psi per type), props[nprops], *sign.
// eval_walker (= eval_pairs then eval_det) returns a status word (ST_*),
// identical in all threads.
//
// Pair passes A and B: writes m.{ltf, g, lap, vp, G3, S3, q, Sb, qbd} and
// zeroes m.{gd, lapd, ph2, ph2d}. With pout (backflow), also the backflow
// spline values of every pair i < j, laid out as in MoveScratch.
// NT threads (a multiple of 32) run the passes; the pair rows (layout
// RowLayout<R>) are read at `rows`, from shared memory when kSh.
// R is the precision of the u2 and v2 terms: double, or float with the pair
// vector from the FP64 minimum image and each lane's sums compensated
// (PairSum); the lanes' sums and all that follows are FP64. The u3 and
// backflow terms are FP64 in both: FP32 u3 terms put the local energy off
// by up to 2e-6 Ry per electron, and an FP32 backflow displacement error
// reaches it through the determinant amplified by the inverse square of the
// distance to the nearest node.
// Sync is the barrier of the NT threads (the CTA, or a named-barrier group
// of a CTA that runs several walkers); tid is the thread's index among them.
template <int NT, bool kSh, class R = double, class Sync = CtaSync, int LG = kGroup>
__device__ inline void eval_pairs(const DevSys &S, const EvalSmem &m, long long &tph,
                                  double *pout, const R *rows, Sync sync = Sync(),
                                  int tid = threadIdx.x) {
  using Lay = RowLayout<R>;
  const int N = S.N;
  const int lane8 = tid & (LG - 1);
  const int per_round = NT / LG;
  const size_t NP = pair_count(N);
  constexpr int RS = kSh ? Lay::sstride : Lay::gstride;
  constexpr bool kF64 = sizeof(R) == 8;
  const Knots<R> K(S);

  // ---- pass A: pair sums of u2, the pair part of u3, u3 G vectors and S,
  // backflow displacement, Jacobian diagonal and Laplacian, pair potential.
  for (int base = 0; base < N; base += per_round) {
    int i = base + tid / LG;
    bool valid = i < N;
    int ti = valid ? type_of(S, i) : 0;
    PairSum<R> ltf, gx, gy, lap, vp;
    PairSum<double> ltf3, gx3, gy3, lap3;  // the u3 terms' share when R = float
    PairSum<double> Gx, Gy, s3xx, s3xy, s3yy;
    PairSum<double> qx, qy, sbxx, sbxy, sbyy, qbx, qby;
    if (valid) {
      for (int j = lane8; j < N; j += LG) {
        if (j == i) continue;
        int tj = type_of(S, j);
        R rx, ry, r, byr, rem;
        double rxd = 0, ryd = 0, rd = 0, byrd = 0, remd = 0;
        int ind;
        if (kF64 || S.has_bf || S.has_u3) {  // FP64 geometry (the u3 and backflow terms)
          pair_geom(S, Knots<double>(S), m.x, i, j, rxd, ryd, rd, byrd, ind, remd);
          rx = (R)rxd;
          ry = (R)ryd;
          r = (R)rd;
          byr = (R)byrd;
          rem = (R)remd;
        } else {
          pair_geom(S, K, m.x, i, j, rx, ry, r, byr, ind, rem);
        }
        const R *row = pair_row<RS>(S, rows, ti, tj, ind);
        if (S.has_u2) {
          R t, dt, ddt;
          spline3<kSh>(K, row + Lay::u2, rem, t, dt, ddt);
          ltf.add((R)0.5 * t);
          R dtr = dt * byr;
          gx.add(dtr * rx);
          gy.add(dtr * ry);
          lap.add(ddt + dtr);
        }
        if (S.has_u3) {
          double t, dt, ddt;
          spline3<kSh>(Knots<double>(S), reinterpret_cast<const double *>(row + Lay::u3), remd, t,
                       dt, ddt);
          Gx.add(-t * rxd);
          Gy.add(-t * ryd);
          double c = dt * byrd;
          s3xx.add(t + c * rxd * rxd);
          s3xy.add(c * rxd * ryd);
          s3yy.add(t + c * ryd * ryd);
          // the two-body piece (xi r)^2 removed from sum |G|^2 (three_body :2824-2832)
          double d3 = 2.0 * (t * t + 4.0 * rd * t * dt + rd * rd * (dt * dt + ddt * t));
          double c3 = 2.0 * t * (t + rd * dt);
          double tr = t * rd;
          if constexpr (kF64) {
            ltf.add(0.5 * tr * tr);
            gx.add(c3 * rxd);
            gy.add(c3 * ryd);
            lap.add(d3 + c3);
          } else {
            ltf3.add(0.5 * tr * tr);
            gx3.add(c3 * rxd);
            gy3.add(c3 * ryd);
            lap3.add(d3 + c3);
          }
        }
        if (S.has_bf && !S.bf_zero) {
          double t, dt, ddt;
          spline3<kSh>(Knots<double>(S), reinterpret_cast<const double *>(row + Lay::bf), remd, t,
                       dt, ddt);
          qx.add(t * rxd);
          qy.add(t * ryd);
          double c = dt * byrd;
          sbxx.add(t + c * rxd * rxd);
          sbxy.add(c * rxd * ryd);
          sbyy.add(t + c * ryd * ryd);
          double w2 = dt * byrd * 3.0 + ddt;
          qbx.add(w2 * rxd);
          qby.add(w2 * ryd);
          if (pout && i < j) {
            const size_t e = pair_tri(N, i, j);
            pout[e] = t;
            pout[NP + e] = c;
            pout[2 * NP + e] = w2;
          }
        }
        if (S.has_v2)
          vp.add((R)0.5 * spline0<kSh>(K, row + Lay::v2, S.tab_iexp[S.iv2[ti][tj]], rem, byr));
      }
    }
    double ltf_v = ltf.value(), gx_v = gx.value(), gy_v = gy.value(), lap_v = lap.value();
    if (!kF64 && S.has_u3) {
      ltf_v += ltf3.value();
      gx_v += gx3.value();
      gy_v += gy3.value();
      lap_v += lap3.value();
    }
    const double ltf_s = group_sum<LG>(ltf_v);
    const double gx_s = group_sum<LG>(gx_v);
    const double gy_s = group_sum<LG>(gy_v);
    const double lap_s = group_sum<LG>(lap_v);
    const double vp_s = group_sum<LG>(vp.value());
    double Gx_s = 0, Gy_s = 0, s3xx_s = 0, s3xy_s = 0, s3yy_s = 0;
    if (S.has_u3) {
      Gx_s = group_sum<LG>(Gx.value());
      Gy_s = group_sum<LG>(Gy.value());
      s3xx_s = group_sum<LG>(s3xx.value());
      s3xy_s = group_sum<LG>(s3xy.value());
      s3yy_s = group_sum<LG>(s3yy.value());
    }
    double qx_s = 0, qy_s = 0, sbxx_s = 0, sbxy_s = 0, sbyy_s = 0, qbx_s = 0, qby_s = 0;
    if (S.has_bf) {
      qx_s = group_sum<LG>(qx.value());
      qy_s = group_sum<LG>(qy.value());
      sbxx_s = group_sum<LG>(sbxx.value());
      sbxy_s = group_sum<LG>(sbxy.value());
      sbyy_s = group_sum<LG>(sbyy.value());
      qbx_s = group_sum<LG>(qbx.value());
      qby_s = group_sum<LG>(qby.value());
    }
    if (valid && lane8 == 0) {
      m.ltf[i] = ltf_s;
      m.g[2 * i] = gx_s;
      m.g[2 * i + 1] = gy_s;
      m.lap[i] = lap_s;
      m.vp[i] = vp_s;
      if (S.has_u3) {
        m.G3[2 * i] = Gx_s;
        m.G3[2 * i + 1] = Gy_s;
        m.S3[3 * i] = s3xx_s;
        m.S3[3 * i + 1] = s3xy_s;
        m.S3[3 * i + 2] = s3yy_s;
      }
      m.q[2 * i] = m.x[2 * i] + qx_s;
      m.q[2 * i + 1] = m.x[2 * i + 1] + qy_s;
      m.Sb[3 * i] = sbxx_s;
      m.Sb[3 * i + 1] = sbxy_s;
      m.Sb[3 * i + 2] = sbyy_s;
      m.qbd[2 * i] = qbx_s;
      m.qbd[2 * i + 1] = qby_s;
      m.gd[2 * i] = 0.0;
      m.gd[2 * i + 1] = 0.0;
      m.lapd[i] = 0.0;
      m.ph2[i] = 0.0;
      m.ph2d[i] = 0.0;
    }
  }
  sync();
  phase_mark(S, PH_PAIRS, tph, tid == 0);

  // ---- pass B: u3 gradient and Laplacian from the G vectors (FP64).
  if (S.has_u3) {
    for (int base = 0; base < N; base += per_round) {
      int k = base + tid / LG;
      bool valid = k < N;
      int tk = valid ? type_of(S, k) : 0;
      double gx = 0, gy = 0, lap = 0;
      double Gkx = valid ? m.G3[2 * k] : 0.0, Gky = valid ? m.G3[2 * k + 1] : 0.0;
      if (valid) {
        for (int j = lane8; j < N; j += LG) {
          if (j == k) continue;
          int tj = type_of(S, j);
          double rx, ry, r, byr, rem;
          int ind;
          pair_geom(S, Knots<double>(S), m.x, k, j, rx, ry, r, byr, ind, rem);
          double t, dt, ddt;
          spline3<kSh>(Knots<double>(S),
                       reinterpret_cast<const double *>(pair_row<RS>(S, rows, tk, tj, ind) + Lay::u3),
                       rem, t, dt, ddt);
          double c = dt * byr;
          double mxx = t + c * rx * rx, mxy = c * rx * ry, myy = t + c * ry * ry;
          double dGx = Gkx - m.G3[2 * j], dGy = Gky - m.G3[2 * j + 1];
          gx += mxx * dGx + mxy * dGy;
          gy += mxy * dGx + myy * dGy;
          double w = ddt + 3.0 * c;
          lap += w * (rx * dGx + ry * dGy) - (mxx * mxx + 2.0 * mxy * mxy + myy * myy);
        }
      }
      gx = group_sum<LG>(gx);
      gy = group_sum<LG>(gy);
      lap = group_sum<LG>(lap);
      if (valid && lane8 == 0) {
        double sxx = m.S3[3 * k], sxy = m.S3[3 * k + 1], syy = m.S3[3 * k + 2];
        m.g[2 * k] += gx;
        m.g[2 * k + 1] += gy;
        m.lap[k] += lap - (sxx * sxx + 2.0 * sxy * sxy + syy * syy);
        m.ltf[k] -= 0.5 * (Gkx * Gkx + Gky * Gky);
      }
    }
    sync();
    phase_mark(S, PH_U3, tph, tid == 0);
  }
}

// Everything after the pair passes: determinants (orbitals, inversion,
// F, drift, Laplacian with the cross term), rho_k, assembly. With pin, the
// backflow Jacobian blocks take the pair spline values written by
// eval_pairs(pout) instead of evaluating them again; with inv_in, the
// orbitals and their inversion come from orb_inv_kernel.
// kSeq (with inv_in, m carved with one_buf): the spins' orbitals and
// inverses are copied in turn into the one buffer, each just before its
// spin's F matrix, since the cross-term matrix M of the spin before it
// overlays the buffer until its last chunk.
template <bool kGmat = false, bool kSeq = false>
__device__ inline int eval_det(const DevSys &S, const EvalSmem &m, double *hl, double *props,
                               double *sign, long long &tph, const double *pin,
                               const double *rhok_in = nullptr,
                               const double *inv_in = nullptr) {
  const int tid = threadIdx.x;
  // rho_k of both slots: copied when given (MoveScratch), else summed
  auto rhok = [&](int t0, int nthr) {
    if (rhok_in && kGmat) {  // plain loads: the HBM-determinant instance's registers are full
      for (int e = t0; e < 4 * S.nk; e += nthr) m.rhok[e] = rhok_in[e];
    } else if (rhok_in) {
      for (int e = t0; e < 4 * S.nk; e += nthr) cp_async8(m.rhok + e, rhok_in + e);
      cp_async_wait_all();
    } else {
      compute_rhok(S, m, t0, nthr);
    }
  };
  const int N = S.N, nt = S.nt;
  const int lane8 = tid & (kGroup - 1);
  const size_t NP = pair_count(N);

  // ---- backflow Slater determinants (slater_excitations, reptation.f:9967)
  int status = ST_OK;
  double logdet_sum = 0.0, ltf_j = 0.0;  // ltf_j: sum of the Jastrow -ln psi terms
  if (S.has_bf) {
    const int n = S.nmax;
    bool reg_path = true;  // the phase the log|det| sum below is counted in
    if (kSeq || inv_in) {  // (kSeq has inv_in: the in-kernel inversion is compiled out)
      // orbitals, inverse, |pivot|^2, pivot rows and singular flags of both
      // spins from orb_inv_kernel (the walker's move scratch)
      const double *src = inv_in;
      for (int sp = 0; sp < nt; sp++) {
        const int ns = S.np[sp], ld = ws_ld(ns);
        const double2 *sA = reinterpret_cast<const double2 *>(src);
        const double2 *sW = sA + (size_t)ns * ns;
        const double *sD = reinterpret_cast<const double *>(sW + (size_t)ns * ld);
        double2 *dA = sp ? m.A[1] : m.A[0], *dW = sp ? m.W[1] : m.W[0];
        // asynchronous 16-byte global-to-shared copies, all in flight at once
        // (kSeq: the first spin's now, the others' before their F matrix)
        if (!kSeq || sp == 0) {
          for (int e = tid; e < ns * ns; e += kThreads) cp_async16(dA + e, sA + e);
          for (int e = tid; e < ns * ld; e += kThreads) cp_async16(dW + e, sW + e);
        }
        for (int k = tid; k < ns; k += kThreads) {
          (sp ? m.dk[1] : m.dk[0])[k] = sD[k];
          (sp ? m.perm[1] : m.perm[0])[k] = (int)sD[ns + k];
        }
        if (tid == sp) m.iscal[sp] = sD[2 * ns] != 0.0;
        src += inv_spin_doubles(ns);
      }
      if (tid == 1 && nt == 1) m.iscal[1] = 0;
      for (int e = tid; e < 2 * n; e += kThreads) m.gsh[e] = __ldg(S.gvec + e);
      cp_async_wait_all();
      __syncthreads();
      phase_mark(S, PH_ORBITALS, tph);
      rhok(tid, kThreads);
      __syncthreads();
    } else {
      // orbitals of both spins (paho_orbitals, reptation.f:10298-10315)
      int tot = 0;
      for (int sp = 0; sp < nt; sp++) tot += S.np[sp] * S.np[sp];
      for (int e = tid; e < tot; e += kThreads) {
        int sp = 0, ee = e;
        if (nt > 1 && ee >= S.np[0] * S.np[0]) {
          ee -= S.np[0] * S.np[0];
          sp = 1;
        }
        const int ns = S.np[sp], ld = ws_ld(ns), f0 = S.ipfrst[sp];
        int k = ee % ns, j = ee / ns;
        double gkx = __ldg(S.gvec + 2 * k), gky = __ldg(S.gvec + 2 * k + 1);
        double kr = m.q[2 * (f0 + j)] * gkx + m.q[2 * (f0 + j) + 1] * gky;
        double sv, cv;
        sincos(kr, &sv, &cv);
        (sp ? m.A[1] : m.A[0])[k + j * ns] = make_double2(cv, sv);
        (sp ? m.W[1] : m.W[0])[k * ld + j] = make_double2(cv, sv);
      }
      for (int e = tid; e < 2 * n; e += kThreads) m.gsh[e] = __ldg(S.gvec + e);
      if (tid < 2) m.iscal[tid] = 0;  // singular flags
      __syncthreads();
      phase_mark(S, PH_ORBITALS, tph);
      // inversion: every warp in registers when each spin's matrix fits that
      // layout (then rho_k), else half the CTA per shared-memory inversion
      // with rho_k on the other warps
      // (determinants in HBM: every warp, coalesced rows, then rho_k)
      const int Gr = gj_reg_warps(nt);
      reg_path = !kGmat && S.tune_inv != 1;
      for (int sp = 0; sp < nt; sp++) reg_path = reg_path && gj_reg_lanes(S.np[sp], 32 * Gr) > 0;
      bool panel_path = reg_path && S.tune_inv == 2;
      for (int sp = 0; sp < nt; sp++) panel_path = panel_path && S.np[sp] <= 32;
      if (panel_path) {
        // blocks of eight pivot steps, one warp per panel, every warp of the
        // spin's group on the rest; then rho_k on every warp
        const int sp = nt > 1 ? (tid >> 5) / Gr : 0, gt = tid - sp * 32 * Gr;
        gj_invert_panel(sp ? m.W[1] : m.W[0], ws_ld(S.np[sp]), S.np[sp],
                        sp ? m.perm[1] : m.perm[0], sp ? m.dk[1] : m.dk[0], &m.iscal[sp], gt, Gr,
                        1 + sp, sp ? m.pscr[1] : m.pscr[0]);
        __syncthreads();
        phase_mark(S, PH_INVERT, tph);
        rhok(tid, kThreads);
        __syncthreads();
      } else if (!kGmat && S.tune_inv == 1) {
        // one warp per spin, warp-synchronous pivot steps; rho_k on the rest
        const int w = tid >> 5;
        if (w < nt) {
          const int ns = S.np[w];
          gj_invert(w ? m.W[1] : m.W[0], ws_ld(ns), ns, w ? m.perm[1] : m.perm[0],
                    w ? m.dk[1] : m.dk[0], w ? m.used[1] : m.used[0], &m.iscal[w], tid & 31, 1,
                    1 + w, m.gval + 8 * w, m.gidx + 8 * w);
        } else {
          rhok(tid - 32 * nt, kThreads - 32 * nt);
        }
        __syncthreads();
      } else if (reg_path) {
        const int sp = nt > 1 ? (tid >> 5) / Gr : 0, gt = tid - sp * 32 * Gr;
        gj_invert_reg(sp ? m.W[1] : m.W[0], ws_ld(S.np[sp]), S.np[sp], sp ? m.perm[1] : m.perm[0],
                      sp ? m.dk[1] : m.dk[0], &m.iscal[sp], gt, Gr, 1 + sp,
                      sp ? m.gslot[1] : m.gslot[0], sp ? m.gkey[1] : m.gkey[0]);
        __syncthreads();
        phase_mark(S, PH_INVERT, tph);
        rhok(tid, kThreads);
        __syncthreads();
      } else {
        // warps per spin: half the CTA for the inversions, the rest for rho_k
        const int G = kGmat ? (kThreads / 32) / nt
                            : ((kThreads / 32) / (2 * nt) > 0 ? (kThreads / 32) / (2 * nt) : 1);
        const int w = tid >> 5;
        if (w < G * nt) {
          const int sp = w / G, gt = tid - sp * 32 * G;
          const int ns = S.np[sp];
          if (kGmat)
            gj_invert_gmem(sp ? m.W[1] : m.W[0], ws_ld(ns), ns, sp ? m.perm[1] : m.perm[0],
                           sp ? m.dk[1] : m.dk[0], sp ? m.used[1] : m.used[0], &m.iscal[sp], gt,
                           G, 1 + sp, m.gval + 8 * sp, m.gidx + 8 * sp,
                           sp ? m.fcol[1] : m.fcol[0]);
          else
            gj_invert(sp ? m.W[1] : m.W[0], ws_ld(ns), ns, sp ? m.perm[1] : m.perm[0],
                      sp ? m.dk[1] : m.dk[0], sp ? m.used[1] : m.used[0], &m.iscal[sp], gt,
                      G, 1 + sp, m.gval + 8 * sp, m.gidx + 8 * sp);
        } else {
          rhok(tid - G * nt * 32, kThreads - G * nt * 32);
        }
        __syncthreads();
        if (G * nt == kThreads / 32) {
          rhok(tid, kThreads);
          __syncthreads();
        }
      }
    }
    {
      double acc[2] = {0.0, 0.0};  // log|det| and the Jastrow terms, one reduction
      for (int sp = 0; sp < nt; sp++)
        for (int k = tid; k < S.np[sp]; k += kThreads)
          acc[0] += 0.5 * log((sp ? m.dk[1] : m.dk[0])[k]);
      for (int i = tid; i < N; i += kThreads) acc[1] += m.ltf[i];
      block_sum_n<2>(acc, m.red);
      logdet_sum = acc[0];
      ltf_j = acc[1];
      if (m.iscal[0] || m.iscal[1]) status |= ST_SINGULAR;
    }
    phase_mark(S, reg_path ? PH_RHOK : PH_INVERT, tph);

    for (int sp = 0; sp < nt; sp++) {
      const int ns = S.np[sp], ld = ws_ld(ns), f0 = S.ipfrst[sp];
      const double2 *A = sp ? m.A[1] : m.A[0], *W = sp ? m.W[1] : m.W[0];
      const int *pm = sp ? m.perm[1] : m.perm[0];
      if (kSeq && sp > 0) {
        // this spin's orbitals and inverse into the buffer that the spin
        // before it has finished with (its last chunk ended on a barrier)
        const double2 *sA = reinterpret_cast<const double2 *>(inv_in);
        for (int t = 0; t < sp; t++) sA += inv_spin_doubles(S.np[t]) / 2;
        const double2 *sW = sA + (size_t)ns * ns;
        double2 *dA = m.A[sp], *dW = m.W[sp];
        for (int e = tid; e < ns * ns; e += kThreads) cp_async16(dA + e, sA + e);
        for (int e = tid; e < ns * ld; e += kThreads) cp_async16(dW + e, sW + e);
        cp_async_wait_all();
        __syncthreads();
      }
      // F_a(l,j) = sum_k Ainv(l,k) (i g_k[a]) A(k,j) (zv, reptation.f:10189-10200)
      // with Ainv(l, pi(c)) = W(pi(l), c).
      if (!kGmat) {
        // On the FP64 tensor cores (mma.m8n8k4, fragments as in the cross
        // term below): F_a = (W_pi diag(g_a)) (i A_pi), rows of W and of A
        // taken in pivot order. A warp takes a row tile of 8 l and two
        // column tiles of 8 j, k-steps of 4 c; its A fragment is
        // W(pi(l), c) g_a(pi(c)) (zero for c >= ns), its B fragment
        // i A(pi(c), j), and per column tile eight products form the real
        // and imaginary parts of F_x and F_y. Rows and columns beyond ns
        // repeat the last one and are not stored.
        const int RTf = (ns + 7) >> 3, KTf = (ns + 3) >> 2, CP = (RTf + 1) >> 1;
        const int warp = tid >> 5, lane = tid & 31, lg = lane >> 2, lt = lane & 3;
        for (int pt = warp; pt < RTf * CP; pt += kThreads / 32) {
          const int Lt = pt / CP, J0 = 2 * (pt - Lt * CP);
          const double2 *wrow = W + pm[min(8 * Lt + lg, ns - 1)] * ld;
          const double2 *acol0 = A + min(8 * J0 + lg, ns - 1) * ns;
          const double2 *acol1 = A + min(8 * J0 + 8 + lg, ns - 1) * ns;
          double acc[2][4][2];  // [column tile][F_x re, F_x im, F_y re, F_y im][column]
#pragma unroll
          for (int t = 0; t < 2; t++)
#pragma unroll
            for (int u = 0; u < 4; u++) acc[t][u][0] = acc[t][u][1] = 0.0;
#pragma unroll 2
          for (int kt = 0; kt < KTf; kt++) {
            const int c = 4 * kt + lt;
            const bool cok = c < ns;
            const int pc = pm[cok ? c : ns - 1];
            const double2 wv = cok ? wrow[c] : make_double2(0.0, 0.0);
            const double gx = m.gsh[2 * pc], gy = m.gsh[2 * pc + 1];
            const double wxr = wv.x * gx, wxi = wv.y * gx, wyr = wv.x * gy, wyi = wv.y * gy;
#pragma unroll
            for (int t = 0; t < 2; t++) {
              const double2 av = (t ? acol1 : acol0)[pc];
              const double nai = -av.y;  // i A = (-Im A, Re A)
              dmma_m8n8k4(acc[t][0], wxr, nai);
              dmma_m8n8k4(acc[t][0], -wxi, av.x);
              dmma_m8n8k4(acc[t][1], wxr, av.x);
              dmma_m8n8k4(acc[t][1], wxi, nai);
              dmma_m8n8k4(acc[t][2], wyr, nai);
              dmma_m8n8k4(acc[t][2], -wyi, av.x);
              dmma_m8n8k4(acc[t][3], wyr, av.x);
              dmma_m8n8k4(acc[t][3], wyi, nai);
            }
          }
          const int l = 8 * Lt + lg;
#pragma unroll
          for (int t = 0; t < 2; t++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
              const int j = 8 * (J0 + t) + 2 * lt + e;
              if (l < ns && j < ns && J0 + t < RTf) {
                m.F0[l + j * ns] = make_double2(acc[t][0][e], acc[t][1][e]);
                m.F1[l + j * ns] = make_double2(acc[t][2][e], acc[t][3][e]);
              }
            }
        }
      } else {
        // determinants in HBM: 2x2 (l,j) tiles per thread
        const int nh = (ns + 1) / 2;
        for (int tile = tid; tile < nh * nh; tile += kThreads) {
          const int l0 = 2 * (tile % nh), j0 = 2 * (tile / nh);
          const bool l1ok = l0 + 1 < ns, j1ok = j0 + 1 < ns;
          const double2 *w0 = W + pm[l0] * ld;
          const double2 *w1 = W + pm[l1ok ? l0 + 1 : l0] * ld;
          const double2 *a0c = A + j0 * ns;
          const double2 *a1c = A + (j1ok ? j0 + 1 : j0) * ns;
          double2 f0[2][2], f1[2][2];
#pragma unroll
          for (int u = 0; u < 2; u++)
#pragma unroll
            for (int v = 0; v < 2; v++) f0[u][v] = f1[u][v] = make_double2(0.0, 0.0);
          // unrolled so that the permuted loads of later columns are in
          // flight while earlier ones are used
#pragma unroll 4
          for (int c = 0; c < ns; c++) {
            const int pc = pm[c];
            const double gx = m.gsh[2 * pc], gy = m.gsh[2 * pc + 1];
            const double2 wv[2] = {w0[c], w1[c]};
            const double2 av[2] = {a0c[pc], a1c[pc]};
#pragma unroll
            for (int u = 0; u < 2; u++)
#pragma unroll
              for (int v = 0; v < 2; v++) {
                double2 pr = cmul(wv[u], av[v]);
                f0[u][v].x -= gx * pr.y;
                f0[u][v].y += gx * pr.x;
                f1[u][v].x -= gy * pr.y;
                f1[u][v].y += gy * pr.x;
              }
          }
#pragma unroll
          for (int u = 0; u < 2; u++)
#pragma unroll
            for (int v = 0; v < 2; v++) {
              int l = l0 + u, j = j0 + v;
              if (l < ns && j < ns) {
                m.F0[l + j * ns] = f0[u][v];
                m.F1[l + j * ns] = f1[u][v];
              }
            }
        }
      }
      // D2(j)[ab] = Re sum_k Ainv(j,k) (-g_ka g_kb) A(k,j)  (ddzorb term),
      // 8 lanes per electron, fixed shuffle order
      for (int base = 0; base < ns; base += kThreads / kGroup) {
        const int j = base + tid / kGroup;
        double dxx = 0, dxy = 0, dyy = 0;
        if (j < ns) {
          const double2 *wj = W + pm[j] * ld;
          for (int c = lane8; c < ns; c += kGroup) {
            const int pc = pm[c];
            double pr = wj[c].x * A[pc + j * ns].x - wj[c].y * A[pc + j * ns].y;
            double gx = m.gsh[2 * pc], gy = m.gsh[2 * pc + 1];
            dxx -= gx * gx * pr;
            dxy -= gx * gy * pr;
            dyy -= gy * gy * pr;
          }
        }
        dxx = group8_sum(dxx);
        dxy = group8_sum(dxy);
        dyy = group8_sum(dyy);
        if (j < ns && lane8 == 0) {
          m.D2[3 * j] = dxx;
          m.D2[3 * j + 1] = dxy;
          m.D2[3 * j + 2] = dyy;
        }
      }
      __syncthreads();
      phase_mark(S, PH_FMAT, tph);
      if (S.bf_zero) {
        // eta = 0: q = x and every Jacobian block is the identity, so only
        // this spin's electrons see this determinant, the drift and phase
        // gradient are the diagonals of F, and the Laplacian terms of the
        // Jacobian build and of the cross term reduce to -tr D2(i) and
        // sum_a Re F_a(i,i)^2 (no M, no GEMM)
        for (int jl = tid; jl < ns; jl += kThreads) {
          const int i = f0 + jl;
          const double2 fx = m.F0[jl + jl * ns], fy = m.F1[jl + jl * ns];
          m.gd[2 * i] -= fx.x;
          m.gd[2 * i + 1] -= fy.x;
          m.ph2d[i] += fx.y * fx.y + fy.y * fy.y;
          m.lapd[i] += -(m.D2[3 * jl] + m.D2[3 * jl + 2]) +
                       ((fx.x * fx.x - fx.y * fx.y) + (fy.x * fy.x - fy.y * fy.y));
        }
        __syncthreads();  // the next spin's F overwrites F0/F1
        phase_mark(S, PH_CROSS, tph);
        continue;
      }
      // cross term: M (2n x 2n, row stride ldM, over A[sp], W[sp]), then
      // per chunk of 16 electrons Y = M U on the FP64 tensor cores and the
      // quadratic forms sum_p U(p,c) Y(p,c). M is symmetric, so in 8 x 8
      // blocks u^T M u = 2 sum_P u_P^T (sum_{Q<P} M_PQ u_Q + M_PP u_P / 2):
      // only the blocks Q <= P are built, the diagonal ones halved, and the
      // padding columns of the last block (up to 4 KT) zero.
      const int n2 = 2 * ns, ldM = xt_ldm(2 * ns), ldU = xt_ldu(2 * ns);
      const int RT = xt_row_tiles(n2), KT = (n2 + 3) / 4;
      const int warp = tid >> 5, lane = tid & 31, lg = lane >> 2, lt = tid & 3;
      double *M = reinterpret_cast<double *>(sp ? m.A[1] : m.A[0]);
      for (int p = warp; p < n2; p += kThreads / 32) {
        const int a = p >= ns ? 1 : 0, j = p - a * ns;
        const double2 *Fa = a ? m.F1 : m.F0;
        const int pb = p >> 3, qend = min(8 * (pb + 1), 4 * KT);
        for (int qq = lane; qq < qend; qq += 32) {
          double v = 0.0;
          if (qq < n2) {
            const int c = qq >= ns ? 1 : 0, k = qq - c * ns;
            const double2 fa = Fa[k + j * ns];
            const double2 fc = (c ? m.F1 : m.F0)[j + k * ns];
            v = fa.x * fc.x - fa.y * fc.y;
            if ((qq >> 3) == pb) v *= 0.5;
          }
          M[p * ldM + qq] = v;
        }
      }
      for (int j = tid; j < ns; j += kThreads) {
        const double2 fx = m.F0[j + j * ns], fy = m.F1[j + j * ns];
        m.fdg[4 * j] = fx.x;
        m.fdg[4 * j + 1] = fx.y;
        m.fdg[4 * j + 2] = fy.x;
        m.fdg[4 * j + 3] = fy.y;
      }
      __syncthreads();
      // UT (over F0/F1, dead now): rows n2 .. ldU-1 of every column stay
      // zero, covering the k padding of the last k-step and the rows of the
      // last row tile beyond n2.
      double *UT = m.U;
      for (int col = warp; col < kChunk; col += kThreads / 32)
        for (int r = n2 + lane; r < ldU; r += 32) UT[col * ldU + r] = 0.0;
      phase_mark(S, PH_MBUILD, tph);
      static_assert(kThreads == 16 * (kChunk / 2), "16 lanes per electron of a chunk");
      for (int i0 = 0; i0 < N; i0 += kChunk / 2) {
        // UT[(i,b)][(a,j)] = J_{j,i}[a][b] for electrons i = i0 .. i0+15,
        // 16 lanes per electron; on the way, this determinant's drift,
        // phase gradient and first two Laplacian terms of electron i
        // (reptation.f:10201-10237), summed over the lanes in a fixed order.
        {
          const int il = tid >> 4, l16 = tid & 15, i = i0 + il;
          const bool valid = i < N;
          const int ti = valid ? type_of(S, i) : 0;
          double zxr = 0, zxi = 0, zyr = 0, zyi = 0, t12 = 0;
          // columns in blocks of 32 (two per lane): the stored pair values of
          // both are requested before either is used
          for (int jb = 0; jb < ns; jb += 32) {
            double pv[2][3];
#pragma unroll
            for (int u = 0; u < 2; u++) {
              const int jl = jb + l16 + 16 * u, j = f0 + jl;
              pv[u][0] = pv[u][1] = pv[u][2] = 0.0;
              if (pin && valid && jl < ns && j != i) {
                const size_t e = i < j ? pair_tri(N, i, j) : pair_tri(N, j, i);
                pv[u][0] = __ldg(pin + e);
                pv[u][1] = __ldg(pin + NP + e);
                pv[u][2] = __ldg(pin + 2 * NP + e);
              }
            }
#pragma unroll
            for (int u = 0; u < 2; u++) {
              const int jl = jb + l16 + 16 * u;
              if (jl >= ns) continue;
              const int j = f0 + jl;
              double jxx = 0, jxy = 0, jyy = 0;
              if (valid) {
                double qbx, qby;  // J[a][b] = dq_j[a]/dx_i[b]
                if (j == i) {
                  jxx = 1.0 + m.Sb[3 * i];
                  jxy = m.Sb[3 * i + 1];
                  jyy = 1.0 + m.Sb[3 * i + 2];
                  qbx = m.qbd[2 * i];
                  qby = m.qbd[2 * i + 1];
                } else if (pin) {
                  double rx = m.x[2 * i] - m.x[2 * j], ry = m.x[2 * i + 1] - m.x[2 * j + 1];
                  rx = rx - S.el[0] * round(S.eli[0] * rx);
                  ry = ry - S.el[1] * round(S.eli[1] * ry);
                  const double t = pv[u][0], c = pv[u][1], w2 = pv[u][2];
                  jxx = -(t + c * rx * rx);
                  jxy = -(c * rx * ry);
                  jyy = -(t + c * ry * ry);
                  qbx = -w2 * rx;
                  qby = -w2 * ry;
                } else {
                  bf_offdiag(S, m.x, i, j, ti, sp, jxx, jxy, jyy, qbx, qby);
                }
                const double fxr = m.fdg[4 * jl], fxi = m.fdg[4 * jl + 1];
                const double fyr = m.fdg[4 * jl + 2], fyi = m.fdg[4 * jl + 3];
                zxr += fxr * jxx + fyr * jxy;
                zxi += fxi * jxx + fyi * jxy;
                zyr += fxr * jxy + fyr * jyy;
                zyi += fxi * jxy + fyi * jyy;
                t12 -= fxr * qbx + fyr * qby;
                const double jtj_xx = jxx * jxx + jxy * jxy;
                const double jtj_xy = jxx * jxy + jxy * jyy;
                const double jtj_yy = jxy * jxy + jyy * jyy;
                t12 -= m.D2[3 * jl] * jtj_xx + 2.0 * m.D2[3 * jl + 1] * jtj_xy +
                       m.D2[3 * jl + 2] * jtj_yy;
              }
              UT[(2 * il + 0) * ldU + 0 * ns + jl] = jxx;  // a=x, b=x
              UT[(2 * il + 1) * ldU + 0 * ns + jl] = jxy;  // a=x, b=y
              UT[(2 * il + 0) * ldU + 1 * ns + jl] = jxy;  // a=y, b=x
              UT[(2 * il + 1) * ldU + 1 * ns + jl] = jyy;  // a=y, b=y
            }
          }
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            zxr += __shfl_xor_sync(0xffffffffu, zxr, o);
            zxi += __shfl_xor_sync(0xffffffffu, zxi, o);
            zyr += __shfl_xor_sync(0xffffffffu, zyr, o);
            zyi += __shfl_xor_sync(0xffffffffu, zyi, o);
            t12 += __shfl_xor_sync(0xffffffffu, t12, o);
          }
          if (valid && l16 == 0) {
            m.gd[2 * i] -= zxr;
            m.gd[2 * i + 1] -= zyr;
            m.ph2d[i] += zxi * zxi + zyi * zyi;
            m.lapd[i] += t12;
          }
        }
        __syncthreads();
        phase_mark(S, PH_DRIFT, tph);
        // Y = M U by warps, 8x8 output tiles (mma.m8n8k4 f64 fragments:
        // A(row lg, col lt), B(row lt, col lg), D(row lg, cols 2lt, 2lt+1)),
        // over the block lower triangle: row tile P takes the k-steps of
        // the column blocks Q <= P. Warp w takes row tiles P = w (mod 8)
        // with column tiles 0-1 and P = RT-1-w (mod 8) with column tiles
        // 2-3, so every warp has 2 (RT + 1) k-steps at RT = 8. Rows of the
        // last row tile beyond n2 reuse row n2-1 (their outputs meet zero
        // rows of UT). Each tile's rows dot their UT rows into
        // part[row tile][column].
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
#pragma unroll 1
          for (int w8 = warp; w8 < RT; w8 += kThreads / 32) {
            const int P = h == 0 ? w8 : RT - 1 - w8;
            const int kend = min(2 * P + 2, KT);
            const double *Ma = M + min(8 * P + lg, n2 - 1) * ldM + lt;
            const double *Ub = UT + (16 * h + lg) * ldU + lt;
            double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
            for (int kt = 0; kt < kend; kt++) {
              const double a = Ma[4 * kt];
              dmma_m8n8k4(acc[0], a, Ub[4 * kt]);
              dmma_m8n8k4(acc[1], a, Ub[8 * ldU + 4 * kt]);
            }
#pragma unroll
            for (int c = 0; c < 2; c++) {
              const int col = 16 * h + 8 * c + 2 * lt;
              double s0 = acc[c][0] * UT[col * ldU + 8 * P + lg];
              double s1 = acc[c][1] * UT[(col + 1) * ldU + 8 * P + lg];
#pragma unroll
              for (int o = 4; o < 32; o <<= 1) {
                s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
              }
              if (lg == 0) {
                m.part[P * kChunk + col] = s0;
                m.part[P * kChunk + col + 1] = s1;
              }
            }
          }
        }
        __syncthreads();
        if (tid < kChunk / 2) {
          int i = i0 + tid;
          if (i < N) {
            double t3 = 0.0;
            for (int rt = 0; rt < RT; rt++)
              t3 += m.part[rt * kChunk + 2 * tid] + m.part[rt * kChunk + 2 * tid + 1];
            m.lapd[i] += 2.0 * t3;
          }
        }
        // The next chunk's Jacobian build touches neither part nor these
        // electrons' sums, and its own barrier precedes the next GEMM; only
        // after the last chunk must everyone wait (the next spin's F
        // overwrites this region, the assembly reads lapd).
        if (i0 + kChunk / 2 >= N) __syncthreads();
        phase_mark(S, PH_CROSS, tph);
      }
    }
  } else {
    rhok(tid, kThreads);
    for (int i = tid; i < N; i += kThreads) ltf_j += m.ltf[i];
    ltf_j = block_sum(ltf_j, m.red);
    phase_mark(S, PH_RHOK, tph);
  }

  // ---- assemble: -ln psi, kinetic (reptation.f:2729), potential (:3986)
  double ltf = ltf_j - logdet_sum;
  bool underflow = false;
  if (S.has_bf && S.ref_underflow) underflow = exp(-ltf * 2.0) <= 0.0;
  if (underflow) status |= ST_UNDERFLOW;
  // determinant terms and the drift cutoff (kinetic, reptation.f:2748-2763),
  // and on the way the per-type sums: Laplacian, |g|^2, pair potential,
  // phase gradient^2 (register arrays with compile-time indices only:
  // nt <= 2), the drift cutoff factors, and the k-space sums of every type
  // pair (reptation.f:4034-4052), all in one block reduction
  double sums[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = tid; i < N; i += kThreads) {
    double gx = m.g[2 * i], gy = m.g[2 * i + 1], lp = m.lap[i], ph = 0.0;
    if (S.has_bf && !underflow) {
      gx += m.gd[2 * i];
      gy += m.gd[2 * i + 1];
      lp += m.lapd[i];
      ph = m.ph2d[i];
    }
    double x2 = gx * gx + gy * gy;
    const int ti = type_of(S, i);
    if (S.adrift != 0.0) {
      double vari = 1.0 / (2.0 * S.hbs2m[ti] * S.delta);
      double gg = x2 * S.adrift * S.delta * S.delta * vari;
      gg = (-1.0 + sqrt(1.0 + 2.0 * gg)) / gg;
      sums[8] += gg;
      gx *= gg;
      gy *= gg;
    }
    m.g[2 * i] = gx;
    m.g[2 * i + 1] = gy;
    m.lap[i] = lp;
    m.ph2[i] = ph;
    m.ph2d[i] = x2;  // |g|^2 before the cutoff, for the kinetic energy
    const bool t1 = ti == 1;
    const double v = m.vp[i];
    sums[0] += t1 ? 0.0 : lp;
    sums[1] += t1 ? 0.0 : x2;
    sums[2] += t1 ? 0.0 : v;
    sums[3] += t1 ? 0.0 : ph;
    sums[4] += t1 ? lp : 0.0;
    sums[5] += t1 ? x2 : 0.0;
    sums[6] += t1 ? v : 0.0;
    sums[7] += t1 ? ph : 0.0;
  }
  {
    // every type pair in one loop, so the four v_k loads of a k are in
    // flight together (the sums keep their order: k ascending per thread)
    int nkp[4], nkmax = 0;
    const double *vkp[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const int it = p >> 1, jt = p & 1;
      const int iv = (it < nt && jt < nt) ? S.iv2[it][jt] : -1;
      nkp[p] = iv >= 0 ? S.tab_nkew[iv] : 0;
      vkp[p] = S.coef + (iv >= 0 ? S.tab_vkoff[iv] : 0);
      nkmax = max(nkmax, nkp[p]);
    }
    for (int k = tid; k < nkmax; k += kThreads) {
      double vk[4];
#pragma unroll
      for (int p = 0; p < 4; p++) vk[p] = k < nkp[p] ? __ldg(vkp[p] + k) : 0.0;
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const int it = p >> 1, jt = p & 1;
        if (k < nkp[p])
          sums[9 + p] += vk[p] * (m.rhok[2 * (it * S.nk + k)] * m.rhok[2 * (jt * S.nk + k)] +
                                  m.rhok[2 * (it * S.nk + k) + 1] * m.rhok[2 * (jt * S.nk + k) + 1]);
      }
    }
  }
  block_sum_n<13>(sums, m.red);
  double kin0 = 0.0, pot0 = 0.0, efp = 0.0;
  double kin_t[2] = {0, 0}, un_t[2] = {0, 0}, pot_t[2] = {0, 0};
#pragma unroll
  for (int t = 0; t < 2; t++) {
    if (t < nt) {
    double hs = sums[4 * t], g2 = sums[4 * t + 1];
    if (tid == 0) hl[t] = hs;
    kin_t[t] = S.hbs2m[t] * (hs - g2);
    kin0 += kin_t[t];
    kin_t[t] /= S.np[t];
    un_t[t] = 1.0 / sqrt(g2);
    pot_t[t] = sums[4 * t + 2];
    efp += S.hbs2m[t] * sums[4 * t + 3];
    }
  }
  kin0 /= S.npnorm;
  // v2 tails (potential, reptation.f:4001-4022)
#pragma unroll
  for (int it = 0; it < 2; it++) {
    if (it >= nt) continue;
    int i = S.iv2[it][it];
    if (i >= 0) pot_t[it] += S.np[it] * (S.np[it] - 1) * 0.5 * S.tab_tail[i];
    if (it == 0 && nt > 1) {
      i = S.iv2[0][1];
      if (i >= 0) {
        double aux = S.np[0] * S.np[1] * S.tab_tail[i];
        pot_t[0] += 0.5 * aux;
        pot_t[1] += 0.5 * aux;
      }
    }
  }
  pot0 = pot_t[0] + pot_t[1];
  // k space (reptation.f:4034-4052): the type pairs' sums from above
#pragma unroll
  for (int it = 0; it < 2; it++)
#pragma unroll
    for (int jt = 0; jt < 2; jt++) {
      if (it >= nt || jt >= nt) continue;
      int iv = S.iv2[it][jt];
      if (iv < 0 || S.tab_nkew[iv] == 0) continue;
      double c = sums[9 + 2 * it + jt] + S.tab_kself[iv] * S.npnorm;
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
    props[QMC2D_JGG] = S.adrift != 0.0 ? sums[8] / N : 1.0;
#pragma unroll
    for (int t = 0; t < 2; t++) {
      if (t >= nt) continue;
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
  // every thread holds the same sums, so the same total energy
  if (!isfinite(pot0 + kin0 + efp) || !isfinite(ltf)) status |= ST_NONFINITE;
  __syncthreads();
  phase_mark(S, PH_ASSEMBLE, tph);
  return status;
}

// The whole evaluation of the configuration in m.x (compute_properties,
// reptation.f:2661), with the u2 and v2 pair terms in precision R.
template <class R = double, bool kGmat = false>
__device__ inline int eval_walker(const DevSys &S, const EvalSmem &m, double *hl, double *props,
                                  double *sign, long long &tph) {
  eval_pairs<kThreads, false>(S, m, tph, nullptr, pair_rows<R>(S));
  return eval_det<kGmat>(S, m, hl, props, sign, tph, nullptr);
}

}  // namespace q2d
