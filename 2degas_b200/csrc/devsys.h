// devsys.h - device-side view of a qmc2d_system and of a walker population.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/qmc2d.h"

namespace q2d {

constexpr int kThreads = 256;  // threads per walker CTA
constexpr int kGroup = 8;      // threads cooperating on one particle's pair sums
constexpr int kChunk = 32;     // (electron, direction) columns per backflow quadratic-form tile

// Per-walker status word bits written by the kernels.
enum : int { ST_OK = 0, ST_SINGULAR = 1, ST_NONFINITE = 2, ST_UNDERFLOW = 4 };

// Flattened system for kernels (passed by value as a kernel parameter).
struct DevSys {
  int N, nt, npnorm, nprops, nscalar, jrhok, nk, ngvec, nrhok;
  int np[2], ipfrst[2], irhok[2];
  int nmax;  // largest spin block
  double hbs2m[2], el[2], eli[2];
  double drt, drti, drti2, v0, adrift, delta;
  int ntheta, ref_underflow;
  int has_u2, has_u3, has_bf, has_v2;
  // reptation options (input keywords ecut, rejection, wpiu, gstorto, nodalaction)
  int ecut, rejection, wpiu, gstorto, nodalaction;
  double value_ecut;
  // table slots per type pair (into the packed coefficient buffer), -1 if none
  int iu2[2][2], iu3[2][2], iub[2][2], iv2[2][2];
  int tab_off[QMC2D_MAX_TABLES];   // offset (doubles) of ut(0,1) of table t
  int tab_ngrid[QMC2D_MAX_TABLES];
  int tab_iexp[QMC2D_MAX_TABLES];
  int tab_nkew[QMC2D_MAX_TABLES];
  int tab_vkoff[QMC2D_MAX_TABLES];  // offset of v_k in the packed buffer
  double tab_tail[QMC2D_MAX_TABLES];
  double tab_kself[QMC2D_MAX_TABLES];  // v_k list's closing (self-term) coefficient
  // Pair rows: for type pair (a, b) (block cmb_blk[a][b] of cmb_ng + 1 rows;
  // type pairs with the same four tables share a block) and knot k, 16
  // doubles = the four-coefficient rows of the u2, u3, backflow and v2
  // tables of that pair side by side (zeros for an absent kind), each
  // table's row min(k, its ngrid). One 128-byte line per pair lookup.
  int cmb_off, cmb_ng;  // offset (doubles, 128-byte aligned) in coef; last knot
  int cmb_blk[2][2], cmb_nblk;
  // Mixed rows at coef + cmbm_off (doubles, 128-byte aligned), read by the
  // pair passes when pair_f32: per knot the backflow and u3 rows in FP64,
  // then the u2 and v2 rows rounded to float, 128 bytes apart.
  int cmbm_off;
  // Precision of the pair passes (qmc2d_set_precision): 0 FP64; 1 the u2
  // and v2 pair terms in FP32 with compensated sums read out in FP64.
  int pair_f32;
  // Launch choices of the pair kernel (host side, qmc2d_autotune): walker
  // groups per CTA (0: the default, 2) and the staging of the pair rows in
  // shared memory (0: when they fit, 1: never).
  int tune_groups, tune_stage;
  // Lanes per particle in the pair kernel's two passes (qmc2d_set_pair_lanes,
  // also timed by qmc2d_autotune): 4, 8 or 16 (0: the default, 8).
  int tune_lanes;
  // Inversion layout of the determinant section (qmc2d_set_inversion):
  // 0 the register-resident Gauss-Jordan over every warp (4 warps per
  // spin, one CTA barrier per pivot step); 1 one warp per spin in shared
  // memory (warp-synchronous steps) with rho_k on the other warps; 2 the
  // panel-blocked form (one-warp panels of eight pivot steps).
  int tune_inv;
  // Moves of spins of at most 32 orbitals (no HBM determinants) may run the
  // orbitals and their inversion in orb_inv_kernel, one warp per spin
  // matrix, between the pair kernel and the move kernel, which then loads
  // A, the inverse, the pivots and |pivot|^2 from the move scratch (host
  // side: 1 once the handle exists; whether a move does so is
  // MoveArgs::orb_inv, qmc2d_set_move_inversion).
  int split_inv;
  // Every backflow table identically zero (set by the handle): q = x and the
  // backflow Jacobian is the identity, so the pair passes skip the backflow
  // terms and the determinant's drift and Laplacian come from the diagonals
  // of F and D2 without the cross-term GEMM.
  int bf_zero;
  // Every Ewald k vector on the reciprocal lattice, k = 2 pi (n1 / Lx,
  // n2 / Ly) to 1e-14 (set by the handle; |n1| <= rk_p1, |n2| <= rk_p2): the
  // pair kernels form rho_k from per-particle tables of exp(2 pi i p x / L)
  // instead of a sincos per (k, particle).
  int rk_lat, rk_p1, rk_p2;
  // Determinants too large for one CTA's shared memory (gmat = 1): the
  // orbital, inversion, F and cross-term matrices of walker (CTA) b live at
  // gmat_base + b * gmat_stride (doubles) in global memory; everything
  // else stays in shared memory.
  int gmat;
  long long gmat_stride;
  double *gmat_base;
  const double *coef;  // packed tables: ut rows (4 doubles each) and v_k lists
  const double *kvec;  // 2*nk
  const double *gvec;  // 2*ngvec
  unsigned long long *phase;  // per-phase SM cycles (qmc2d_phase_timers), null when off
};

// Phases of one walker move timed by qmc2d_phase_timers.
enum : int {
  PH_PROPOSE = 0, PH_PAIRS = 1, PH_RHOK = 2, PH_U3 = 3, PH_ORBITALS = 4, PH_INVERT = 5,
  PH_FMAT = 6, PH_DRIFT = 7, PH_MBUILD = 8, PH_CROSS = 9, PH_ASSEMBLE = 10, PH_ACCEPT = 11,
  PH_PATH = 12,  // reptation: path_props rescan, action deltas and the global accept
  PH_COUNT = 16
};

// Walker population in HBM: one block of each field per walker slot
// (walker-major; inside a walker the reference's x(2,N) order).
struct DevPop {
  double *x, *g, *h, *p, *s, *age;  // 2N, 2N, nt, nprops, 1, 1 per walker
};

// Pair rows of s appended to rows; sets s->cmb_ng and s->cmb_blk (host side).
void pack_pair_rows(const qmc2d_system *sys, DevSys *s, std::vector<double> *rows);

// Shared-memory footprint (bytes) of the walker evaluation for this system.
size_t eval_smem_bytes(const DevSys &s);
// Extra shared memory a move kernel adds for the walker's own state.
size_t move_smem_bytes(const DevSys &s);
// Doubles of global memory per walker for the determinant matrices when
// s.gmat is set (a multiple of 32, so that every block is 256-byte aligned);
// 0 otherwise.
size_t gmat_doubles(const DevSys &s);

}  // namespace q2d
