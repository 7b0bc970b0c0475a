// handle.h - the state behind a qmc2d_handle (shared by capi.cu and rmc.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/qmc2d.h"
#include "devsys.h"
#include "kernels.cuh"
#include "rmc.cuh"

struct qmc2d_handle {
  q2d::DevSys hs{};
  q2d::DevSys *ds = nullptr;
  double *d_coef = nullptr, *d_kvec = nullptr, *d_gvec = nullptr;
  int gvec_cap = 0;  // wave vectors d_gvec holds
  int cap = 0, nw = 0, cur = 0;
  int nt = 0, N = 0, nprops = 0;
  q2d::DevPop pop[2]{};
  double *d_blk = nullptr, *d_norm = nullptr, *d_cnt = nullptr, *d_wate = nullptr;
  int *d_status = nullptr;
  int *h_status = nullptr;  // cap status words in pinned host memory (sync_status)
  double *d_mscr = nullptr;  // move scratch: cap * move_scratch_doubles(hs)
  double *d_blksum = nullptr;  // n_props + 1: block sums over the population
  double *d_gmat = nullptr;    // cap * hs.gmat_stride: determinant matrices (hs.gmat)
  q2d::BranchScratch br{};
  // staging for the batched evaluation entry point
  double *d_x = nullptr, *d_g = nullptr, *d_h = nullptr, *d_p = nullptr, *d_s = nullptr;
  cudaStream_t stream = nullptr;
  // qmc2d_population_load_async: the records other than x and g go through
  // this stream, ordered after the stream's earlier work (ev_fork), and the
  // stream joins them (ev_side) before anything else reads the population
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_side = nullptr;
  bool side_pending = false;
  int device = 0;
  int nsm = 0;  // the device's SMs
  // qmc2d_set_move_inversion: 1 the batched orbital-and-inversion kernel
  // when the population gives it at least kOrbInvMinPerSM spin matrices per
  // SM, 2 always (where it fits), 0 never
  int move_inv_mode = 1;
  // qmc2d_set_autotune_scope: 1 the pair kernel's groups and staging, 2 its
  // lanes per particle, 4 the inversion layout
  int tune_scope = 7;
  uint64_t seed = 0;
  uint32_t move_counter = 0, gen_counter = 0;
  uint32_t sweep_counter = 0;  // Philox c2 of single-electron sweeps (qmc2d_vmc_single)
  int bf_zero = 0;             // every backflow table identically zero (a plain determinant)
  double *d_sdrift = nullptr;  // cap: inverse drift of the last qmc2d_vmc_single
  double dmc_ecut = 0.0;  // qmc2d_set_dmc_ecut (0: the reference's weights)
  q2d::RmcState rmc{};
  // per-kernel CUDA-event timing (qmc2d_profile)
  bool prof = false;
  std::vector<cudaEvent_t> ev[QMC2D_NKERNELS];  // event pairs, reused
  int ev_used[QMC2D_NKERNELS] = {0};
  double prof_ms[QMC2D_NKERNELS] = {0};
  long prof_n[QMC2D_NKERNELS] = {0};
};

// Spin matrices per SM below which a move inverts inside the move kernel
// instead of in orb_inv_kernel (qmc2d_set_move_inversion mode 1). With the
// batched form the move runs in the one-buffer move kernel (three CTAs per
// SM). Measured crossovers (DMC, 512 to 2048 walkers): two spins of 29
// orbitals lose 3% at 7 matrices per SM and gain 6% at 14, two of 13
// orbitals break even at 7 and gain 13% at 14; a single spin of 25
// orbitals, whose in-kernel inversion spreads one matrix over every warp
// of the CTA, gains 4% at 3.5 and 21% at 7.
constexpr int kOrbInvMinPerSM = 10, kOrbInvMinPerSMSmall = 10, kOrbInvMinPerSMOneSpin = 3;

// Whether this handle's next move batches its orbitals and inversion.
inline bool move_orb_inv(const qmc2d_handle *h) {
  if (h->move_inv_mode == 0) return false;
  const int need = h->move_inv_mode == 2 ? 0
                   : h->hs.nt == 1       ? kOrbInvMinPerSMOneSpin
                   : h->hs.nmax <= 16    ? kOrbInvMinPerSMSmall
                                         : kOrbInvMinPerSM;
  return q2d::orb_inv_pays(h->hs, h->nw, h->nsm, need);
}

// Orders the handle's stream after the side copies of the last
// qmc2d_population_load_async (nothing when none are pending). Every entry
// point that touches the population calls it first; a move calls it after
// its pair kernel, which reads only x and g.
inline cudaError_t join_side(qmc2d_handle *h) {
  if (!h->side_pending) return cudaSuccess;
  h->side_pending = false;
  return cudaStreamWaitEvent(h->stream, h->ev_side, 0);
}

// Bracket one launch of kernel k with an event pair when profiling is on.
struct ProfScope {
  qmc2d_handle *h;
  int k, idx = -1;
  cudaStream_t st;
  ProfScope(qmc2d_handle *h_, int k_, cudaStream_t s) : h(h_), k(k_), st(s) {
    if (!h->prof) return;
    idx = h->ev_used[k]++;
    while ((int)h->ev[k].size() < 2 * (idx + 1)) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      h->ev[k].push_back(e);
    }
    cudaEventRecord(h->ev[k][2 * idx], st);
  }
  ~ProfScope() {
    if (idx >= 0) cudaEventRecord(h->ev[k][2 * idx + 1], st);
  }
};

// Reads the per-walker status words of the first n slots; maps them to a
// qmc2d_status code (capi.cu).
int q2d_sync_status(qmc2d_handle *h, int n);
