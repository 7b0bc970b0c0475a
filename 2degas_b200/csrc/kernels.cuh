// kernels.cuh - launchers of the walker kernels (kernels.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "devsys.h"

namespace q2d {

// One walker-move of a population: pairs kernel then move kernel.
struct MoveArgs {
  int nw;
  int first;          // first move of a DMC generation (weights restart at 1)
  int dmc;            // 0: VMC averages (weight 1), 1: DMC weights
  double delta;
  double mage;        // forced-move age (compared with ==, as the reference)
  double etrial, mmult;
  double ecut;        // > 0: clamp E_L in the DMC weight to etrial +- ecut
  uint64_t seed;
  uint32_t step0;     // Philox c2 of this move
  double *scr;        // nw * move_scratch(s).stride doubles (MoveScratch blocks)
  double *blk;        // nw * nprops block sums of p_old (* weight)
  double *blk_norm;   // nw
  double *cnt;        // nw * 4: accepted, proposed, forced, nonzero status
  double *wate;       // nw DMC weights (product over the generation's moves)
  int *status;        // nw status words (OR-ed)
  int orb_inv;        // 1: orb_inv_kernel ran before the move kernel (its output is in scr)
  // Device counters {move, generation} added to step0 (and to the comb's
  // generation) when non-null: a CUDA graph replays its launches with the
  // same arguments, so the Philox counters that must advance are read here.
  const uint32_t *ctr;
};

// Raise (never lower) kernel fn's dynamic shared-memory limit on the current
// device to bytes; safe to call from several host threads.
cudaError_t raise_smem_limit(const void *fn, size_t bytes);

// Evaluate nw configurations x (2N each) -> g, hl, props, s.
cudaError_t launch_eval(const DevSys &hs, const DevSys *ds, int nw, const double *x, double *g,
                        double *hl, double *props, double *s, int *status, cudaStream_t st);

// One move of a resident population: the proposal and pair passes into the
// move scratch (launch_pairs), the orbitals and their inversion into the
// move scratch when MoveArgs::orb_inv is set (launch_orb_inv, otherwise
// nothing), then the rest of the evaluation, the acceptance and the
// averages (launch_move).
cudaError_t launch_pairs(const DevSys &hs, const DevSys *ds, DevPop pop, const MoveArgs &a,
                         cudaStream_t st);
cudaError_t launch_orb_inv(const DevSys &hs, const DevSys *ds, const MoveArgs &a,
                           cudaStream_t st);
// launch_orb_inv can run (DevSys::split_inv and a scratch region for it),
// and whether it pays for a population of nw walkers on nsm SMs: the
// batched kernel wants at least min_per_sm spin matrices per SM.
bool orb_inv_applies(const DevSys &hs);
bool orb_inv_pays(const DevSys &hs, int nw, int nsm, int min_per_sm);
cudaError_t launch_move(const DevSys &hs, const DevSys *ds, DevPop pop, const MoveArgs &a,
                        cudaStream_t st);
// Doubles of move scratch per walker.
size_t move_scratch_doubles(const DevSys &hs);

// out[0..np) = per-property sums of blk (n walkers x np), out[np] = sum of
// norm: the block accumulators over the population, on the device.
cudaError_t launch_block_reduce(const double *blk, const double *norm, int n, int np,
                                double *out, cudaStream_t st);

// branch2's comb: wate -> src (new slot j copies old slot src[j]).
struct BranchScratch {
  double *delt, *csum;
  int *mult, *src, *ecum, *zrank;
  int *ncapped;
};
cudaError_t launch_branch(int nw, double *wate, uint64_t seed, uint32_t gen, BranchScratch b,
                          cudaStream_t st, const uint32_t *ctr = nullptr);
// ctr[0] += steps, ctr[1] += gens (one thread; ordered on st).
cudaError_t launch_counters_add(uint32_t *ctr, uint32_t steps, uint32_t gens, cudaStream_t st);
// new[j] = old[src[j]] for every walker field.
cudaError_t launch_gather(const DevSys &hs, DevPop from, DevPop to, const int *src, int nw,
                          cudaStream_t st);

// Walker records [x(2N), g(2N), h(nt), p(np), s, age] of slots[0..n) into
// rows of buf (unpack = 0) or from them (unpack = 1); slots in device memory.
cudaError_t launch_records(const DevSys &hs, DevPop pop, const int *slots, double *buf, int n,
                           int unpack, cudaStream_t st);

// Device Philox4x32-10 check: out[4*i..] = philox(ctr_i, key) for testing.
cudaError_t launch_philox_probe(uint64_t seed, const uint32_t *ctr, uint32_t *out, int n,
                                cudaStream_t st);

}  // namespace q2d
