// single.cuh - launcher of the single-electron VMC sweeps (single.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "devsys.h"

namespace q2d {

struct SingleArgs {
  int nw, nsweep;
  int refresh;       // single-electron moves between full inverse recomputes (0: only at start)
  double delta;
  uint64_t seed;
  uint32_t sweep0;   // Philox c2 of the first sweep
  DevPop pop;
  double *blk, *blk_norm, *cnt;
  double *drift;     // nw: largest |W D - I| seen before a recompute (max-ed in)
  int *status;
};

// Shared memory one walker's warp uses (bytes).
size_t single_smem_per_walker(const DevSys &s);
// nsweep sweeps of single-electron moves over every walker of pop.
cudaError_t launch_single(const DevSys &hs, const DevSys *ds, const SingleArgs &a,
                          cudaStream_t st);

}  // namespace q2d
