// handle.h - the state behind a qmc2d_handle (shared by capi.cu and rmc.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/qmc2d.h"
#include "devsys.h"
#include "kernels.cuh"
#include "rmc.cuh"

struct qmc2d_handle {
  q2d::DevSys hs{};
  q2d::DevSys *ds = nullptr;
  double *d_coef = nullptr, *d_kvec = nullptr, *d_gvec = nullptr;
  int cap = 0, nw = 0, cur = 0;
  int nt = 0, N = 0, nprops = 0;
  q2d::DevPop pop[2]{};
  double *d_blk = nullptr, *d_norm = nullptr, *d_cnt = nullptr, *d_wate = nullptr;
  int *d_status = nullptr;
  q2d::BranchScratch br{};
  // staging for the batched evaluation entry point
  double *d_x = nullptr, *d_g = nullptr, *d_h = nullptr, *d_p = nullptr, *d_s = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0;
  uint64_t seed = 0;
  uint32_t move_counter = 0, gen_counter = 0;
  q2d::RmcState rmc{};
};

// Reads the per-walker status words of the first n slots; maps them to a
// qmc2d_status code (capi.cu).
int q2d_sync_status(qmc2d_handle *h, int n);
