// rmc.cuh - reptile storage for reptation QMC (rmc.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "devsys.h"

namespace q2d {

// One reptile per CTA; its path is a ring of nbuf = ntau + mdelta beads in
// HBM (x_stack/g_stack/p_stack/s_stack/age_stack/w_stack of ewald.h:166-173),
// plus the path scalars of /c_path/ (jfirst, jlast, p_p_old, age).
struct RmcState {
  int nrep = 0, ntau = 0, ntauskip = 0, mdelta = 0, nbuf = 0;
  double delta = 0.0, etrial = 0.0;
  int mage = 0, mage_r = 0;
  double *x = nullptr, *g = nullptr, *p = nullptr, *h = nullptr, *s = nullptr;
  double *age_stack = nullptr, *w = nullptr;
  int *ends = nullptr;        // nrep * 2: jfirst, jlast
  double *pp_old = nullptr;   // nrep * nprops
  double *psum = nullptr;     // nrep * nprops: the accepted path's window sums (path_props)
  double *age = nullptr;      // nrep
  uint32_t step = 0;
  int split = 1;  // qmc2d_rmc_set_launch: pair kernel + determinant kernel per growth
  double *est = nullptr;  // path estimators: nrep rows and their mean (qmc2d_rmc_estimators)
  size_t est_cap = 0;
};

void rmc_free(RmcState *r);

}  // namespace q2d
