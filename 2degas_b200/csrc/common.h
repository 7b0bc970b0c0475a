// common.h - internal helpers shared by the host-side sources of libqmc2d.
#pragma once

#include <string>

namespace q2d {

// Thread-local last error message, returned by qmc2d_last_error().
void set_error(const std::string &msg);

// SORTTF (reptation.f:9514): heapsort of a 1-based index vector by a().
void sorttf(int n, const double *a, int *index);

}  // namespace q2d
