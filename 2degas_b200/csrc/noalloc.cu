// noalloc.cu - compute_properties for callers that cannot allocate device
// memory.
//
// Some callers own every byte of device memory themselves: a host code that
// hands all its buffers out of one pool it manages, or a serving loop that
// must never trigger a cudaMalloc (which can synchronise the device) between
// requests. They cannot create a qmc2d_handle, because creating one
// allocates. For them, qmc2d_compute_properties_noalloc evaluates a batch of
// walkers with the same kernel as qmc2d_compute_properties_dev, but keeps
// what the handle would have allocated - the device copy of the system
// (tables, k vectors, orbital wave vectors) and the per-walker status words -
// in one fixed array of this file, sized at load time.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/qmc2d.h"
#include "common.h"
#include "devsys.h"
#include "kernels.cuh"

namespace {

// 2 MiB per GPU, held from library load until exit. Layout of one call:
// [DevSys][packed tables][k vectors][orbital wave vectors][status words].
constexpr size_t kScratchDoubles = size_t(1) << 18;
constexpr int kMaxWalkers = 65536;  // status words kept at the end of the array
constexpr size_t kStatusDoubles = kMaxWalkers / 2;

static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_dev_addr[kMaxDevices] = {nullptr};

// Device address of g_scratch on the current device; looked up once per
// device (the array's name is only a host-side stand-in for it).
int scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    q2d::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return QMC2D_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    q2d::set_error("qmc2d_compute_properties_noalloc: device ordinal out of range");
    return QMC2D_ERR_LIMIT;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_dev_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      q2d::set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return QMC2D_ERR_CUDA;
    }
    g_dev_addr[dev] = static_cast<double *>(p);
  }
  *out = g_dev_addr[dev];
  return QMC2D_OK;
}

}  // namespace

extern "C" int qmc2d_compute_properties_noalloc(const qmc2d_system *sys, int nw,
                                                const double *x_dev, double *g_dev,
                                                double *hl_dev, double *props_dev,
                                                double *s_dev, void *stream) {
  if (!sys || nw < 0 || (nw > 0 && (!x_dev || !g_dev || !hl_dev || !props_dev || !s_dev))) {
    q2d::set_error("qmc2d_compute_properties_noalloc: bad argument");
    return QMC2D_ERR_ARG;
  }
  if (nw > kMaxWalkers) {
    char buf[128];
    std::snprintf(buf, sizeof buf,
                  "qmc2d_compute_properties_noalloc: %d walkers, at most %d per call", nw,
                  kMaxWalkers);
    q2d::set_error(buf);
    return QMC2D_ERR_LIMIT;
  }
  if (sys->ndim != 2 || sys->ntypes < 1 || sys->ntypes > 2 || sys->nptot > QMC2D_MAX_NP) {
    q2d::set_error("qmc2d_compute_properties_noalloc: unsupported system size");
    return QMC2D_ERR_LIMIT;
  }
  // Every array the copies below read must be there: a missing one would
  // leave the previous call's contents of the shared array in its place.
  if ((sys->nk > 0 && !sys->kvec) || (sys->ngvec > 0 && !sys->gvec) || sys->ntables < 0 ||
      sys->ntables > QMC2D_MAX_TABLES) {
    q2d::set_error("qmc2d_compute_properties_noalloc: system without its k or wave vectors");
    return QMC2D_ERR_ARG;
  }
  for (int t = 0; t < sys->ntables; t++)
    if (!sys->tables[t].ut || (sys->tables[t].nk_ewald > 0 && !sys->tables[t].vk)) {
      q2d::set_error("qmc2d_compute_properties_noalloc: table without coefficients");
      return QMC2D_ERR_ARG;
    }
  // The copies below read pageable host memory that is gone when the call
  // returns; a captured graph would replay them from freed memory.
  {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cap);
    if (ce != cudaSuccess) {
      q2d::set_error(std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
      return QMC2D_ERR_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) {
      q2d::set_error("qmc2d_compute_properties_noalloc: not allowed while the stream is captured");
      return QMC2D_ERR_ARG;
    }
  }
  // The device view of the system, built on the stack; offsets count doubles
  // from the start of the scratch array.
  q2d::DevSys s;
  std::memset(&s, 0, sizeof s);
  s.N = sys->nptot;
  s.nt = sys->ntypes;
  s.npnorm = sys->npnorm;
  s.nprops = sys->n_props;
  s.nscalar = sys->n_scalar_props;
  s.jrhok = sys->jrhok;
  s.nk = sys->nk;
  s.ngvec = sys->ngvec;
  s.nrhok = sys->nrhok;
  for (int t = 0; t < 2; t++) {
    bool in = t < sys->ntypes;
    s.np[t] = in ? sys->np[t] : 0;
    s.ipfrst[t] = in ? sys->ipfrst[t] : sys->nptot;
    s.irhok[t] = in ? sys->irhok[t] : 0;
    s.hbs2m[t] = in ? sys->hbs2m[t] : 0.0;
    if (in && sys->np[t] > s.nmax) s.nmax = sys->np[t];
  }
  for (int d = 0; d < 2; d++) {
    s.el[d] = sys->el[d];
    s.eli[d] = sys->eli[d];
  }
  s.drt = sys->drt;
  s.drti = sys->drti;
  s.drti2 = sys->drti2;
  s.v0 = sys->v0;
  s.adrift = sys->adrift;
  s.delta = sys->delta;
  s.ntheta = sys->ntheta;
  s.ref_underflow = sys->ref_underflow_return;
  s.ecut = sys->ecut;
  s.value_ecut = sys->value_ecut;
  s.rejection = sys->rejection;
  s.wpiu = sys->wpiu;
  s.gstorto = sys->gstorto;
  s.nodalaction = sys->nodalaction;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      bool in = a < sys->ntypes && b < sys->ntypes;
      s.iu2[a][b] = in ? sys->iu2[a][b] : -1;
      s.iu3[a][b] = in ? sys->iu3[a][b] : -1;
      s.iub[a][b] = in ? sys->iub[a][b] : -1;
      s.iv2[a][b] = in ? sys->iv2[a][b] : -1;
    }
  s.has_u2 = s.iu2[0][0] >= 0;
  s.has_u3 = s.iu3[0][0] >= 0;
  s.has_bf = s.iub[0][0] >= 0;
  s.has_v2 = s.iv2[0][0] >= 0;
  s.phase = nullptr;
  size_t off = (sizeof(q2d::DevSys) + 15) / 16 * 2;  // doubles, 16-byte aligned
  const size_t limit = kScratchDoubles - kStatusDoubles;
  for (int t = 0; t < sys->ntables && t < QMC2D_MAX_TABLES; t++) {
    const qmc2d_table &tb = sys->tables[t];
    off = (off + 3) & ~size_t(3);  // 32-byte rows (one 256-bit load each)
    s.tab_off[t] = (int)off;
    s.tab_ngrid[t] = tb.ngrid;
    s.tab_iexp[t] = tb.iexp;
    s.tab_tail[t] = tb.tail;
    off += 4 * (size_t)(tb.ngrid + 1);
    s.tab_nkew[t] = tb.nk_ewald;
    s.tab_kself[t] = tb.nk_ewald > 0 ? tb.vk[tb.nk_ewald] : 0.0;
    s.tab_vkoff[t] = (int)off;
    if (tb.nk_ewald > 0) off += tb.nk_ewald + 1;
  }
  off = (off + 15) & ~size_t(15);  // 128-byte pair rows
  s.cmb_off = (int)off;
  std::vector<double> rows;
  q2d::pack_pair_rows(sys, &s, &rows);
  off += rows.size();
  const size_t kvec_off = off;
  off += 2 * (size_t)(sys->nk > 0 ? sys->nk : 0);
  const size_t gvec_off = off;
  off += 2 * (size_t)(sys->ngvec > 0 ? sys->ngvec : 0);
  if (off > limit) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "qmc2d_compute_properties_noalloc: system needs %zu doubles of tables, "
                  "at most %zu",
                  off, limit);
    q2d::set_error(buf);
    return QMC2D_ERR_LIMIT;
  }
  // One walker's evaluation must fit one CTA's shared memory: there is no
  // room here for the per-walker determinant blocks that a handle puts in
  // device memory for larger shells.
  {
    int dev = 0, optin = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce == cudaSuccess)
      ce = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (ce != cudaSuccess) {
      q2d::set_error(std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(ce));
      return QMC2D_ERR_CUDA;
    }
    const size_t need = q2d::eval_smem_bytes(s) + sizeof(q2d::DevSys);
    if (need > (size_t)optin) {
      char buf[200];
      std::snprintf(buf, sizeof buf,
                    "qmc2d_compute_properties_noalloc: one walker needs %zu bytes of shared "
                    "memory, the device gives %d (determinants this large need a handle)",
                    need, optin);
      q2d::set_error(buf);
      return QMC2D_ERR_LIMIT;
    }
  }
  double *base = nullptr;
  int st = scratch_address(&base);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  s.coef = base;
  s.kvec = base + kvec_off;
  s.gvec = base + gvec_off;
  int *status = reinterpret_cast<int *>(base + (kScratchDoubles - kStatusDoubles));
  auto fail = [](cudaError_t e, const char *what) {
    q2d::set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return QMC2D_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMemcpyAsync(base, &s, sizeof s, cudaMemcpyHostToDevice, cs)) != cudaSuccess)
    return fail(e, "cudaMemcpyAsync(system)");
  for (int t = 0; t < sys->ntables && t < QMC2D_MAX_TABLES; t++) {
    const qmc2d_table &tb = sys->tables[t];
    if ((e = cudaMemcpyAsync(base + s.tab_off[t], tb.ut, sizeof(double) * 4 * (tb.ngrid + 1),
                             cudaMemcpyHostToDevice, cs)) != cudaSuccess)
      return fail(e, "cudaMemcpyAsync(table)");
    if (tb.nk_ewald > 0 &&
        (e = cudaMemcpyAsync(base + s.tab_vkoff[t], tb.vk, sizeof(double) * (tb.nk_ewald + 1),
                             cudaMemcpyHostToDevice, cs)) != cudaSuccess)
      return fail(e, "cudaMemcpyAsync(v_k)");
  }
  // rows is pageable: the copy is staged before cudaMemcpyAsync returns
  if (!rows.empty() &&
      (e = cudaMemcpyAsync(base + s.cmb_off, rows.data(), sizeof(double) * rows.size(),
                           cudaMemcpyHostToDevice, cs)) != cudaSuccess)
    return fail(e, "cudaMemcpyAsync(pair rows)");
  if (sys->nk > 0 && (e = cudaMemcpyAsync(base + kvec_off, sys->kvec, sizeof(double) * 2 * sys->nk,
                                          cudaMemcpyHostToDevice, cs)) != cudaSuccess)
    return fail(e, "cudaMemcpyAsync(kvec)");
  if (sys->ngvec > 0 && sys->gvec &&
      (e = cudaMemcpyAsync(base + gvec_off, sys->gvec, sizeof(double) * 2 * sys->ngvec,
                           cudaMemcpyHostToDevice, cs)) != cudaSuccess)
    return fail(e, "cudaMemcpyAsync(gvec)");
  if (nw == 0) return QMC2D_OK;
  // status words must start at zero for this call
  if ((e = cudaMemsetAsync(status, 0, sizeof(int) * nw, cs)) != cudaSuccess)
    return fail(e, "cudaMemsetAsync(status)");
  if ((e = q2d::launch_eval(s, reinterpret_cast<const q2d::DevSys *>(base), nw, x_dev, g_dev,
                            hl_dev, props_dev, s_dev, status, cs)) != cudaSuccess)
    return fail(e, "eval kernel");
  return QMC2D_OK;
}

// Status of the last qmc2d_compute_properties_noalloc call: waits for
// `stream`, then ORs the first nw per-walker status words of the shared
// array, 1024 at a time through a buffer on the host stack.
extern "C" int qmc2d_compute_properties_noalloc_status(int nw, void *stream) {
  if (nw < 0 || nw > kMaxWalkers) {
    q2d::set_error("qmc2d_compute_properties_noalloc_status: bad walker count");
    return QMC2D_ERR_ARG;
  }
  double *base = nullptr;
  int st = scratch_address(&base);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const int *status = reinterpret_cast<const int *>(base + (kScratchDoubles - kStatusDoubles));
  int words[1024];
  int any = 0;
  cudaError_t e = cudaStreamSynchronize(cs);
  for (int i = 0; e == cudaSuccess && i < nw; i += 1024) {
    const int n = nw - i < 1024 ? nw - i : 1024;
    e = cudaMemcpyAsync(words, status + i, sizeof(int) * n, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    for (int k = 0; e == cudaSuccess && k < n; k++) any |= words[k];
  }
  if (e != cudaSuccess) {
    q2d::set_error(std::string("qmc2d_compute_properties_noalloc_status: ") +
                   cudaGetErrorString(e));
    return QMC2D_ERR_CUDA;
  }
  if (any & q2d::ST_SINGULAR) {
    q2d::set_error("zero pivot in a Slater matrix");
    return QMC2D_ERR_SINGULAR;
  }
  if (any & q2d::ST_NONFINITE) {
    q2d::set_error("non-finite local energy or -ln psi");
    return QMC2D_ERR_NONFINITE;
  }
  return QMC2D_OK;
}
