// capi.cu - the C-ABI of include/qmc2d.h: handle lifetime, device copies of
// the system, populations in HBM and the drivers that replace the
// reference's compute_properties / vmc / dmc loops.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"
#include "devsys.h"
#include "kernels.cuh"
#include "rmc.cuh"
#include "handle.h"

namespace q2d {

void pack_pair_rows(const qmc2d_system *sys, DevSys *s, std::vector<double> *rows) {
  int ng = 0;
  for (int a = 0; a < s->nt; a++)
    for (int b = 0; b < s->nt; b++)
      for (int t : {s->iu2[a][b], s->iu3[a][b], s->iub[a][b], s->iv2[a][b]})
        if (t >= 0 && sys->tables[t].ngrid > ng) ng = sys->tables[t].ngrid;
  s->cmb_ng = ng;
  std::vector<std::vector<int>> blocks;  // distinct (u2, u3, bf, v2) table tuples
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      s->cmb_blk[a][b] = 0;
      if (a >= s->nt || b >= s->nt) continue;
      std::vector<int> key = {s->iu2[a][b], s->iu3[a][b], s->iub[a][b], s->iv2[a][b]};
      size_t k = 0;
      while (k < blocks.size() && blocks[k] != key) k++;
      if (k == blocks.size()) blocks.push_back(key);
      s->cmb_blk[a][b] = (int)k;
    }
  s->cmb_nblk = (int)blocks.size();
  const size_t start = rows->size();
  for (const std::vector<int> &tab : blocks)
    for (int k = 0; k <= ng; k++)
      for (int q = 0; q < 4; q++) {
        if (tab[q] < 0) {
          rows->insert(rows->end(), 4, 0.0);
          continue;
        }
        const qmc2d_table &tb = sys->tables[tab[q]];
        const double *r = tb.ut + 4 * (size_t)std::min(k, tb.ngrid);
        rows->insert(rows->end(), r, r + 4);
      }
  // the mixed rows: per knot the backflow and u3 parts (doubles 8..11 and
  // 4..7 of the FP64 row), then the u2 and v2 parts rounded to float, then 32
  // bytes of padding (16 doubles)
  const size_t nrow = (rows->size() - start) / 16;
  s->cmbm_off = s->cmb_off + (int)(rows->size() - start);
  const size_t at = rows->size();
  rows->resize(at + 16 * nrow, 0.0);
  for (size_t k = 0; k < nrow; k++) {
    const double *src = rows->data() + start + 16 * k;
    double *dst = rows->data() + at + 16 * k;
    std::memcpy(dst, src + 8, sizeof(double) * 4);
    std::memcpy(dst + 4, src + 4, sizeof(double) * 4);
    float f[8];
    for (int q = 0; q < 4; q++) {
      f[q] = (float)src[q];           // u2
      f[4 + q] = (float)src[12 + q];  // v2
    }
    std::memcpy(dst + 8, f, sizeof f);
  }
}

}  // namespace q2d

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  q2d::set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return QMC2D_ERR_CUDA;
}

#define CK(call)                                      \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, sizeof(T) * (n > 0 ? n : 1));
}


int build_devsys(const qmc2d_system *sys, q2d::DevSys *hs, std::vector<double> *coef) {
  q2d::DevSys s{};
  s.N = sys->nptot;
  s.nt = sys->ntypes;
  s.npnorm = sys->npnorm;
  s.nprops = sys->n_props;
  s.nscalar = sys->n_scalar_props;
  s.jrhok = sys->jrhok;
  s.nk = sys->nk;
  s.ngvec = sys->ngvec;
  s.nrhok = sys->nrhok;
  s.nmax = 0;
  for (int t = 0; t < 2; t++) {
    s.np[t] = t < sys->ntypes ? sys->np[t] : 0;
    s.ipfrst[t] = t < sys->ntypes ? sys->ipfrst[t] : sys->nptot;
    s.irhok[t] = t < sys->ntypes ? sys->irhok[t] : 0;
    s.hbs2m[t] = t < sys->ntypes ? sys->hbs2m[t] : 0.0;
    if (t < sys->ntypes) s.nmax = std::max(s.nmax, sys->np[t]);
  }
  for (int d = 0; d < 2; d++) {
    s.el[d] = sys->el[d];
    s.eli[d] = sys->eli[d];
  }
  // rho_k from lattice power tables (DevSys::rk_lat) when every k vector is
  // 2 pi n / L per axis to 1e-14 and the tables stay small
  if (sys->nk > 0 && sys->kvec) {
    const double twopi = 6.283185307179586;
    bool lat = true;
    int pmax[2] = {0, 0};
    for (int k = 0; k < sys->nk && lat; k++)
      for (int d = 0; d < 2; d++) {
        const double kv = sys->kvec[2 * k + d], unit = twopi / sys->el[d];
        const double a = kv / unit;
        const long n = std::lround(a);
        if (!(std::fabs(a) < 64.0) || std::fabs(kv - n * unit) > 1e-14 * std::max(std::fabs(kv), unit)) {
          lat = false;
          break;
        }
        pmax[d] = std::max(pmax[d], (int)std::labs(n));
      }
    const size_t tbytes = sizeof(double) * 2 * (pmax[0] + pmax[1] + 2) * (size_t)sys->nptot;
    if (lat && tbytes <= 48 * 1024) {
      s.rk_lat = 1;
      s.rk_p1 = pmax[0];
      s.rk_p2 = pmax[1];
    }
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
  coef->clear();
  for (int t = 0; t < sys->ntables; t++) {
    const qmc2d_table &tb = sys->tables[t];
    while (coef->size() % 4) coef->push_back(0.0);  // 32-byte rows (one 256-bit load each)
    s.tab_off[t] = (int)coef->size();
    s.tab_ngrid[t] = tb.ngrid;
    s.tab_iexp[t] = tb.iexp;
    s.tab_tail[t] = tb.tail;
    coef->insert(coef->end(), tb.ut, tb.ut + 4 * (size_t)(tb.ngrid + 1));
    s.tab_nkew[t] = tb.nk_ewald;
    s.tab_kself[t] = tb.nk_ewald > 0 ? tb.vk[tb.nk_ewald] : 0.0;
    s.tab_vkoff[t] = (int)coef->size();
    if (tb.nk_ewald > 0) coef->insert(coef->end(), tb.vk, tb.vk + tb.nk_ewald + 1);
  }
  while (coef->size() % 16) coef->push_back(0.0);  // 128-byte pair rows
  s.cmb_off = (int)coef->size();
  q2d::pack_pair_rows(sys, &s, coef);
  *hs = s;
  return QMC2D_OK;
}

int alloc_pop(q2d::DevPop *p, int cap, int N, int nt, int np) {
  CK(dalloc(&p->x, (size_t)cap * 2 * N));
  CK(dalloc(&p->g, (size_t)cap * 2 * N));
  CK(dalloc(&p->h, (size_t)cap * nt));
  CK(dalloc(&p->p, (size_t)cap * np));
  CK(dalloc(&p->s, (size_t)cap));
  CK(dalloc(&p->age, (size_t)cap));
  return QMC2D_OK;
}

void free_pop(q2d::DevPop *p) {
  cudaFree(p->x);
  cudaFree(p->g);
  cudaFree(p->h);
  cudaFree(p->p);
  cudaFree(p->s);
  cudaFree(p->age);
  *p = q2d::DevPop{};
}

int sync_status(qmc2d_handle *h, int nw) {
  // the status words follow the kernels on the handle's stream into pinned
  // host memory: one synchronisation for both (and for pending side copies)
  CK(join_side(h));
  if (nw > 0)
    CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int) * nw, cudaMemcpyDeviceToHost,
                       h->stream));
  CK(cudaStreamSynchronize(h->stream));
  int any = 0;
  for (int i = 0; i < nw; i++) any |= h->h_status[i];
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

}  // namespace

int q2d_sync_status(qmc2d_handle *h, int n) { return sync_status(h, n); }

// Device bytes qmc2d_create allocates for sys at this capacity (each
// allocation rounded up to cudaMalloc's 512-byte granularity); the list is
// the one qmc2d_create allocates, in the same order.
size_t handle_bytes(const qmc2d_system *sys, const q2d::DevSys &hs, size_t ncoef, int cap) {
  auto al = [](size_t n, size_t elem) { return ((std::max<size_t>(n, 1) * elem) + 511) & ~size_t(511); };
  const size_t N = sys->nptot, nt = sys->ntypes, np = sys->n_props, c = cap;
  size_t b = al(ncoef, 8) + al(2 * (size_t)std::max(1, sys->nk), 8) +
             al(2 * (size_t)std::max(1, sys->ngvec), 8) + al(1, sizeof(q2d::DevSys));
  const size_t pop = al(c * 2 * N, 8) * 2 + al(c * nt, 8) + al(c * np, 8) + al(c, 8) * 2;
  b += 2 * pop;
  b += al(c * np, 8) + al(c, 8) + al(c * 4, 8) + al(c, 8) + al(c, 4);  // blk norm cnt wate status
  b += al(c, 8) * 2 + al(c, 4) * 4 + al(1, 4);                           // branch scratch
  b += al(c * 2 * N, 8) * 2 + al(c * nt, 8) + al(c * np, 8) + al(c, 8);  // staging
  b += al(c * q2d::move_scratch_doubles(hs), 8) + al(np + 1, 8);
  b += al(c, 8);  // inverse drift of the single-electron sweeps
  // determinants beyond shared memory: qmc2d_create moves them to HBM when
  // the walker exceeds the device's opt-in shared memory per block; this
  // count is made without a device, at the B200's 227 KB
  constexpr size_t kSmemOptinB200 = 232448;
  const size_t smem = std::max(q2d::move_smem_bytes(hs), q2d::eval_smem_bytes(hs));
  if (hs.gmat || (hs.has_bf && smem + sizeof(q2d::DevSys) > kSmemOptinB200)) {
    q2d::DevSys g = hs;
    g.gmat = 1;
    b += al(c * q2d::gmat_doubles(g), 8);
  }
  return b;
}

extern "C" int qmc2d_footprint(const qmc2d_system *sys, int capacity, uint64_t *bytes) {
  if (!sys || !bytes || capacity <= 0) {
    q2d::set_error("qmc2d_footprint: bad argument");
    return QMC2D_ERR_ARG;
  }
  if (sys->ndim != 2 || sys->ntypes < 1 || sys->ntypes > 2 || sys->nptot > QMC2D_MAX_NP) {
    q2d::set_error("qmc2d_footprint: unsupported system size");
    return QMC2D_ERR_LIMIT;
  }
  q2d::DevSys hs;
  std::vector<double> coef;
  build_devsys(sys, &hs, &coef);
  *bytes = handle_bytes(sys, hs, coef.size(), capacity);
  return QMC2D_OK;
}

extern "C" int qmc2d_create(const qmc2d_system *sys, const qmc2d_options *opt,
                            qmc2d_handle **out) {
  if (!sys || !opt || !out || opt->capacity <= 0) {
    q2d::set_error("qmc2d_create: bad argument");
    return QMC2D_ERR_ARG;
  }
  *out = nullptr;
  if (sys->ndim != 2 || sys->ntypes < 1 || sys->ntypes > 2 || sys->nptot > QMC2D_MAX_NP) {
    q2d::set_error("qmc2d_create: unsupported system size");
    return QMC2D_ERR_LIMIT;
  }
  qmc2d_handle *h = new qmc2d_handle();
  h->device = opt->device;
  h->seed = opt->seed;
  h->cap = opt->capacity;
  std::vector<double> coef;
  build_devsys(sys, &h->hs, &coef);
  h->nt = sys->ntypes;
  h->N = sys->nptot;
  h->nprops = sys->n_props;
  auto fail = [&](int code) {
    qmc2d_destroy(h);
    return code;
  };
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
  int smem_max = 0;
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  size_t need = std::max(q2d::move_smem_bytes(h->hs), q2d::eval_smem_bytes(h->hs));
  if (need + sizeof(q2d::DevSys) > (size_t)smem_max && h->hs.has_bf) {
    // the determinant matrices go to a per-walker block of global memory
    h->hs.gmat = 1;
    need = std::max(q2d::move_smem_bytes(h->hs), q2d::eval_smem_bytes(h->hs));
  }
  if (need + sizeof(q2d::DevSys) > (size_t)smem_max) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "walker needs %zu bytes of shared memory, device has %d",
                  need, smem_max);
    q2d::set_error(buf);
    return fail(QMC2D_ERR_LIMIT);
  }
  h->hs.split_inv = 1;  // moves may take orb_inv_kernel: the scratch has its region
  cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device);
  if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(cuda_fail(e, "cudaStreamCreate"));
  if ((e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&h->ev_side, cudaEventDisableTiming)) != cudaSuccess)
    return fail(cuda_fail(e, "cudaEventCreate"));
  int st;
  if ((e = dalloc(&h->d_coef, coef.size())) != cudaSuccess) return fail(cuda_fail(e, "alloc"));
  if ((e = dalloc(&h->d_kvec, 2 * (size_t)std::max(1, sys->nk))) != cudaSuccess)
    return fail(cuda_fail(e, "alloc"));
  if ((e = dalloc(&h->d_gvec, 2 * (size_t)std::max(1, sys->ngvec))) != cudaSuccess)
    return fail(cuda_fail(e, "alloc"));
  cudaMemcpy(h->d_coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice);
  if (sys->nk > 0)
    cudaMemcpy(h->d_kvec, sys->kvec, sizeof(double) * 2 * sys->nk, cudaMemcpyHostToDevice);
  if (sys->ngvec > 0 && sys->gvec)
    cudaMemcpy(h->d_gvec, sys->gvec, sizeof(double) * 2 * sys->ngvec, cudaMemcpyHostToDevice);
  h->hs.coef = h->d_coef;
  h->hs.kvec = h->d_kvec;
  h->hs.gvec = h->d_gvec;
  h->gvec_cap = std::max(1, sys->ngvec);
  if (h->hs.gmat) {
    h->hs.gmat_stride = (long long)q2d::gmat_doubles(h->hs);
    if ((e = dalloc(&h->d_gmat, (size_t)h->cap * h->hs.gmat_stride)) != cudaSuccess)
      return fail(cuda_fail(e, "cudaMalloc"));
    h->hs.gmat_base = h->d_gmat;
  }
  if ((e = dalloc(&h->ds, 1)) != cudaSuccess) return fail(cuda_fail(e, "alloc"));
  cudaMemcpy(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice);
  int cap = h->cap, N = h->N, nt = h->nt, np = h->nprops;
  for (int k = 0; k < 2; k++)
    if ((st = alloc_pop(&h->pop[k], cap, N, nt, np))) return fail(st);
  if ((e = dalloc(&h->d_blk, (size_t)cap * np)) != cudaSuccess ||
      (e = dalloc(&h->d_norm, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->d_cnt, (size_t)cap * 4)) != cudaSuccess ||
      (e = dalloc(&h->d_wate, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->d_status, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.delt, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.csum, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.mult, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.src, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.ecum, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.zrank, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->br.ncapped, 1)) != cudaSuccess ||
      (e = dalloc(&h->d_x, (size_t)cap * 2 * N)) != cudaSuccess ||
      (e = dalloc(&h->d_g, (size_t)cap * 2 * N)) != cudaSuccess ||
      (e = dalloc(&h->d_h, (size_t)cap * nt)) != cudaSuccess ||
      (e = dalloc(&h->d_p, (size_t)cap * np)) != cudaSuccess ||
      (e = dalloc(&h->d_s, (size_t)cap)) != cudaSuccess ||
      (e = dalloc(&h->d_mscr, (size_t)cap * q2d::move_scratch_doubles(h->hs))) != cudaSuccess ||
      (e = dalloc(&h->d_blksum, (size_t)np + 1)) != cudaSuccess ||
      (e = dalloc(&h->d_sdrift, (size_t)cap)) != cudaSuccess)
    return fail(cuda_fail(e, "cudaMalloc"));
  if ((e = cudaMallocHost((void **)&h->h_status, sizeof(int) * (size_t)cap)) != cudaSuccess)
    return fail(cuda_fail(e, "cudaMallocHost"));
  // a backflow table of zeros only: the determinant of plain plane waves
  h->bf_zero = 0;
  if (h->hs.has_bf) {
    bool zero = true;
    for (int a = 0; a < sys->ntypes; a++)
      for (int b = 0; b < sys->ntypes; b++) {
        const int t = sys->iub[a][b];
        if (t < 0) continue;
        const qmc2d_table &tb = sys->tables[t];
        for (size_t q = 0; q < 4 * (size_t)(tb.ngrid + 1) && zero; q++) zero = tb.ut[q] == 0.0;
      }
    h->bf_zero = zero ? 1 : 0;
  }
  h->hs.bf_zero = h->bf_zero;
  cudaMemcpy(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice);
  cudaMemset(h->d_blk, 0, sizeof(double) * cap * np);
  cudaMemset(h->d_norm, 0, sizeof(double) * cap);
  cudaMemset(h->d_cnt, 0, sizeof(double) * cap * 4);
  cudaMemset(h->d_status, 0, sizeof(int) * cap);
  cudaMemset(h->br.ncapped, 0, sizeof(int));
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(cuda_fail(e, "create"));
  *out = h;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_precision(qmc2d_handle *h, int precision) {
  if (!h || (precision != QMC2D_PRECISION_FP64 && precision != QMC2D_PRECISION_MIXED)) {
    q2d::set_error("qmc2d_set_precision: bad argument");
    return QMC2D_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  h->hs.pair_f32 = precision == QMC2D_PRECISION_MIXED ? 1 : 0;
  CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return QMC2D_OK;
}

extern "C" int qmc2d_set_dmc_ecut(qmc2d_handle *h, double ecut) {
  if (!h || !(ecut >= 0.0)) {
    q2d::set_error("qmc2d_set_dmc_ecut: bad argument");
    return QMC2D_ERR_ARG;
  }
  h->dmc_ecut = ecut;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_launch(qmc2d_handle *h, int groups, int stage) {
  if (!h || groups < 0 || groups > 2 || stage < 0 || stage > 1) {
    q2d::set_error("qmc2d_set_launch: bad argument");
    return QMC2D_ERR_ARG;
  }
  h->hs.tune_groups = groups;
  h->hs.tune_stage = stage;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_pair_lanes(qmc2d_handle *h, int lanes) {
  if (!h || (lanes != 0 && lanes != 4 && lanes != 8 && lanes != 16)) {
    q2d::set_error("qmc2d_set_pair_lanes: lanes must be 0 (the default), 4, 8 or 16");
    return QMC2D_ERR_ARG;
  }
  h->hs.tune_lanes = lanes;  // host-side launch choice (the kernel is templated on it)
  return QMC2D_OK;
}

extern "C" int qmc2d_get_pair_lanes(qmc2d_handle *h, int *lanes) {
  if (!h || !lanes) return QMC2D_ERR_ARG;
  *lanes = h->hs.tune_lanes == 4 || h->hs.tune_lanes == 16 ? h->hs.tune_lanes : 8;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_move_inversion(qmc2d_handle *h, int mode) {
  if (!h || mode < 0 || mode > 2) {
    q2d::set_error("qmc2d_set_move_inversion: mode must be 0, 1 or 2");
    return QMC2D_ERR_ARG;
  }
  h->move_inv_mode = mode;  // host-side launch choice (MoveArgs::orb_inv)
  return QMC2D_OK;
}

extern "C" int qmc2d_get_move_inversion(qmc2d_handle *h, int *batched) {
  if (!h || !batched) return QMC2D_ERR_ARG;
  *batched = move_orb_inv(h) ? 1 : 0;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_inversion(qmc2d_handle *h, int layout) {
  if (!h || layout < 0 || layout > 2) {
    q2d::set_error("qmc2d_set_inversion: bad argument");
    return QMC2D_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  h->hs.tune_inv = layout;
  CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return QMC2D_OK;
}

extern "C" int qmc2d_autotune(qmc2d_handle *h, int *groups, int *stage, double *ms) {
  if (!h) return QMC2D_ERR_ARG;
  if (h->nw <= 0) {
    q2d::set_error("qmc2d_autotune: empty population");
    return QMC2D_ERR_STACK;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  q2d::MoveArgs a{};
  a.nw = h->nw;
  a.scr = h->d_mscr;
  a.delta = h->hs.delta > 0.0 ? h->hs.delta : 0.01;
  a.seed = h->seed;
  a.step0 = h->move_counter;  // the next move's proposal; the scratch is rewritten by that move
  a.blk = h->d_blk;
  a.blk_norm = h->d_norm;
  a.cnt = h->d_cnt;
  a.status = h->d_status;
  const int var[4][2] = {{2, 0}, {2, 1}, {1, 0}, {1, 1}};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  int bg = h->hs.tune_groups ? h->hs.tune_groups : 2, bs = h->hs.tune_stage;
  const int lanes_in = h->hs.tune_lanes;
  h->hs.tune_lanes = 8;  // the groups and staging are compared at the default lanes
  for (const auto &v : var) {
    if (!(h->tune_scope & 1)) break;
    h->hs.tune_groups = v[0];
    h->hs.tune_stage = v[1];
    CK(q2d::launch_pairs(h->hs, h->ds, h->pop[h->cur], a, h->stream));  // warm-up
    CK(cudaEventRecord(e0, h->stream));
    for (int r = 0; r < 3; r++) CK(q2d::launch_pairs(h->hs, h->ds, h->pop[h->cur], a, h->stream));
    CK(cudaEventRecord(e1, h->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    if (t / 3.0 < best) {
      best = t / 3.0;
      bg = v[0];
      bs = v[1];
    }
  }
  h->hs.tune_groups = bg;
  h->hs.tune_stage = bs;
  h->hs.tune_lanes = lanes_in;
  // lanes per particle of the pair passes, with the chosen groups and staging
  // (8 first: the other two must beat it)
  if (h->tune_scope & 2) {
    const int lanes[3] = {8, 4, 16};
    int bl = 8;
    for (int l : lanes) {
      h->hs.tune_lanes = l;
      CK(q2d::launch_pairs(h->hs, h->ds, h->pop[h->cur], a, h->stream));  // warm-up
      CK(cudaEventRecord(e0, h->stream));
      for (int r = 0; r < 3; r++)
        CK(q2d::launch_pairs(h->hs, h->ds, h->pop[h->cur], a, h->stream));
      CK(cudaEventRecord(e1, h->stream));
      CK(cudaEventSynchronize(e1));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      if (l == 8 || t / 3.0 < best) {
        best = t / 3.0;
        bl = l;
      }
    }
    h->hs.tune_lanes = bl;
  }
  // inversion layout of the determinant section, timed on the evaluation
  // kernel over the population's configurations (into the staging buffers;
  // the population is not changed)
  if ((h->tune_scope & 4) && h->hs.has_bf && !h->hs.gmat) {
    double best_inv = 1e300;
    int bi = 0;
    for (int layout = 0; layout < 3; layout++) {
      h->hs.tune_inv = layout;
      CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
      const q2d::DevPop &p = h->pop[h->cur];
      CK(q2d::launch_eval(h->hs, h->ds, h->nw, p.x, h->d_g, h->d_h, h->d_p, h->d_s, h->d_status,
                          h->stream));  // warm-up
      CK(cudaEventRecord(e0, h->stream));
      for (int r = 0; r < 3; r++)
        CK(q2d::launch_eval(h->hs, h->ds, h->nw, p.x, h->d_g, h->d_h, h->d_p, h->d_s,
                            h->d_status, h->stream));
      CK(cudaEventRecord(e1, h->stream));
      CK(cudaEventSynchronize(e1));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      if (t / 3.0 < best_inv) {
        best_inv = t / 3.0;
        bi = layout;
      }
    }
    h->hs.tune_inv = bi;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream));
  }
  CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (groups) *groups = bg;
  if (stage) *stage = bs;
  if (ms) *ms = best;
  return QMC2D_OK;
}

extern "C" int qmc2d_set_autotune_scope(qmc2d_handle *h, int mask) {
  if (!h || mask < 0 || mask > 7) {
    q2d::set_error("qmc2d_set_autotune_scope: mask must be in 0..7");
    return QMC2D_ERR_ARG;
  }
  h->tune_scope = mask;
  return QMC2D_OK;
}

extern "C" int qmc2d_get_launch(qmc2d_handle *h, int *groups, int *stage, int *inversion) {
  if (!h) return QMC2D_ERR_ARG;
  if (groups) *groups = h->hs.tune_groups;
  if (stage) *stage = h->hs.tune_stage;
  if (inversion) *inversion = h->hs.tune_inv;
  return QMC2D_OK;
}

extern "C" int qmc2d_update_twist(qmc2d_handle *h, const qmc2d_system *sys) {
  if (!h || !sys || !sys->gvec || sys->ngvec <= 0 || sys->nptot != h->N) {
    q2d::set_error("qmc2d_update_twist: bad argument");
    return QMC2D_ERR_ARG;
  }
  if (sys->ngvec > h->gvec_cap) {
    q2d::set_error("qmc2d_update_twist: more wave vectors than the handle was created with");
    return QMC2D_ERR_LIMIT;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaMemcpyAsync(h->d_gvec, sys->gvec, sizeof(double) * 2 * sys->ngvec,
                     cudaMemcpyHostToDevice, h->stream));
  h->hs.ngvec = sys->ngvec;
  CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
  // sys->gvec is replaced by the next qmc2d_system_set_twist: finish reading it
  CK(cudaStreamSynchronize(h->stream));
  return QMC2D_OK;
}

extern "C" int qmc2d_destroy(qmc2d_handle *h) {
  if (!h) return QMC2D_OK;
  if (h->side) cudaStreamSynchronize(h->side);
  if (h->stream) cudaStreamSynchronize(h->stream);
  q2d::rmc_free(&h->rmc);
  for (int k = 0; k < 2; k++) free_pop(&h->pop[k]);
  void *bufs[] = {h->ds, h->d_coef, h->d_kvec, h->d_gvec, h->d_blk, h->d_norm, h->d_cnt,
                  h->d_wate, h->d_status, h->br.delt, h->br.csum, h->br.mult, h->br.src,
                  h->br.ecum, h->br.zrank, h->br.ncapped, h->d_x, h->d_g, h->d_h, h->d_p,
                  h->d_s, h->d_mscr, h->d_blksum, h->hs.phase, h->d_gmat, h->d_sdrift};
  for (void *b : bufs) cudaFree(b);
  if (h->h_status) cudaFreeHost(h->h_status);
  for (int k = 0; k < QMC2D_NKERNELS; k++)
    for (cudaEvent_t e : h->ev[k]) cudaEventDestroy(e);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_side) cudaEventDestroy(h->ev_side);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return QMC2D_OK;
}

extern "C" int qmc2d_stream(qmc2d_handle *h, void **stream) {
  if (!h || !stream) return QMC2D_ERR_ARG;
  *stream = (void *)h->stream;
  return QMC2D_OK;
}

extern "C" int qmc2d_profile(qmc2d_handle *h, int enable) {
  if (!h) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaStreamSynchronize(h->stream));
  h->prof = enable != 0;
  for (int k = 0; k < QMC2D_NKERNELS; k++) {
    h->ev_used[k] = 0;
    h->prof_ms[k] = 0.0;
    h->prof_n[k] = 0;
  }
  return QMC2D_OK;
}

extern "C" int qmc2d_phase_timers(qmc2d_handle *h, int enable, unsigned long long *cycles) {
  if (!h) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaStreamSynchronize(h->stream));
  if (enable) {
    if (!h->hs.phase) CK(dalloc(&h->hs.phase, q2d::PH_COUNT));
    CK(cudaMemset(h->hs.phase, 0, sizeof(unsigned long long) * q2d::PH_COUNT));
  } else if (h->hs.phase) {
    if (cycles)
      CK(cudaMemcpy(cycles, h->hs.phase, sizeof(unsigned long long) * q2d::PH_COUNT,
                    cudaMemcpyDeviceToHost));
    cudaFree(h->hs.phase);
    h->hs.phase = nullptr;
  }
  CK(cudaMemcpy(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice));
  return QMC2D_OK;
}

extern "C" int qmc2d_profile_get(qmc2d_handle *h, int kernel, double *ms, long *launches) {
  if (!h || kernel < 0 || kernel >= QMC2D_NKERNELS) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaStreamSynchronize(h->stream));
  for (int i = 0; i < h->ev_used[kernel]; i++) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->ev[kernel][2 * i], h->ev[kernel][2 * i + 1]));
    h->prof_ms[kernel] += t;
    h->prof_n[kernel]++;
  }
  h->ev_used[kernel] = 0;
  if (ms) *ms = h->prof_ms[kernel];
  if (launches) *launches = h->prof_n[kernel];
  return QMC2D_OK;
}

extern "C" int qmc2d_compute_properties_dev(qmc2d_handle *h, int nw, const double *x_dev,
                                            double *g_dev, double *hl_dev, double *props_dev,
                                            double *s_dev, void *stream) {
  if (!h || nw < 0 || nw > h->cap) {
    q2d::set_error("qmc2d_compute_properties_dev: bad argument");
    return QMC2D_ERR_ARG;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  if (nw > 0) CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * nw, st));
  ProfScope ps(h, QMC2D_KERNEL_EVAL, st);
  CK(q2d::launch_eval(h->hs, h->ds, nw, x_dev, g_dev, hl_dev, props_dev, s_dev, h->d_status,
                      st));
  return QMC2D_OK;
}

extern "C" int qmc2d_compute_properties_dev_status(qmc2d_handle *h, int nw, void *stream) {
  if (!h || nw < 0 || nw > h->cap) {
    q2d::set_error("qmc2d_compute_properties_dev_status: bad argument");
    return QMC2D_ERR_ARG;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  if (stream) CK(cudaStreamSynchronize((cudaStream_t)stream));
  return sync_status(h, nw);
}

extern "C" int qmc2d_compute_properties(qmc2d_handle *h, int nw, const double *x, double *g,
                                        double *hl, double *props, double *s) {
  if (!h || !x || nw < 0 || nw > h->cap) {
    q2d::set_error("qmc2d_compute_properties: bad argument");
    return QMC2D_ERR_ARG;
  }
  if (nw == 0) return QMC2D_OK;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  size_t N2 = 2 * (size_t)h->N;
  CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * nw, h->stream));
  CK(cudaMemcpyAsync(h->d_x, x, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, h->stream));
  {
    ProfScope ps(h, QMC2D_KERNEL_EVAL, h->stream);
    CK(q2d::launch_eval(h->hs, h->ds, nw, h->d_x, h->d_g, h->d_h, h->d_p, h->d_s, h->d_status,
                        h->stream));
  }
  if (g) CK(cudaMemcpyAsync(g, h->d_g, sizeof(double) * N2 * nw, cudaMemcpyDeviceToHost, h->stream));
  if (hl)
    CK(cudaMemcpyAsync(hl, h->d_h, sizeof(double) * h->nt * nw, cudaMemcpyDeviceToHost,
                       h->stream));
  if (props)
    CK(cudaMemcpyAsync(props, h->d_p, sizeof(double) * h->nprops * nw, cudaMemcpyDeviceToHost,
                       h->stream));
  if (s) CK(cudaMemcpyAsync(s, h->d_s, sizeof(double) * nw, cudaMemcpyDeviceToHost, h->stream));
  return sync_status(h, nw);
}

extern "C" int qmc2d_population_set(qmc2d_handle *h, int nw, const double *x) {
  if (!h || !x || nw <= 0 || nw > h->cap) {
    q2d::set_error("qmc2d_population_set: population outside capacity");
    return QMC2D_ERR_POPULATION;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  q2d::DevPop &p = h->pop[h->cur];
  size_t N2 = 2 * (size_t)h->N;
  CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * nw, h->stream));
  CK(cudaMemcpyAsync(p.x, x, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, h->stream));
  CK(q2d::launch_eval(h->hs, h->ds, nw, p.x, p.g, p.h, p.p, p.s, h->d_status, h->stream));
  // read_conf's metropolis_test(1): accepted, p_old(jacc) = 1, age = 0
  std::vector<double> one(nw, 1.0), zero(nw, 0.0);
  CK(cudaMemcpy2DAsync(p.p + QMC2D_JACC, sizeof(double) * h->nprops, one.data(), sizeof(double),
                       sizeof(double), nw, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(p.age, zero.data(), sizeof(double) * nw, cudaMemcpyHostToDevice,
                     h->stream));
  h->nw = nw;
  return sync_status(h, nw);
}

extern "C" int qmc2d_population_size(qmc2d_handle *h, int *nw) {
  if (!h || !nw) return QMC2D_ERR_ARG;
  *nw = h->nw;
  return QMC2D_OK;
}

extern "C" int qmc2d_population_get(qmc2d_handle *h, double *x, double *g, double *hl,
                                    double *props, double *s, double *age) {
  if (!h) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  q2d::DevPop &p = h->pop[h->cur];
  size_t N2 = 2 * (size_t)h->N, nw = h->nw;
  cudaStream_t st = h->stream;
  if (x) CK(cudaMemcpyAsync(x, p.x, sizeof(double) * N2 * nw, cudaMemcpyDeviceToHost, st));
  if (g) CK(cudaMemcpyAsync(g, p.g, sizeof(double) * N2 * nw, cudaMemcpyDeviceToHost, st));
  if (hl) CK(cudaMemcpyAsync(hl, p.h, sizeof(double) * h->nt * nw, cudaMemcpyDeviceToHost, st));
  if (props)
    CK(cudaMemcpyAsync(props, p.p, sizeof(double) * h->nprops * nw, cudaMemcpyDeviceToHost, st));
  if (s) CK(cudaMemcpyAsync(s, p.s, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
  if (age) CK(cudaMemcpyAsync(age, p.age, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return QMC2D_OK;
}

extern "C" int qmc2d_population_load(qmc2d_handle *h, int nw, const double *x, const double *g,
                                     const double *hl, const double *props, const double *s,
                                     const double *age) {
  if (!h || !x || !g || !hl || !props || !s || !age || nw <= 0 || nw > h->cap) {
    q2d::set_error("qmc2d_population_load: bad argument or population outside capacity");
    return QMC2D_ERR_POPULATION;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  q2d::DevPop &p = h->pop[h->cur];
  size_t N2 = 2 * (size_t)h->N;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(p.x, x, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p.g, g, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p.h, hl, sizeof(double) * h->nt * nw, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p.p, props, sizeof(double) * h->nprops * nw, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p.s, s, sizeof(double) * nw, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p.age, age, sizeof(double) * nw, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));  // the caller may reuse its buffers on return
  h->nw = nw;
  return QMC2D_OK;
}

extern "C" int qmc2d_population_load_async(qmc2d_handle *h, int nw, const double *x,
                                           const double *g, const double *hl,
                                           const double *props, const double *s,
                                           const double *age) {
  if (!h || !x || !g || !hl || !props || !s || !age || nw <= 0 || nw > h->cap) {
    q2d::set_error("qmc2d_population_load_async: bad argument or population outside capacity");
    return QMC2D_ERR_POPULATION;
  }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  q2d::DevPop &p = h->pop[h->cur];
  const size_t N2 = 2 * (size_t)h->N;
  // the side copies overwrite buffers that earlier work on the stream uses
  CK(cudaEventRecord(h->ev_fork, h->stream));
  CK(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
  CK(cudaMemcpyAsync(p.x, x, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(p.g, g, sizeof(double) * N2 * nw, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(p.h, hl, sizeof(double) * h->nt * nw, cudaMemcpyHostToDevice, h->side));
  CK(cudaMemcpyAsync(p.p, props, sizeof(double) * h->nprops * nw, cudaMemcpyHostToDevice,
                     h->side));
  CK(cudaMemcpyAsync(p.s, s, sizeof(double) * nw, cudaMemcpyHostToDevice, h->side));
  CK(cudaMemcpyAsync(p.age, age, sizeof(double) * nw, cudaMemcpyHostToDevice, h->side));
  CK(cudaEventRecord(h->ev_side, h->side));
  h->side_pending = true;
  h->nw = nw;
  return QMC2D_OK;
}

extern "C" int qmc2d_block_reset(qmc2d_handle *h) {
  if (!h) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaMemsetAsync(h->d_blk, 0, sizeof(double) * h->cap * h->nprops, h->stream));
  CK(cudaMemsetAsync(h->d_norm, 0, sizeof(double) * h->cap, h->stream));
  CK(cudaMemsetAsync(h->d_cnt, 0, sizeof(double) * h->cap * 4, h->stream));
  CK(cudaMemsetAsync(h->br.ncapped, 0, sizeof(int), h->stream));
  return QMC2D_OK;
}

extern "C" int qmc2d_block_get(qmc2d_handle *h, double *blk_av, double *blk_norm) {
  if (!h) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  const int np = h->nprops, n = std::max(h->nw, h->rmc.nrep);
  std::vector<double> sums((size_t)np + 1, 0.0);
  if (n > 0) {
    CK(q2d::launch_block_reduce(h->d_blk, h->d_norm, n, np, h->d_blksum, h->stream));
    CK(cudaMemcpyAsync(sums.data(), h->d_blksum, sizeof(double) * (np + 1),
                       cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  if (blk_av)
    for (int j = 0; j < np; j++) blk_av[j] = sums[j];
  if (blk_norm) *blk_norm = sums[np];
  return QMC2D_OK;
}

extern "C" int qmc2d_counters_get(qmc2d_handle *h, qmc2d_counters *c) {
  if (!h || !c) return QMC2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaStreamSynchronize(h->stream));
  int n = std::max(h->nw, h->rmc.nrep);
  std::vector<double> v((size_t)n * 4);
  int ncap = 0;
  CK(cudaMemcpy(v.data(), h->d_cnt, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&ncap, h->br.ncapped, sizeof(int), cudaMemcpyDeviceToHost));
  std::memset(c, 0, sizeof(*c));
  for (int w = 0; w < n; w++) {
    c->accepted += v[4 * w];
    c->proposed += v[4 * w + 1];
    c->forced += v[4 * w + 2];
  }
  c->max_weight_capped = ncap;
  return QMC2D_OK;
}

static int run_moves(qmc2d_handle *h, int nstp, int dmc, double delta, double etrial,
                     double mmult, int mage) {
  q2d::MoveArgs a{};
  a.nw = h->nw;
  a.dmc = dmc;
  a.scr = h->d_mscr;
  a.delta = delta;
  a.mage = mage;
  a.etrial = etrial;
  a.mmult = mmult;
  a.ecut = dmc ? h->dmc_ecut : 0.0;
  a.seed = h->seed;
  a.step0 = h->move_counter;
  a.blk = h->d_blk;
  a.blk_norm = h->d_norm;
  a.cnt = h->d_cnt;
  a.wate = dmc ? h->d_wate : nullptr;
  a.status = h->d_status;
  a.orb_inv = move_orb_inv(h) ? 1 : 0;
  if (h->hs.delta != delta && h->hs.adrift != 0.0) {
    h->hs.delta = delta;
    CK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
  }
  for (int istp = 0; istp < nstp; istp++) {
    a.step0 = h->move_counter + (uint32_t)istp;
    a.first = istp == 0;
    {
      ProfScope ps(h, QMC2D_KERNEL_PAIRS, h->stream);
      CK(q2d::launch_pairs(h->hs, h->ds, h->pop[h->cur], a, h->stream));
    }
    if (a.orb_inv) {
      ProfScope ps(h, QMC2D_KERNEL_ORB_INV, h->stream);
      CK(q2d::launch_orb_inv(h->hs, h->ds, a, h->stream));
    }
    CK(join_side(h));  // the pair and inversion kernels read only x, g and the scratch
    {
      ProfScope ps(h, QMC2D_KERNEL_MOVE, h->stream);
      CK(q2d::launch_move(h->hs, h->ds, h->pop[h->cur], a, h->stream));
    }
  }
  h->move_counter += (uint32_t)nstp;
  return QMC2D_OK;
}

extern "C" int qmc2d_vmc(qmc2d_handle *h, int nstp, double delta, int mage) {
  if (!h || nstp < 0 || !(delta > 0.0)) return QMC2D_ERR_ARG;
  if (h->nw <= 0) {
    q2d::set_error("qmc2d_vmc: empty population");
    return QMC2D_ERR_STACK;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream));
  int st = run_moves(h, nstp, 0, delta, 0.0, 0.0, mage);
  if (st) return st;
  return sync_status(h, h->nw);
}

extern "C" int qmc2d_dmc(qmc2d_handle *h, int nstp, int mmstep, double delta, double etrial,
                         double mmult, int mage) {
  if (!h || nstp < 0 || mmstep <= 0 || !(delta > 0.0)) return QMC2D_ERR_ARG;
  if (h->nw <= 0) {
    q2d::set_error("qmc2d_dmc: empty population");
    return QMC2D_ERR_STACK;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream));
  for (int gen = 0; gen < nstp; gen++) {
    int st = run_moves(h, mmstep, 1, delta, etrial, mmult, mage);
    if (st) return st;
    {
      ProfScope ps(h, QMC2D_KERNEL_BRANCH, h->stream);
      CK(q2d::launch_branch(h->nw, h->d_wate, h->seed, h->gen_counter, h->br, h->stream));
    }
    int nxt = 1 - h->cur;
    {
      ProfScope ps(h, QMC2D_KERNEL_GATHER, h->stream);
      CK(q2d::launch_gather(h->hs, h->pop[h->cur], h->pop[nxt], h->br.src, h->nw, h->stream));
    }
    h->cur = nxt;
    h->gen_counter++;
  }
  return sync_status(h, h->nw);
}

// ------------------------------------------- DMC across ranks (branch2)
extern "C" int qmc2d_dmc_weights(qmc2d_handle *h, int mmstep, double delta, double etrial,
                                 double mmult, int mage, double *wate) {
  if (!h || mmstep <= 0 || !(delta > 0.0) || !wate) return QMC2D_ERR_ARG;
  if (h->nw <= 0) {
    q2d::set_error("qmc2d_dmc_weights: empty population");
    return QMC2D_ERR_STACK;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream));
  int st = run_moves(h, mmstep, 1, delta, etrial, mmult, mage);
  if (st) return st;
  CK(cudaMemcpyAsync(wate, h->d_wate, sizeof(double) * h->nw, cudaMemcpyDeviceToHost,
                     h->stream));
  return sync_status(h, h->nw);
}

extern "C" int qmc2d_population_resample(qmc2d_handle *h, const int *src) {
  if (!h || !src) return QMC2D_ERR_ARG;
  for (int j = 0; j < h->nw; j++)
    if (src[j] < 0 || src[j] >= h->nw) {
      q2d::set_error("qmc2d_population_resample: source slot out of range");
      return QMC2D_ERR_ARG;
    }
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  CK(cudaMemcpyAsync(h->br.src, src, sizeof(int) * h->nw, cudaMemcpyHostToDevice, h->stream));
  const int nxt = 1 - h->cur;
  {
    ProfScope ps(h, QMC2D_KERNEL_GATHER, h->stream);
    CK(q2d::launch_gather(h->hs, h->pop[h->cur], h->pop[nxt], h->br.src, h->nw, h->stream));
  }
  h->cur = nxt;
  h->gen_counter++;
  CK(cudaStreamSynchronize(h->stream));
  return QMC2D_OK;
}

extern "C" int qmc2d_record_len(qmc2d_handle *h, int *len) {
  if (!h || !len) return QMC2D_ERR_ARG;
  *len = 4 * h->N + h->nt + h->nprops + 2;
  return QMC2D_OK;
}

static int records(qmc2d_handle *h, int n, const int *slots, double *buf_dev, void *stream,
                   int unpack) {
  if (!h || n < 0 || n > h->cap || (n > 0 && (!slots || !buf_dev))) return QMC2D_ERR_ARG;
  for (int k = 0; k < n; k++)
    if (slots[k] < 0 || slots[k] >= h->cap) {
      q2d::set_error("qmc2d_records_pack/unpack: slot out of range");
      return QMC2D_ERR_ARG;
    }
  if (n == 0) return QMC2D_OK;
  CK(cudaSetDevice(h->device));
  CK(join_side(h));
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  // the slot list goes through the comb's rank scratch (cap ints), which no
  // other call uses between a generation's weights and its resample
  CK(cudaMemcpyAsync(h->br.zrank, slots, sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CK(q2d::launch_records(h->hs, h->pop[h->cur], h->br.zrank, buf_dev, n, unpack, st));
  CK(cudaStreamSynchronize(st));
  return QMC2D_OK;
}

extern "C" int qmc2d_records_pack(qmc2d_handle *h, int n, const int *slots, double *buf_dev,
                                  void *stream) {
  return records(h, n, slots, buf_dev, stream, 0);
}

extern "C" int qmc2d_records_unpack(qmc2d_handle *h, int n, const int *slots,
                                    const double *buf_dev, void *stream) {
  return records(h, n, slots, const_cast<double *>(buf_dev), stream, 1);
}
