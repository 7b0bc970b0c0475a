// batch.cu - many independent populations stepped together (C-ABI
// qmc2d_batch_*). Each population is a handle of its own system (its own
// N, density, polarisation and walker count); one call advances all of them
// by the same number of VMC steps or DMC generations.
//
// One CUDA graph holds an even number of generations of every population
// (a call of n generations: n rounded down to even, at most
// kMaxGraphGenerations): the launches of population k (pair kernel, move
// kernel and, for DMC, the comb and the gather) go on handle k's stream,
// forked from and joined back to the batch's capture stream, so the
// populations' kernels overlap on the GPU and the host issues one graph
// launch per replay instead of 4-8 launches per population per generation.
// An even number, because the gather ping-pongs between the handle's two
// population buffers: after an even number the buffers are back where the
// graph began, so the same graph replays. The join at the end of a replay
// waits for the slowest population, so longer graphs leave the GPU idle
// less often when the populations' costs differ; what the graph does not
// cover (an odd last generation, or the rest of n) is launched directly.
//
// Lanes (qmc2d_batch_set_lanes): by default every population forks from the
// capture stream at once. With S lanes, at most S populations run at a
// time: the populations are dealt to S chains, largest estimated cost
// first onto the least loaded chain, and each waits for the one before it
// in its chain. Fewer populations in flight keep fewer working sets (move
// scratch, determinant blocks) competing for L2.
//
// A replay repeats the launches' arguments; the Philox move and comb
// counters that must advance are read from a per-population device pair
// {move, generation} (MoveArgs::ctr) set from the handle's host counters
// before the first replay and advanced by a one-thread kernel at the end of
// each replay. The kernels then draw exactly the random numbers that
// qmc2d_vmc / qmc2d_dmc draw for the same handle: a batch call and the same
// calls made handle by handle give the same walkers bit for bit.
//
// The graph is captured again when a call's parameters (time steps, trial
// energies, population sizes, buffer parity) differ from the cached one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"
#include "handle.h"
#include "kernels.cuh"

constexpr int kMaxGraphGenerations = 16;

struct qmc2d_batch {
  std::vector<qmc2d_handle *> h;
  int device = 0;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  uint32_t *d_ctr = nullptr;  // 2 per population: {move, generation}
  cudaGraphExec_t exec = nullptr;
  std::vector<double> key;  // parameters the cached graph was captured with
  int lanes = 0;             // concurrent chains of populations (0: all at once)
};

namespace {

int bfail(cudaError_t e, const char *what) {
  q2d::set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return QMC2D_ERR_CUDA;
}

#define BCK(call)                                          \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return bfail(e_, #call);        \
  } while (0)

// Launches of `ngen` generations of population k on its stream, starting at
// generation offset g0 of the current call (counters read from d_ctr + 2k).
cudaError_t enqueue(qmc2d_batch *b, int k, int g0, int ngen, int dmc, double delta,
                    double etrial, double mmult, int mage) {
  qmc2d_handle *h = b->h[k];
  cudaStream_t st = h->stream;
  const uint32_t *ctr = b->d_ctr + 2 * k;
  cudaError_t e;
  for (int g = 0; g < ngen; g++) {
    const int cur = dmc ? (h->cur + g0 + g) & 1 : h->cur;  // only the comb's gather swaps
    q2d::MoveArgs a{};
    a.nw = h->nw;
    a.dmc = dmc;
    a.first = 1;
    a.scr = h->d_mscr;
    a.delta = delta;
    a.mage = mage;
    a.etrial = etrial;
    a.mmult = mmult;
    a.ecut = dmc ? h->dmc_ecut : 0.0;
    a.seed = h->seed;
    a.step0 = (uint32_t)(g0 + g);
    a.blk = h->d_blk;
    a.blk_norm = h->d_norm;
    a.cnt = h->d_cnt;
    a.wate = dmc ? h->d_wate : nullptr;
    a.status = h->d_status;
    a.orb_inv = move_orb_inv(h) ? 1 : 0;
    a.ctr = ctr;
    if ((e = q2d::launch_pairs(h->hs, h->ds, h->pop[cur], a, st)) != cudaSuccess) return e;
    if ((e = q2d::launch_orb_inv(h->hs, h->ds, a, st)) != cudaSuccess) return e;
    if ((e = q2d::launch_move(h->hs, h->ds, h->pop[cur], a, st)) != cudaSuccess) return e;
    if (dmc) {
      if ((e = q2d::launch_branch(h->nw, h->d_wate, h->seed, (uint32_t)(g0 + g), h->br, st,
                                  ctr)) != cudaSuccess)
        return e;
      if ((e = q2d::launch_gather(h->hs, h->pop[cur], h->pop[1 - cur], h->br.src, h->nw, st)) !=
          cudaSuccess)
        return e;
    }
  }
  return cudaSuccess;
}

// Estimated cost of one generation of population k: the pair terms and,
// per spin, the determinant work (O(N n^2)).
double pop_cost(const qmc2d_handle *h) {
  double c = 0.5 * h->N * h->N;
  for (int t = 0; t < h->hs.nt; t++) c += (double)h->N * h->hs.np[t] * h->hs.np[t];
  return c * h->nw;
}

// The order to enqueue the populations in and, for each, the population it
// waits for (-1: the fork), for the batch's lanes.
void lane_plan(const qmc2d_batch *b, std::vector<int> *order, std::vector<int> *prev) {
  const int np = (int)b->h.size();
  const int S = b->lanes > 0 && b->lanes < np ? b->lanes : np;
  order->resize(np);
  prev->assign(np, -1);
  for (int k = 0; k < np; k++) (*order)[k] = k;
  if (S == np) return;
  std::vector<double> cost(np);
  for (int k = 0; k < np; k++) cost[k] = pop_cost(b->h[k]);
  std::stable_sort(order->begin(), order->end(),
                   [&](int a, int c) { return cost[a] > cost[c]; });
  std::vector<double> load(S, 0.0);
  std::vector<int> last(S, -1);
  for (int k : *order) {
    const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    (*prev)[k] = last[l];
    last[l] = k;
    load[l] += cost[k];
  }
}

// One step of every population: fork from the master stream (or wait for
// the population before it in its lane), enqueue, advance the counters by
// the generations enqueued, join.
cudaError_t enqueue_all(qmc2d_batch *b, int g0, int ngen, int dmc, const double *delta,
                        const double *etrial, double mmult, int mage) {
  cudaError_t e;
  std::vector<int> order, prev;
  lane_plan(b, &order, &prev);
  if ((e = cudaEventRecord(b->fork, b->master)) != cudaSuccess) return e;
  for (int k : order) {
    qmc2d_handle *h = b->h[k];
    if ((e = cudaStreamWaitEvent(h->stream, prev[k] < 0 ? b->fork : b->join[prev[k]], 0)) !=
        cudaSuccess)
      return e;
    if ((e = enqueue(b, (int)k, g0, ngen, dmc, delta[k], dmc ? etrial[k] : 0.0, mmult, mage)) !=
        cudaSuccess)
      return e;
    if ((e = q2d::launch_counters_add(b->d_ctr + 2 * k, (uint32_t)ngen, dmc ? (uint32_t)ngen : 0u,
                                      h->stream)) != cudaSuccess)
      return e;
    if ((e = cudaEventRecord(b->join[k], h->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(b->master, b->join[k], 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int run(qmc2d_batch *b, int n, int dmc, const double *delta, const double *etrial, double mmult,
        int mage) {
  if (!b || n < 0 || !delta || (dmc && !etrial)) return QMC2D_ERR_ARG;
  const size_t np = b->h.size();
  for (size_t k = 0; k < np; k++) {
    if (!(delta[k] > 0.0)) return QMC2D_ERR_ARG;
    if (b->h[k]->nw <= 0) {
      q2d::set_error("qmc2d_batch: a population is empty");
      return QMC2D_ERR_STACK;
    }
  }
  if (n == 0) return QMC2D_OK;
  BCK(cudaSetDevice(b->device));
  std::vector<uint32_t> ctr(2 * np);
  for (size_t k = 0; k < np; k++) {
    qmc2d_handle *h = b->h[k];
    BCK(join_side(h));
    BCK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * h->nw, h->stream));
    if (h->hs.delta != delta[k] && h->hs.adrift != 0.0) {  // the drift cutoff reads delta
      h->hs.delta = delta[k];
      BCK(cudaMemcpyAsync(h->ds, &h->hs, sizeof(q2d::DevSys), cudaMemcpyHostToDevice, h->stream));
    }
    ctr[2 * k] = h->move_counter;
    ctr[2 * k + 1] = h->gen_counter;
  }
  // the counters and every handle's pending work precede the first replay
  BCK(cudaMemcpy(b->d_ctr, ctr.data(), sizeof(uint32_t) * 2 * np, cudaMemcpyHostToDevice));
  for (size_t k = 0; k < np; k++) BCK(cudaStreamSynchronize(b->h[k]->stream));
  const int gpg = std::min(n & ~1, kMaxGraphGenerations);  // generations per replay
  const int replays = gpg > 0 ? n / gpg : 0;
  if (replays > 0) {
    std::vector<double> key = {(double)dmc, mmult, (double)mage, (double)gpg,
                               (double)b->lanes};
    for (size_t k = 0; k < np; k++) {
      key.push_back(delta[k]);
      key.push_back(dmc ? etrial[k] : 0.0);
      key.push_back((double)b->h[k]->nw);
      key.push_back((double)b->h[k]->cur);
      key.push_back((double)(intptr_t)b->h[k]);
      key.push_back(b->h[k]->dmc_ecut);
    }
    if (!b->exec || key != b->key) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      BCK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeRelaxed));
      cudaError_t e = enqueue_all(b, 0, gpg, dmc, delta, etrial, mmult, mage);
      cudaError_t e2 = cudaStreamEndCapture(b->master, &g);
      if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bfail(e, "qmc2d_batch: capture");
      }
      BCK(e2);
      e = cudaGraphInstantiate(&b->exec, g, 0);
      cudaGraphDestroy(g);
      BCK(e);
      b->key = key;
    }
    for (int r = 0; r < replays; r++) BCK(cudaGraphLaunch(b->exec, b->master));
  }
  const int rest = n - replays * gpg;
  if (rest > 0) BCK(enqueue_all(b, 0, rest, dmc, delta, etrial, mmult, mage));
  BCK(cudaStreamSynchronize(b->master));
  int worst = QMC2D_OK;
  for (size_t k = 0; k < np; k++) {
    qmc2d_handle *h = b->h[k];
    h->move_counter += (uint32_t)n;
    if (dmc) {
      h->gen_counter += (uint32_t)n;
      h->cur = (h->cur + n) & 1;
    }
    const int st = q2d_sync_status(h, h->nw);
    if (st && !worst) worst = st;
  }
  return worst;
}

}  // namespace

extern "C" int qmc2d_batch_create(qmc2d_handle *const *handles, int n, qmc2d_batch **out) {
  if (!handles || n <= 0 || !out) {
    q2d::set_error("qmc2d_batch_create: bad argument");
    return QMC2D_ERR_ARG;
  }
  *out = nullptr;
  qmc2d_batch *b = new qmc2d_batch();
  b->device = handles[0]->device;
  for (int k = 0; k < n; k++) {
    if (!handles[k] || handles[k]->device != b->device) {
      delete b;
      q2d::set_error("qmc2d_batch_create: null handle or handles on different devices");
      return QMC2D_ERR_ARG;
    }
    for (int j = 0; j < k; j++)
      if (handles[j] == handles[k]) {
        delete b;
        q2d::set_error("qmc2d_batch_create: a handle appears twice");
        return QMC2D_ERR_ARG;
      }
    b->h.push_back(handles[k]);
  }
  auto fail = [&](cudaError_t e, const char *what) {
    qmc2d_batch_destroy(b);
    return bfail(e, what);
  };
  cudaError_t e;
  if ((e = cudaSetDevice(b->device)) != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "cudaStreamCreate");
  if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
    return fail(e, "cudaEventCreate");
  b->join.assign(n, nullptr);
  for (int k = 0; k < n; k++)
    if ((e = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e, "cudaEventCreate");
  if ((e = cudaMalloc(&b->d_ctr, sizeof(uint32_t) * 2 * n)) != cudaSuccess)
    return fail(e, "cudaMalloc");
  *out = b;
  return QMC2D_OK;
}

extern "C" int qmc2d_batch_destroy(qmc2d_batch *b) {
  if (!b) return QMC2D_OK;
  cudaSetDevice(b->device);
  if (b->master) cudaStreamSynchronize(b->master);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->master) cudaStreamDestroy(b->master);
  cudaFree(b->d_ctr);
  delete b;
  return QMC2D_OK;
}

extern "C" int qmc2d_batch_set_lanes(qmc2d_batch *b, int lanes) {
  if (!b || lanes < 0) {
    q2d::set_error("qmc2d_batch_set_lanes: bad argument");
    return QMC2D_ERR_ARG;
  }
  b->lanes = lanes;
  return QMC2D_OK;
}

extern "C" int qmc2d_batch_vmc(qmc2d_batch *b, int nstp, const double *delta, int mage) {
  return run(b, nstp, 0, delta, nullptr, 0.0, mage);
}

extern "C" int qmc2d_batch_dmc(qmc2d_batch *b, int ngen, const double *delta,
                               const double *etrial, double mmult, int mage) {
  return run(b, ngen, 1, delta, etrial, mmult, mage);
}
