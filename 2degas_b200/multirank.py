"""DMC over several ranks: one population (handle) per rank and GPU, and
branch2's comb over the walkers of all ranks (reptation.f:2162-2273).

Per generation every rank
  1. advances its walkers and weights (qmc2d_dmc_weights; dmc,
     reptation.f:894-906),
  2. all-gathers the weights (MPI_ALLGATHER, :2185; here torch.distributed,
     NCCL between GPUs or gloo on CPU),
  3. computes the same comb and exchange plan (qmc2d_comb_plan: the global
     comb, the reference's send/receive loop :2214-2249 and prov_dest's
     in-rank distribution :2250-2258),
  4. packs the walker records it sends into one device buffer per peer,
     exchanges them with batched point-to-point sends and receives
     (send/receive, :2275-2318) and unpacks the ones it receives into their
     empty slots,
  5. copies walkers within the rank (qmc2d_population_resample).

The comb's uniforms come from one Philox stream shared by all ranks (the
reference's rannyu2), keyed by `comb_seed`; with one rank a generation is
exactly qmc2d_dmc's.
"""
import ctypes

import numpy as np

from . import _capi


def comb_plan(lib, wate_all, nproc, nconf, seed, gen, rank):
    """qmc2d_comb_plan: returns (src, sends, recvs, ncapped); sends and
    recvs are lists of (peer rank, slot) in exchange order."""
    w = np.ascontiguousarray(wate_all, dtype=np.float64)
    src = np.zeros(nconf, dtype=np.int32)
    srank, sslot, rrank, rslot = (np.zeros(max(nconf, 1), dtype=np.int32) for _ in range(4))
    ns, nr, nc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    pi = lambda a: a.ctypes.data_as(_capi.PI)  # noqa: E731
    _capi.check(lib, lib.qmc2d_comb_plan(nproc, nconf, w.ctypes.data_as(_capi.PD), seed,
                                         gen & 0xFFFFFFFF, rank, pi(src), ctypes.byref(ns),
                                         pi(srank), pi(sslot), ctypes.byref(nr), pi(rrank),
                                         pi(rslot), ctypes.byref(nc)))
    sends = list(zip(srank[:ns.value].tolist(), sslot[:ns.value].tolist()))
    recvs = list(zip(rrank[:nr.value].tolist(), rslot[:nr.value].tolist()))
    return src, sends, recvs, nc.value


class HandleRecords:
    """The walker records of a Handle as device tensors (the device of the
    handle's stream); what dmc_generations needs from a population."""

    def __init__(self, h, device):
        self.h = h
        self.device = device
        self.nw = h.population_size()
        self.record_len = h.record_len()
        self.lib = h.lib

    def weights(self, mmstep, delta, etrial, mmult, mage):
        return self.h.dmc_weights(mmstep, delta, etrial, mmult, mage)

    def pack(self, slots):
        import torch

        buf = torch.empty((len(slots), self.record_len), dtype=torch.float64, device=self.device)
        self.h.records_pack(slots, buf.data_ptr())  # synchronous on the handle's stream
        return buf

    def empty(self, n):
        import torch

        return torch.empty((n, self.record_len), dtype=torch.float64, device=self.device)

    def unpack(self, slots, buf):
        import torch

        if buf.is_cuda:  # the receive ran on the process group's stream
            torch.cuda.current_stream(buf.device).synchronize()
        self.h.records_unpack(slots, buf.data_ptr())

    def resample(self, src):
        self.h.population_resample(src)


def _by_peer(pairs):
    out = {}
    for peer, slot in pairs:
        out.setdefault(peer, []).append(slot)
    return out


def dmc_generations(pop, dist, ngen, mmstep, delta, etrial, mmult, mage, comb_seed, gen0=0,
                    device="cpu"):
    """ngen generations of DMC over all ranks of `dist` (a
    torch.distributed module with an initialised process group, or None for
    one rank); pop is a HandleRecords (or an object with the same methods).
    Every rank takes the same collective steps in the same order. Returns
    the weights capped this rank over the generations."""
    import torch

    rank = dist.get_rank() if dist else 0
    world = dist.get_world_size() if dist else 1
    nconf = pop.nw
    capped = 0
    for g in range(ngen):
        w = np.asarray(pop.weights(mmstep, delta, etrial, mmult, mage), dtype=np.float64)
        if world > 1:
            t = torch.tensor(w, dtype=torch.float64, device=device)
            parts = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(parts, t)
            w_all = torch.cat(parts).cpu().numpy()
        else:
            w_all = w
        src, sends, recvs, nc = comb_plan(pop.lib, w_all, world, nconf, comb_seed, gen0 + g,
                                          rank)
        capped += nc
        ops, incoming = [], []
        for peer, slots in sorted(_by_peer(sends).items()):
            ops.append(dist.P2POp(dist.isend, pop.pack(slots), peer))
        for peer, slots in sorted(_by_peer(recvs).items()):
            buf = pop.empty(len(slots))
            ops.append(dist.P2POp(dist.irecv, buf, peer))
            incoming.append((slots, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for slots, buf in incoming:
            pop.unpack(slots, buf)
        pop.resample(src)
    return capped
