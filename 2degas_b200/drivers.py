"""The reference's method loops over the C-ABI, block by block: vmc
(reptation.f:970-1016), dmc (:872-922) and rmc (:1286-1311), each ending a
block the way averages(3) does (:4305-4434): the cumulative sums, the block
report of the scalar properties (unit 6), the rho_k files, the reptation
estimator files, and restart(1).

Arguments follow the reference's input commands (reptation.f:737-807):
    vmc nblk nstp delta nskip       -> vmc(handle, nblk, nstp, delta)
    dmc nblk nstp delta ntarget mmstep etrial mage mmult
                                    -> dmc(handle, nblk, nstp, delta, etrial,
                                           mmstep, mage, mmult)
    rmc nblk nstp delta ntau ntauskip mdelta etrial mage mage_r
                                    -> rmc(handle, nblk, nstp) after
                                       handle.rmc_init(...) or
                                       handle.restart_read_rmc(...)
The population (vmc, dmc) or the reptiles (rmc) must already be on the
handle (population_set / restart_read, rmc_init / restart_read_rmc). With
out=None nothing is written, and the report goes to log only.
"""
import numpy as np

from . import Stats


def _block_end(handle, st, blk, norm, iblk, who, out, runid, rank, log):
    """averages(3): cumulative sums, report, rho_k files, restart(1)."""
    st.add_block(blk, norm)
    if log is not None:
        log(st.report(blk, norm, who))
    if out is not None:
        if handle.system.s.nrhok > 0:
            st.write_rhok(blk, norm, out, runid)
        handle.restart_write(st, iblk, who, out, runid, rank)


def vmc(handle, nblk, nstp, delta, iblk0=1, stats=None, out=None, runid="run", rank=0,
        log=print):
    """nblk - iblk0 + 1 blocks of nstp VMC steps; mage = nstp * nblk as the
    vmc command sets it. Returns the Stats."""
    st = stats if stats is not None else Stats(handle.system)
    for iblk in range(iblk0, nblk + 1):
        handle.block_reset()
        handle.vmc(nstp, delta, nstp * nblk)
        blk, norm = handle.block_get()
        _block_end(handle, st, blk, norm, iblk, "vmc", out, runid, rank, log)
    return st


def dmc(handle, nblk, nstp, delta, etrial, mmstep=1, mage=50, mmult=2.0, iblk0=1, stats=None,
        out=None, runid="run", rank=0, log=print):
    """DMC blocks of nstp generations; after every block the trial energy
    becomes the cumulative mean energy, as averages(3) sets it. Returns
    (Stats, etrial)."""
    st = stats if stats is not None else Stats(handle.system)
    for iblk in range(iblk0, nblk + 1):
        handle.block_reset()
        handle.dmc(nstp, mmstep, delta, etrial, mmult, mage)
        blk, norm = handle.block_get()
        _block_end(handle, st, blk, norm, iblk, "dmc", out, runid, rank, log)
        mean, _, _, _ = st.get()
        etrial = float(mean[0])
    return st, etrial


def rmc(handle, nblk, nstp, est=None, iblk0=1, stats=None, est_stats=None, out=None,
        runid="run", rank=0, log=print):
    """Reptation blocks of nstp moves on the handle's reptiles. With est (a
    qmc2d_rmc_estimators from System.rmc_estimators_setup) the path
    estimators are taken after every move and averaged over the block like
    the path properties, and their files written with the block's.
    Returns (Stats, estimator Stats or None)."""
    st = stats if stats is not None else Stats(handle.system)
    est_st = None
    if est is not None and est.nvalues > 0:
        est_st = est_stats if est_stats is not None else Stats(handle.system, est.nvalues)
    for iblk in range(iblk0, nblk + 1):
        handle.block_reset()
        acc = np.zeros(est.nvalues) if est_st is not None else None
        for _ in range(nstp):
            handle.rmc(1)
            if acc is not None:
                acc += handle.rmc_estimators(est)
        blk, norm = handle.block_get()
        _block_end(handle, st, blk, norm, iblk, "rmc", out, runid, rank, log)
        if est_st is not None:
            # the block sums of the path properties carry weight 1 per
            # reptile and move: the estimators (means over reptiles) likewise
            eblk, enorm = acc * (norm / nstp), norm
            est_st.add_block(eblk, enorm)
            if out is not None:
                est_st.write_estimators(est, eblk, enorm, out, runid)
    return st, est_st
