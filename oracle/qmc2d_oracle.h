/*
 * qmc2d_oracle.h - CPU oracle for the walker-propagation path of 2degas.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C, FP64, loop-for-loop
 * restatement of the reference Fortran (reptation.f) used to check the CUDA
 * path and as the timed CPU baseline. Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product library never
 * links or calls it.
 *
 * Parity unpinned at the per-configuration level: the reference cannot be
 * compiled here (no Fortran compiler) and ships no per-configuration golden
 * values. What holds it: the loop-for-loop restatement; the reference's own
 * self-check (testd, finite differences of -ln psi against the drift and
 * Laplacian); the reference RNG against the LCG it implements; branch2
 * against a line-by-line transcription; and a coarse statistical match to
 * the one recorded VMC block (n26.res: E_L within 3 %, E_pot within 0.5 %).
 * That block is not reproducible to its error bar (its per-spin kinetic
 * energies are strongly asymmetric although the deck's wave function is
 * spin-symmetric), so it came from a different build than the sources.
 */
#ifndef QMC2D_ORACLE_H
#define QMC2D_ORACLE_H

#include <stdint.h>
#include "../include/qmc2d.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- RNG: the reference's 48-bit LCG in four 12-bit limbs
 * (rannyu/setrn/savern, reptation.f:5247-5351). */
typedef struct oracle_rng {
  int m[4];
  int l[4];
} oracle_rng;
void oracle_setrn(oracle_rng *r, const int seed[4]);
void oracle_savern(const oracle_rng *r, int seed[4]);
double oracle_rannyu(oracle_rng *r);

/* ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based
 * generator the device path uses; restated so the oracle can replay the
 * device's random streams. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Two uniforms in (0,1) from one Philox block (53-bit mantissas). */
void oracle_philox_uniform2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
                            uint32_t c3, double u[2]);

/* ---- the oracle's own reader of a run directory (oracle_input.c): input,
 * readwords, t_read, kread, twistg/SORTTF and read_conf restated
 * (reptation.f:12-708, 4689-4842, 9514, 9818, 2452). Independent of the
 * product library's reader; the data layout is include/qmc2d.h's. */
int oracle_system_read(const char *dir, const char *runid, qmc2d_system **out);
void oracle_system_free(qmc2d_system *sys);
/* Orbital wave vectors of twist (ith, jth); 0, 0: the Gamma-point list. */
int oracle_system_set_twist(qmc2d_system *sys, int ith, int jth);
int oracle_read_configs(const qmc2d_system *sys, const char *dir, const char *suffix,
                        int first, int count, double *x, int *nread);
void oracle_system_sizes(const qmc2d_system *sys, int *nptot, int *ntypes, int *n_props);

/* ---- per-evaluation scratch (the reference's /c_dist/, /scratch/ commons) */
typedef struct oracle_work oracle_work;
oracle_work *oracle_work_new(const qmc2d_system *sys);
void oracle_work_free(oracle_work *w);

/* compute_properties(1) (reptation.f:2661-2727): x(2,N) ->
 * g = -grad ln psi (2,N), hl = -lap ln psi per type, p (n_props), s.
 * Returns 0, or QMC2D_ERR_SINGULAR on a zero pivot. Sets *underflow to 1 if
 * the reference's early return of slater_excitations fired (exp(-2 ltf) <= 0,
 * reptation.f:10087-10092). */
int oracle_compute_properties(const qmc2d_system *sys, oracle_work *w, const double *x,
                              double *g, double *hl, double *p, double *s, int *underflow);

/* ---- walker record (x_old, g_old, h_old, p_old, s_old, age) */
typedef struct oracle_walker {
  double *x, *g, *p;
  double h[QMC2D_MAX_TYPES];
  double s;
  double age;
} oracle_walker;

/* Random draws for one move. kind: 0 = the cos(pi u) draw of coordinate j,
 * 1 = the log(u) draw of coordinate j, 2 = the Metropolis draw (j = 0). */
typedef double (*oracle_uniform_fn)(void *ctx, int kind, int j);

/* move + metropolis_test (reptation.f:4617-4680, 2622-2659) on one walker.
 * new_* are scratch for the proposal (x/g 2N, p n_props). Returns the
 * acceptance probability; *accepted and *elocal are metropolis_test's
 * outcome (elocal = 0.5*(E_new+E_old) on acceptance, E_old otherwise). */
double oracle_move(const qmc2d_system *sys, oracle_work *w, oracle_walker *wk, double delta,
                   int mage, oracle_uniform_fn U, void *ctx, double *xn, double *gn,
                   double *pn, int *accepted, double *elocal, int *status);

/* The reference's VMC for one block of nstp steps from configuration x0
 * (read_conf + vmc, reptation.f:973-1017, 2452-2491) with its own RNG
 * seeded as `input` does for rank 0 (seed(4)=2*seed(4)+1, reptation.f:38).
 * rng_order selects which rannyu() of cos(pi*rannyu())*sqrt(-2 var
 * log(rannyu())) is drawn first (0: cos argument first).
 * Outputs: blk (n_props block sums of p_old), x_final (2N), seed_out (the
 * savern state), naccept. Returns 0 or an error status. */
int oracle_vmc_rannyu(const qmc2d_system *sys, const double *x0, int nstp, double delta,
                      int mage, const int seed[4], int rng_order, double *blk,
                      double *x_final, int seed_out[4], long *naccept);

/* VMC with the device's Philox streams: nw walkers, nstp steps starting at
 * global step `step0`. Walker w, step t, coordinate j = 2*ip + d draws
 * (u_cos, u_log) = philox(seed, c0 = j, c1 = w, c2 = t, c3 = 0) and the
 * Metropolis draw is u[0] of c0 = 0xFFFFFFFE.
 * x,g,p,h,s,age hold the population on entry/exit (walker-major).
 * blk accumulates sum over walkers and steps of p_old (weight 1). */
int oracle_vmc_philox(const qmc2d_system *sys, int nw, int nstp, double delta, int mage,
                      uint64_t seed, long step0, double *x, double *g, double *hl, double *p,
                      double *s, double *age, double *blk, long *naccept);

/* Evaluate nw configurations into walker records (read_conf). */
int oracle_population_init(const qmc2d_system *sys, int nw, const double *x, double *g,
                           double *hl, double *p, double *s, double *age);

/* branch2's fixed-population comb (reptation.f:2162-2273) for one rank:
 * wate (nw, capped at wmult=10 in place), uniforms r[] drawn in order
 * (as many as nint(sum of fractional parts) requests; pass at least nw).
 * Output mult[nw] and src[nw]: the walker slot each new slot copies from,
 * with prov_dest's in-rank assignment (reptation.f:2260-2271, 2320).
 * Returns the number of uniforms consumed, or -1 on error. */
int oracle_branch2(int nw, double *wate, const double *r, int *mult, int *src, int *ncapped);

/* DMC generations with the device's Philox streams (dmc, reptation.f:872-922).
 * Comb uniform i of generation t: philox(seed, c0 = i, c1 = 0xFFFFFFFF,
 * c2 = t, c3 = 1). Walker moves as oracle_vmc_philox with c2 = global move
 * index. blk accumulates p_old * running weight after every move. */
int oracle_dmc_philox(const qmc2d_system *sys, int nw, int ngen, int mmstep, double delta,
                      double etrial, double mmult, int mage, uint64_t seed, long gen0,
                      long move0, double *x, double *g, double *hl, double *p, double *s,
                      double *age, double *blk, double *blk_norm, long *naccept);

/* Single-electron VMC sweeps with the device's Philox streams
 * (qmc2d_vmc_single; oracle_single.c): nsweep sweeps over electrons 0..N-1
 * of each walker, every ratio and drift from a full evaluation. x holds the
 * walkers on entry; x, g, hl, p, s, age the final records; blk accumulates
 * the walker's properties after every sweep (p(jacc) = the sweep's mean
 * acceptance probability); naccept counts accepted single-electron moves. */
int oracle_vmc_single(const qmc2d_system *sys, int nw, int nsweep, double delta, uint64_t seed,
                      long sweep0, double *x, double *g, double *hl, double *p, double *s,
                      double *age, double *blk, long *naccept);

/* ---- reptation (rmc, reptation.f:1286-2160) for one reptile with Philox
 * draws. Path beads are held in a ring of n_buffer = ntau + mdelta slots. */
typedef struct oracle_reptile oracle_reptile;
oracle_reptile *oracle_reptile_new(const qmc2d_system *sys, const qmc2d_rmc_params *prm);
void oracle_reptile_free(oracle_reptile *r);
/* read_path (reptation.f:1775-1802) from ntau configurations. */
int oracle_reptile_init(const qmc2d_system *sys, oracle_reptile *r, const double *x);
/* nstp reptation moves; reptile id `rid` selects the Philox stream:
 * move t draws (direction, length) = philox(seed, c0=0xFFFFFFF0, c1=rid, c2=t, c3=2),
 * bead b's Gaussians (u_cos, u_log) from c0 = j, c1 = rid, c2 = t, c3 = 3 + b,
 * bead b's Langevin accept from u[0] of c0 = 0xFFFFFFFE, c3 = 3 + b, and the
 * global accept from u[0] of c0 = 0xFFFFFFFD, c3 = 2. blk accumulates p_old. */
int oracle_reptile_run(const qmc2d_system *sys, oracle_reptile *r, int rid, uint64_t seed,
                       long step0, int nstp, double *blk, long *naccept);
/* Copy the current path out (ntau beads in path order): x and props. */
void oracle_reptile_path(const oracle_reptile *r, double *x, double *p);

#ifdef __cplusplus
}
#endif
#endif
