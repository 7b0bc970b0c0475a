/*
 * qmc2d.h - C-ABI of the B200 walker-propagation library for the 2D
 * electron-gas QMC code 2degas (Slater-Jastrow-backflow VMC/DMC/RQMC).
 *
 * The reference has no formal plugin API: its hot path is a set of Fortran
 * subroutines without arguments that talk through COMMON blocks (ewald.h).
 * Every entry point below replaces one of those subroutines (or a loop of
 * them) and takes the COMMON-block arrays as plain pointers, in the same
 * Fortran column-major layout, so that a Fortran iso_c_binding shim can pass
 * x_new(mdim,mnp), g_new(mdim,mnp), h_new(mtypes), p_new(m_props) directly.
 *
 * Conventions
 *   - Positions/drifts are x(2,N): interleaved (x,y) per electron, electrons
 *     ordered type by type (all "up" then all "down"), as ewald.h's x_new.
 *   - Property vectors follow the reference's p_new index map (input,
 *     reptation.f:577-637), 0-based here: see QMC2D_J* below.
 *   - All pointers are HOST pointers unless the name ends in _dev.
 *   - Every call returns an int status (QMC2D_OK == 0); nothing throws
 *     across the ABI. Device-side failures (singular Slater matrix,
 *     non-finite energy) are reported through status words read after
 *     each launch.
 *   - One handle per host thread; each handle owns one CUDA stream.
 */
#ifndef QMC2D_H
#define QMC2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---------------------------------------------------------------- status */
enum qmc2d_status {
  QMC2D_OK = 0,
  QMC2D_ERR_ARG = 1,          /* bad argument / size */
  QMC2D_ERR_IO = 2,           /* input file missing or unreadable */
  QMC2D_ERR_PARSE = 3,        /* malformed keyword record or table */
  QMC2D_ERR_UNSUPPORTED = 4,  /* keyword/feature outside the walker path */
  QMC2D_ERR_CUDA = 5,         /* CUDA runtime error (message in qmc2d_last_error) */
  QMC2D_ERR_NOMEM = 6,        /* device or host allocation failed */
  QMC2D_ERR_SINGULAR = 7,     /* zero pivot in a Slater matrix
                                 (reference: stop 'slater_bckflw_orbitals', reptation.f:10318) */
  QMC2D_ERR_NONFINITE = 8,    /* NaN/Inf local energy or weight */
  QMC2D_ERR_POPULATION = 9,   /* population outside the handle's capacity */
  QMC2D_ERR_LIMIT = 10,       /* size beyond a compiled limit */
  QMC2D_ERR_STACK = 11        /* walker stack empty/full (reptation.f:2374, 2416) */
};

/* Compiled limits. The reference's ewald.h limits (mnp=166, morbit=42,
 * mgrid=901, mnk=196) are dropped where the device code does not need them. */
#define QMC2D_MAX_TYPES 2
#define QMC2D_MAX_TABLES 16
#define QMC2D_MAX_NP 162          /* electrons per walker */
#define QMC2D_MAX_ORB 162         /* orbitals (electrons) per spin determinant */
#define QMC2D_MAX_NK 512          /* half-space k vectors */
#define QMC2D_NAME_LEN 64
#define QMC2D_MAX_EST 4           /* path-estimator records of each kind */
#define QMC2D_RECORD_LEN 256

/* ------------------------------------------------------- property layout
 * Scalar properties, reference names and 1-based indices from
 * reptation.f:577-628 (jetot=1, jltf=2, jacc=3, jpot(0)=4, jkin(0)=5, je2=6,
 * jgg=7, then pot_<t>, kin_<t>, un_<t> per type, then efp), followed by
 * rhok (2*nk doubles per type that has 'rhok'). Here 0-based. */
#define QMC2D_JETOT 0
#define QMC2D_JLTF 1
#define QMC2D_JACC 2
#define QMC2D_JPOT0 3
#define QMC2D_JKIN0 4
#define QMC2D_JE2 5
#define QMC2D_JGG 6
#define QMC2D_JPOT(nt, it) (7 + (it))
#define QMC2D_JKIN(nt, it) (7 + (nt) + (it))
#define QMC2D_JUN(nt, it) (7 + 2 * (nt) + (it))
#define QMC2D_JEFP(nt) (7 + 3 * (nt))
#define QMC2D_NSCALAR(nt) (8 + 3 * (nt))

/* ------------------------------------------------------------- the system
 * What the reference's `input` (reptation.f:12-710) leaves in COMMON for the
 * walker path: particle types, box, k vectors, orbital wave vectors, spline
 * tables and option flags. Filled by qmc2d_system_read() or by the caller. */
typedef struct qmc2d_table {
  char name[QMC2D_NAME_LEN];
  int ngrid;        /* knots 0..ngrid (t_read, reptation.f:4701-4704) */
  double *ut;       /* (ngrid+1)*4: ut[4*i+c] == ut(i,c+1,table) */
  double tail;      /* v2 tail constant (reptation.f:250) */
  int iexp;         /* getf_0 multiplies by (1/r)**iexp (reptation.f:4110) */
  int nk_ewald;     /* number of k-space v_k after the knots, 0 if none */
  double *vk;       /* nk_ewald+1: v_k (k=1..nk_ewald) then v_k0 (reptation.f:4714-4720) */
} qmc2d_table;

typedef struct qmc2d_system {
  int ndim;                                /* must be 2 */
  int ntypes;                              /* 1 or 2 */
  char type_name[QMC2D_MAX_TYPES][QMC2D_NAME_LEN];
  char x_file[QMC2D_MAX_TYPES][QMC2D_NAME_LEN];
  int np[QMC2D_MAX_TYPES];                 /* particles per type */
  int ipfrst[QMC2D_MAX_TYPES];             /* 0-based first particle of the type */
  int nptot;
  int npnorm;                              /* moving particles (hbs2m != 0) */
  double hbs2m[QMC2D_MAX_TYPES];           /* hbar^2/2m per type */
  double el[2], eli[2];                    /* box sides and inverses ('pbc') */
  int nk;                                  /* k vectors read by kread */
  double *kvec;                            /* 2*nk */
  int ngvec;                               /* 2*nk+1 orbital wave vectors */
  double *gvec;                            /* 2*ngvec, in the order the determinant uses */
  double drt, drti, drti2;                 /* knot spacing (shared by all tables) */
  int ntables;
  qmc2d_table tables[QMC2D_MAX_TABLES];
  int iu2[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES];   /* table index, -1 if none */
  int iu3[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES];
  int iub[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES];   /* backflow eta tables */
  int iv2[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES];   /* pair potential tables */
  int irhok[QMC2D_MAX_TYPES];              /* 1-based rhok slot, 0 if not requested */
  int nrhok;
  double v0;                               /* constant potential (Madelung) */
  double adrift;                           /* drift cutoff parameter */
  double delta;                            /* time step of the current run (COMMON /c_sim/);
                                              kinetic's adrift cutoff reads it */
  int ecut;                                /* cut E_L in the RQMC action (fgg) */
  double value_ecut;
  int ntheta;                              /* twists per direction; efp added when != 0 */
  int ith, jth;                            /* current twist (1-based), 0 at Gamma */
  int ibckf;
  int gstorto, wpiu, nodalaction, rejection;
  int seed[4];                             /* 'seed' file / keyword */
  int n_scalar_props;
  int n_props;                             /* scalars + rhok */
  int jrhok;                               /* first rhok index (0-based) */
  int ref_underflow_return;                /* 1: keep the reference's early return when
                                              exp(-2*(-ln psi)) underflows (reptation.f:10087) */
  /* 'mstar', 'cmass' and 'itc' records of the deck (the words after the
   * keyword, reptation.f:210-224), for qmc2d_rmc_estimators_setup */
  int nmstar, ncmass, nitc;
  char mstar_record[QMC2D_MAX_EST][QMC2D_RECORD_LEN];
  char cmass_record[QMC2D_MAX_EST][QMC2D_RECORD_LEN];
  char itc_record[QMC2D_MAX_EST][QMC2D_RECORD_LEN];
} qmc2d_system;

/* Read <dir>/<runid>.sy and every table it names (input, t_read, kread:
 * reptation.f:12-710, 4689-4769). The orbital wave vectors are built at the
 * Gamma point (reptation.f:674-708) or, when 'ntwists' is present, for twist
 * (1,1) (tabc, reptation.f:9559). Unsupported keywords give
 * QMC2D_ERR_UNSUPPORTED with the keyword in qmc2d_last_error(). */
int qmc2d_system_read(const char *dir, const char *runid, qmc2d_system **out);
void qmc2d_system_free(qmc2d_system *sys);

/* Rebuild gvec for twist (ith, jth) of an ntheta x ntheta grid: +-k + theta,
 * sorted by |g|^2 with the reference's heapsort (twistg, reptation.f:9818;
 * SORTTF, reptation.f:9514). ith = jth = 0 restores the Gamma-point list. */
int qmc2d_system_set_twist(qmc2d_system *sys, int ith, int jth);

/* Read `count` configurations of all types starting at configuration `first`
 * (0-based) from the per-type files <dir>/<x_file><suffix> (read_conf,
 * reptation.f:2452-2491). x receives count*2*nptot doubles. Returns the
 * number of configurations read in *nread. */
int qmc2d_read_configs(const qmc2d_system *sys, const char *dir, const char *suffix,
                       int first, int count, double *x, int *nread);

const char *qmc2d_last_error(void);
const char *qmc2d_version(void);

/* ------------------------------------------------------------ the handle */
typedef struct qmc2d_handle qmc2d_handle;

typedef struct qmc2d_options {
  int capacity;          /* walkers (or reptile beads) the handle can hold */
  int device;            /* CUDA device ordinal */
  uint64_t seed;         /* Philox key for the device random streams */
} qmc2d_options;

/* Copy the system's tables to the device and allocate walker storage.
 * When one walker's evaluation does not fit a CTA's shared memory (backflow
 * determinants above 45 electrons per spin unpolarised, 49 polarised), each
 * walker slot also gets a block of device memory for its determinant
 * matrices; QMC2D_ERR_LIMIT only if the rest does not fit either. */
int qmc2d_create(const qmc2d_system *sys, const qmc2d_options *opt, qmc2d_handle **out);
int qmc2d_destroy(qmc2d_handle *h);
/* Device memory (bytes, each allocation rounded to 512) that qmc2d_create
 * would allocate for sys at this capacity, computed on the host without a
 * GPU (the per-walker determinant blocks included, sized for the B200's
 * 227 KB of shared memory per CTA); reptation storage (qmc2d_rmc_init) is
 * not included. For admitting
 * work by HBM footprint; the reference has no counterpart (it allocates
 * its COMMON blocks statically). */
int qmc2d_footprint(const qmc2d_system *sys, int capacity, uint64_t *bytes);
/* After qmc2d_system_set_twist on the handle's system, make the handle's
 * orbitals use the new wave vectors (the gvec/gtens reset at each twist of
 * tabc, reptation.f:9581-9616); the population is left as it is, as in the
 * reference, which carries its walkers from one twist to the next. */
int qmc2d_update_twist(qmc2d_handle *h, const qmc2d_system *sys);

/* Precision of the pair passes in compute_properties, VMC and DMC
 * (reptation stays FP64). QMC2D_PRECISION_FP64, the default: every
 * operation in FP64, as the reference. QMC2D_PRECISION_MIXED: the two-body
 * Jastrow pair terms (two_body, reptation.f:2981-3046) and the real-space
 * Ewald pair potential (potential, reptation.f:3986-4030) are evaluated in
 * FP32 from an FP32 copy of their tables, the pair vector coming from the
 * FP64 minimum image; each thread's sums of those terms are compensated
 * (Kahan) and read out in FP64. The u3 and backflow terms, the
 * determinants and inverse, the k-space Ewald sum, energies, weights and
 * accumulators stay FP64. The reference has no counterpart: it computes in
 * FP64 only. */
enum { QMC2D_PRECISION_FP64 = 0, QMC2D_PRECISION_MIXED = 1 };
int qmc2d_set_precision(qmc2d_handle *h, int precision);

/* DMC weight with a local-energy cutoff: with ecut > 0 (Ry per electron)
 * qmc2d_dmc and qmc2d_batch_dmc clamp the E_L that enters the weight
 * exp(-npnorm (E_L - etrial) delta) to etrial +- ecut, which keeps a rare
 * walker with a very negative E_L (near a node or a coalescence) from taking
 * over the population. The reference's dmc (reptation.f:898-903) has no
 * such cutoff; ecut = 0, the default, gives its weights. */
int qmc2d_set_dmc_ecut(qmc2d_handle *h, double ecut);

/* Launch choices of the pair kernel (the proposal and pair passes of a
 * move): walker groups per CTA (1 or 2; 0 = the default, 2) and whether the
 * pair rows are staged in shared memory (stage 0: when they fit; 1: never,
 * read from global memory). Every choice computes the same values.
 * qmc2d_autotune times the four choices on the handle's current population
 * (three launches each after a warm-up; the population is not changed),
 * keeps the fastest and returns it with its time per launch. The reference
 * has no counterpart. */
int qmc2d_set_launch(qmc2d_handle *h, int groups, int stage);
/* Inversion layout of the determinant section (compute_properties, VMC,
 * DMC, reptation) for determinants held in shared memory: 0 (the default)
 * the register-resident Gauss-Jordan over every warp of the CTA, 1 one warp
 * per spin in shared memory with rho_k on the other warps, 2 blocks of
 * eight pivot steps whose panels one warp factors in registers while the
 * spin's other warps wait for the block update (spins of at most 32
 * orbitals; larger ones take layout 0's route). All pivot as zgefa does (the
 * unused row of largest |re|+|im|, reptation.f:9079-9227) and give the same
 * values up to round-off. The reference has no counterpart. */
int qmc2d_set_inversion(qmc2d_handle *h, int layout);
/* Lanes per particle in the pair kernel's two pair passes: 4, 8 or 16
 * (0: the default, 8). Each particle's sums over its partners are split
 * over that many lanes and meet in a fixed shuffle order, so a choice
 * other than 8 changes the sums' rounding (round-off only). qmc2d_autotune
 * times the three after the groups and staging; qmc2d_get_pair_lanes
 * reports the choice in force. */
int qmc2d_set_pair_lanes(qmc2d_handle *h, int lanes);
int qmc2d_get_pair_lanes(qmc2d_handle *h, int *lanes);
/* Where the moves (VMC, DMC) invert their determinants. The batched form
 * runs the orbitals and their inversion in a kernel of its own between the
 * pair kernel and the move kernel, one warp per spin matrix, for spins of
 * at most 32 orbitals held in shared memory; otherwise the move kernel
 * inverts with the inversion layout in force. mode 1 (the default): batched
 * when the population gives at least 10 spin matrices per SM (3 for a
 * single spin): a fuller GPU hides the
 * pivot chains, small populations finish sooner inside the move kernel;
 * 2: batched whenever it fits; 0: never. Both pivot as zgefa does
 * and agree to round-off. get reports whether the next move is batched. The
 * reference has no counterpart. */
int qmc2d_set_move_inversion(qmc2d_handle *h, int mode);
int qmc2d_get_move_inversion(qmc2d_handle *h, int *batched);
/* qmc2d_autotune also times the three inversion layouts on the evaluation
 * kernel over the population's configurations (three launches each into the
 * handle's staging buffers; the population is not changed) and keeps the
 * faster; *ms is the chosen pair-kernel time per launch. */
int qmc2d_autotune(qmc2d_handle *h, int *groups, int *stage, double *ms);
/* What qmc2d_autotune times (a bit mask, 7 by default): 1 the pair kernel's
 * walker groups and staging (every choice gives the same values bit for
 * bit), 2 its lanes per particle, 4 the inversion layout (these two change
 * the rounding). Choices outside the mask keep their current values. */
int qmc2d_set_autotune_scope(qmc2d_handle *h, int mask);
/* The launch choices in force: pair-kernel walker groups and staging, and
 * the inversion layout. */
int qmc2d_get_launch(qmc2d_handle *h, int *groups, int *stage, int *inversion);

/* Batches: many independent populations (handles of different systems, on
 * one device) advanced together. The reference runs one population per
 * process and has no counterpart. A call of n steps captures one CUDA
 * graph holding min(n rounded down to even, 16) steps of every population
 * (each handle's launches on its own stream, forked from and joined to the
 * batch's stream), replays it, and launches the rest directly; the
 * populations' kernels overlap on the GPU. The Philox counters advance in
 * device memory, so a batch call gives the walkers, block sums and
 * counters that the same qmc2d_vmc / qmc2d_dmc calls made handle by handle
 * give. The handles stay usable on their own between batch calls, and must
 * outlive the batch. */
typedef struct qmc2d_batch qmc2d_batch;
int qmc2d_batch_create(qmc2d_handle *const *handles, int n, qmc2d_batch **out);
int qmc2d_batch_destroy(qmc2d_batch *b);
/* At most `lanes` populations in flight at a time (0, the default: all):
 * the populations are dealt to that many chains, largest estimated cost
 * (walkers x (N^2/2 + N sum n^2)) first onto the least loaded chain, each
 * waiting for the one before it. Results do not depend on it. */
int qmc2d_batch_set_lanes(qmc2d_batch *b, int lanes);
/* nstp VMC steps of every population; delta[k]: population k's time step
 * (qmc2d_vmc per handle). */
int qmc2d_batch_vmc(qmc2d_batch *b, int nstp, const double *delta, int mage);
/* ngen DMC generations of one move each (qmc2d_dmc with mmstep 1 per
 * handle); delta[k] and etrial[k] per population. */
int qmc2d_batch_dmc(qmc2d_batch *b, int ngen, const double *delta, const double *etrial,
                    double mmult, int mage);

/* compute_properties (reptation.f:2661): for nw configurations x (2*nptot
 * each) compute g = -grad ln psi (2*nptot), hlap = -lap ln psi per type
 * (ntypes), props (n_props) and the sign s. Host buffers, synchronous. */
int qmc2d_compute_properties(qmc2d_handle *h, int nw, const double *x,
                             double *g, double *hlap, double *props, double *s);

/* Same on device-resident buffers, asynchronous on `stream` (a cudaStream_t,
 * or NULL for the handle's stream). */
int qmc2d_compute_properties_dev(qmc2d_handle *h, int nw, const double *x_dev,
                                 double *g_dev, double *hlap_dev, double *props_dev,
                                 double *s_dev, void *stream);
/* Status of the last qmc2d_compute_properties_dev call on nw walkers: waits
 * for `stream` (NULL: the handle's stream) and reports QMC2D_ERR_SINGULAR
 * or QMC2D_ERR_NONFINITE if any walker had a zero pivot or a non-finite
 * result (the reference stops there, reptation.f:10318), else QMC2D_OK. */
int qmc2d_compute_properties_dev_status(qmc2d_handle *h, int nw, void *stream);

/* No counterpart in the reference. The same evaluation as
 * qmc2d_compute_properties_dev for callers that cannot allocate device
 * memory - a host code that hands out every device buffer from a pool of its
 * own, or a serving loop that must not trigger a cudaMalloc (which can
 * synchronise the device) between requests - and so cannot create a handle.
 * It needs no handle and allocates nothing: the device copy of `sys` and the
 * status words live in a fixed 2 MiB array that every GPU loading the
 * library holds until exit. The caller passes device buffers for the inputs
 * and outputs; the call is asynchronous on `stream` (NULL: the legacy default
 * stream). Limits: at most 65536 walkers per call and tables, k vectors and
 * orbital wave vectors of at most 229376 doubles together; larger requests
 * return QMC2D_ERR_LIMIT, and so does a system whose determinants are too
 * large for one CTA's shared memory (backflow above 45 electrons per spin
 * unpolarised, 49 polarised: a handle keeps those in device memory it
 * allocates). The call copies the system from pageable host memory, so it
 * must never be made while `stream` is being captured into a CUDA graph
 * (QMC2D_ERR_ARG). The first call on a device looks up the array's
 * device address. All
 * calls share the array: calls that overlap on the GPU (other streams, other
 * threads) race on it and must be serialised by the caller. */
int qmc2d_compute_properties_noalloc(const qmc2d_system *sys, int nw, const double *x_dev,
                                     double *g_dev, double *hlap_dev, double *props_dev,
                                     double *s_dev, void *stream);
/* No counterpart in the reference. Status of the last
 * qmc2d_compute_properties_noalloc call on nw walkers, read from the same
 * fixed array without allocating device memory: waits for `stream`, then
 * returns QMC2D_ERR_SINGULAR or QMC2D_ERR_NONFINITE if any walker had a
 * zero pivot or a non-finite result, else QMC2D_OK. A later call on the
 * array overwrites the words, so read them before the next call. */
int qmc2d_compute_properties_noalloc_status(int nw, void *stream);

/* ---------------------------------------------------------- populations
 * A population is the reference's walker stack (x_stack, g_stack, h_stack,
 * s_stack, age_stack, p_stack; ewald.h:166-173) held in HBM. */

/* read_conf (reptation.f:2452): evaluate nw configurations and make them the
 * population (x_old = x, g_old = g, p_old = props, age = 0, p_old(jacc)=1). */
int qmc2d_population_set(qmc2d_handle *h, int nw, const double *x);
int qmc2d_population_size(qmc2d_handle *h, int *nw);
/* Copy the population out (any pointer may be NULL): the walker records of
 * getconf (reptation.f:2369) - x, g (2N each), hl (ntypes), props
 * (n_props), sign and age per walker. */
int qmc2d_population_get(qmc2d_handle *h, double *x, double *g, double *hl, double *props,
                         double *s, double *age);
/* putconf (reptation.f:2409) for a whole population: load walker records
 * that the caller already holds (as returned by qmc2d_population_get),
 * without re-evaluating them. Pinned host buffers make the copies faster. */
int qmc2d_population_load(qmc2d_handle *h, int nw, const double *x, const double *g,
                          const double *hl, const double *props, const double *s,
                          const double *age);
/* The same load without waiting for it: x and g are copied on the handle's
 * stream, the other records on a second stream, and the call returns at
 * once. The next move's pair kernel (which reads only x and g) runs while
 * the other records are still arriving; the move kernel and every other
 * call that uses the population wait for them. The caller must leave the
 * buffers untouched until a call that synchronises the handle (any move,
 * qmc2d_population_get, qmc2d_block_get) has returned; with pageable
 * buffers the copies complete before the call returns. */
int qmc2d_population_load_async(qmc2d_handle *h, int nw, const double *x, const double *g,
                                const double *hl, const double *props, const double *s,
                                const double *age);

/* Block accumulators (averages(1/2), reptation.f:4283-4304): weighted sums
 * of p_old over all walkers and steps since the last reset. */
int qmc2d_block_reset(qmc2d_handle *h);
int qmc2d_block_get(qmc2d_handle *h, double *blk_av /* n_props */, double *blk_norm);

/* Counters of the last run: accepted moves, proposed moves, forced moves. */
typedef struct qmc2d_counters {
  double accepted, proposed, forced, sign_changes;
  double max_weight_capped;   /* branch2 wmult caps (reptation.f:2175) */
} qmc2d_counters;
int qmc2d_counters_get(qmc2d_handle *h, qmc2d_counters *c);

/* ------------------------------------------------------ block statistics
 * averages(3) (reptation.f:4305-4352) on the host: cumulative sums over
 * blocks, the error bars, the block report and the rho_k files. */
typedef struct qmc2d_stats qmc2d_stats;
int qmc2d_stats_create(int n_props, qmc2d_stats **out);
int qmc2d_stats_destroy(qmc2d_stats *st);
/* Fold one block (sums and norm as from qmc2d_block_get, over all walkers):
 * cml_av += blk, cml2 += blk^2 / blk_norm, cml_norm += blk_norm, iblk += 1
 * (reptation.f:4318-4322). */
int qmc2d_stats_add_block(qmc2d_stats *st, const double *blk, double blk_norm);
/* Cumulative means cml_av/cml_norm, errors
 * sqrt(|cml2/cml_norm - mean^2| / (iblk-1)) (0 for one block,
 * reptation.f:4336-4341), cml_norm and the block count; pointers may be NULL.
 * The DMC trial energy of dmc blocks is mean[QMC2D_JETOT] (:4328). */
int qmc2d_stats_get(const qmc2d_stats *st, double *mean, double *err, double *cml_norm,
                    int *iblk);
/* The block report of averages(3): " ===>> <who> block <iblk>", then per
 * scalar property block mean, cumulative mean, error, block norm and name in
 * the reference's format (2e19.11,e9.2,e10.3,2x,a20; :4343-4345), into buf
 * (NUL-terminated; QMC2D_ERR_LIMIT if len is short). *needed gets the size. */
int qmc2d_stats_report(const qmc2d_stats *st, const qmc2d_system *sys, const double *blk,
                       double blk_norm, const char *who, char *buf, size_t len, size_t *needed);
/* write_nonscalar_props for the rho_k slots (reptation.f:4349-4357, 4582):
 * <dir>/<runid>.rhok_<type>, one line per component
 * (2e19.11,e9.2,e10.3,1x,a7,i5). */
int qmc2d_stats_write_rhok(const qmc2d_stats *st, const qmc2d_system *sys, const double *blk,
                           double blk_norm, const char *dir, const char *runid);

/* ---------------------------------------------------------- checkpoints */
/* write_conf (reptation.f:2504): the population's coordinates to the
 * per-type files <dir>/<x_file(type)>.<rank>, one "x y" line per particle,
 * walker after walker; qmc2d_read_configs reads them with suffix ".<rank>". */
int qmc2d_write_conf(qmc2d_handle *h, const qmc2d_system *sys, const char *dir, int rank);
/* restart(1) (reptation.f:4448-4507): <dir>/<runid>.res holds "iblk who",
 * cml_norm, one "cml_av cml2" line per property, the random-stream state
 * line and, when ntheta != 0, "ith jth"; the coordinates go to
 * <dir>/<x_file(type)>.res.<rank>: every walker for who "vmc" or "dmc",
 * every reptile's ntau-bead path for "rmc". The state line holds this
 * library's counter-based streams (seed low and high words, move,
 * generation and reptation counters, three zeros) in the place of the
 * rannyu/rannyu2 seed words. */
int qmc2d_restart_write(qmc2d_handle *h, const qmc2d_system *sys, const qmc2d_stats *st,
                        int iblk, const char *who, const char *dir, const char *runid,
                        int rank);
/* restart(0) (reptation.f:4508-4540) for who "vmc" or "dmc": the .res file
 * back into st and the handle's streams, *iblk = the stored block (the
 * caller continues at mod(iblk, nblk)+1), *etrial = cml_av(jetot)/cml_norm,
 * and the stored configurations become the population (as
 * qmc2d_population_set). */
int qmc2d_restart_read(qmc2d_handle *h, const qmc2d_system *sys, qmc2d_stats *st,
                       const char *who, const char *dir, const char *runid, int rank,
                       int *iblk, double *etrial);
/* restart(0) for who "rmc" followed by read_path (reptation.f:4508-4540,
 * 1775-1802): the .res file back into st and the handle's streams, the
 * stored paths (nrep*prm->ntau configurations, reptile-major, as
 * qmc2d_restart_write writes them) become prm->ntau-bead reptiles as
 * qmc2d_rmc_init makes them: every bead evaluated again, the bead
 * acceptances and path properties recomputed, ages zero, as read_path does.
 * The reptation counter continues from the stored one. */

/* VMC: nstp steps of move + metropolis_test + averages(2) on every walker
 * (vmc loop body, reptation.f:995-1003; move :4617; metropolis_test :2622).
 * mage forces a move after that many consecutive rejections (<=0: never). */
int qmc2d_vmc(qmc2d_handle *h, int nstp, double delta, int mage);

/* DMC: nstp generations; each walker makes mmstep moves, its weight is
 * multiplied by min(mmult, exp(-npnorm*(E_L-etrial)*delta)) after each, and
 * the population is resampled with branch2's fixed-population comb
 * (dmc, reptation.f:872-922; branch2 :2162-2273). */
int qmc2d_dmc(qmc2d_handle *h, int nstp, int mmstep, double delta, double etrial,
              double mmult, int mage);

/* Single-electron moves. The reference moves all electrons at once (move,
 * reptation.f:4617-4680); this is the same importance-sampled Metropolis
 * step (drift from -grad ln|psi|, the Green's-function ratio and the
 * acceptance of metropolis_test, :2622-2659) applied to one electron at a
 * time, for decks whose wave function is a Slater determinant of plane
 * waves times a two-body Jastrow: no u3, and backflow tables that are
 * identically zero (the reference carries its determinant in the backflow
 * routine, so a plain determinant is a zero eta table). Otherwise
 * QMC2D_ERR_UNSUPPORTED.
 * nsweep sweeps of every walker of the population: each sweep moves
 * electrons 0..N-1 in turn; the determinant ratio comes from the inverse
 * Slater matrices, which stay resident on the device for the whole call and
 * are updated by Sherman-Morrison after every accepted move, and rebuilt
 * from the positions and inverted from scratch (FP64) at the start and
 * after every `refresh` single-electron moves (0: at the start only).
 * After each sweep the walker's properties are measured and added to the
 * block sums with weight 1, as qmc2d_vmc does per step, p(jacc) being the
 * mean acceptance probability of the sweep's N moves. The counters count
 * single-electron moves. Random draws: electron i, coordinate d of walker
 * slot w in sweep t uses Philox (c0 = 2i+d, c1 = w, c2 = t, c3 = 0x5100)
 * and its acceptance u[0] of (c0 = 0x80000000|i, c1 = w, c2 = t,
 * c3 = 0x5100), t counting the handle's sweeps. */
int qmc2d_vmc_single(qmc2d_handle *h, int nsweep, double delta, int refresh);
/* The largest max_jm |sum_k W(j,k) D(k,m) - delta_jm| over the walkers of
 * the last qmc2d_vmc_single call, measured on the updated inverse just
 * before each recompute: the round-off drift of the Sherman-Morrison
 * updates between refreshes (0 when no recompute happened within the call). */
int qmc2d_single_drift(qmc2d_handle *h, double *max_err);

/* ------------------------------------------------- DMC across ranks
 * branch2 (reptation.f:2162-2273) over the walkers of several ranks, one
 * population (handle) per rank and GPU: each rank advances its walkers and
 * weights (qmc2d_dmc_weights), the weights are all-gathered by the caller
 * (MPI_ALLGATHER in the reference, :2185), every rank computes the same
 * plan (qmc2d_comb_plan), ships the records it sends (qmc2d_records_pack
 * into a device buffer, then the caller's send; the reference's
 * send/receive, :2275-2318) and places the ones it receives
 * (qmc2d_records_unpack), and finally copies walkers within the rank
 * (qmc2d_population_resample; prov_dest, :2320). With one rank this is the
 * comb of qmc2d_dmc. */
/* One DMC generation's moves and weights without the comb: mmstep moves of
 * every walker, the weight the product of min(mmult, exp(-npnorm (E_L -
 * etrial) delta)) over them (dmc, reptation.f:894-906); wate[nw] receives
 * the weights (host). */
int qmc2d_dmc_weights(qmc2d_handle *h, int mmstep, double delta, double etrial, double mmult,
                      int mage, double *wate);
/* The comb of nproc ranks of nconf walkers each, from the weights of all
 * ranks (wate_all[p * nconf + i], as all-gathered), for `rank`: the same on
 * every rank. Weights are capped at 10 (wmult, :2174); the comb's uniforms
 * are Philox u[0] of (c0 = tooth, c1 = 0xFFFFFFFF, c2 = gen, c3 = 1) keyed
 * by `seed`, which all ranks share (the reference's rannyu2 stream). Out:
 * sends (send_rank[k], send_slot[k]) and receives (recv_rank[k],
 * recv_slot[k]) in exchange order (each list has room for nconf entries),
 * then src[nconf]: after the exchange, new slot j copies slot src[j].
 * ncapped: this rank's weights that were capped. Host only. */
int qmc2d_comb_plan(int nproc, int nconf, const double *wate_all, uint64_t seed, uint32_t gen,
                    int rank, int *src, int *nsend, int *send_rank, int *send_slot, int *nrecv,
                    int *recv_rank, int *recv_slot, int *ncapped);
/* Doubles of one walker record: x (2N), g (2N), h (ntypes), props
 * (n_props), sign, age. */
int qmc2d_record_len(qmc2d_handle *h, int *len);
/* Records of the n slots[] (host) of the current population to or from
 * rows of buf_dev (device, n * record_len doubles); synchronous on
 * `stream` (NULL: the handle's stream). */
int qmc2d_records_pack(qmc2d_handle *h, int n, const int *slots, double *buf_dev, void *stream);
int qmc2d_records_unpack(qmc2d_handle *h, int n, const int *slots, const double *buf_dev,
                         void *stream);
/* new[j] = old[src[j]] for every walker slot (src host, nw entries); the
 * comb's generation counter advances as qmc2d_dmc's does. */
int qmc2d_population_resample(qmc2d_handle *h, const int *src);

/* ------------------------------------------------------------- reptation */
typedef struct qmc2d_rmc_params {
  int ntau, ntauskip, mdelta;
  double delta, etrial;
  int mage, mage_r;
} qmc2d_rmc_params;

/* read_path (reptation.f:1775): set up one reptile per slot from
 * nrep*ntau configurations (reptile-major, bead order); nrep is at most the
 * handle's capacity. For systems whose determinants live in device memory
 * (qmc2d_create) each reptile uses one walker slot's determinant block. */
int qmc2d_rmc_init(qmc2d_handle *h, int nrep, const qmc2d_rmc_params *prm,
                   const double *x);
/* nstp reptation moves (reptation_move + reptation_metropolis_test,
 * reptation.f:1897-1895) on every reptile, accumulating p_old into the
 * block sums. */
int qmc2d_rmc(qmc2d_handle *h, int nstp);
/* Launch choice of qmc2d_rmc (the reference has no counterpart): split = 1
 * (the default) runs each bead growth as two kernels, the pair passes with
 * the pair rows staged in shared memory and then the rest of the evaluation
 * and the tests, as a VMC/DMC move; split = 0 runs whole moves in one
 * kernel per launch. Both compute the same values up to round-off. */
int qmc2d_rmc_set_launch(qmc2d_handle *h, int split);
/* Copy reptile r's path (ntau beads, x then props) out. */
int qmc2d_rmc_get_path(qmc2d_handle *h, int r, double *x, double *props);
/* Reptation restart: see the restart(0) comment above qmc2d_vmc. */
int qmc2d_restart_read_rmc(qmc2d_handle *h, const qmc2d_system *sys, qmc2d_stats *st,
                           const qmc2d_rmc_params *prm, const char *dir, const char *runid,
                           int rank, int *iblk);

/* ------------------------------------------------ reptation path estimators
 * The imaginary-time estimators of path_props (reptation.f:1578-1737):
 * - mstar: per type, the mean over particles and bead pairs of
 *   |x(itau) - x(jtau)|^2 against the lag jtau - itau (in steps of the
 *   record's tau skip), beads ntauskip+1 .. ntau-ntauskip;
 * - cmass: per type, cos and sin of 2 pi np x_cm / L of the middle bead's
 *   centre of mass (z), and the mean of |x_cm(itau) - x_cm(jtau)|^2
 *   against the lag for each of the record's bead skips (diffusion);
 * - itc: imaginary-time correlations sum_i a(itau) b(jtau) of stored bead
 *   properties a, b (each a sum of named properties; complex pairs of
 *   rhok entries when flagged 'complex', conjugated for 'conjg').
 * The reference sets them up from the deck's records when rmc starts
 * (cmass_setup, mstar_setup, itc_setup; reptation.f:1378-1553) and appends
 * them to the path properties in that order: cmass z, cmass diffusion,
 * mstar, itc. Here they form their own vector in the same order. */
#define QMC2D_MAX_ADD 4           /* properties summed in one itc factor */
#define QMC2D_MAX_CMSKIP 8        /* bead skips of one cmass record */
typedef struct qmc2d_rmc_estimators {
  int ntau, ntauskip;
  int nmstar;
  int mstar_type[QMC2D_MAX_EST], mstar_tau_skip[QMC2D_MAX_EST];
  int ncmass;
  int cmass_type[QMC2D_MAX_EST], cmass_tau_skip[QMC2D_MAX_EST];
  int cmass_nskip;                                   /* bead skips (one count for all records) */
  int cmass_ntauskip[QMC2D_MAX_EST][QMC2D_MAX_CMSKIP];
  int nitc;
  int itc_add[QMC2D_MAX_EST], itc_start[QMC2D_MAX_EST][QMC2D_MAX_ADD];
  int itc_count[QMC2D_MAX_EST], itc_complex[QMC2D_MAX_EST];  /* 0, 1 complex, -1 conjg */
  int jtc_add[QMC2D_MAX_EST], jtc_start[QMC2D_MAX_EST][QMC2D_MAX_ADD];
  int jtc_complex[QMC2D_MAX_EST], itc_tau_skip[QMC2D_MAX_EST];
  int jcmass_z, jcmass_d, jmstar, jitc, nvalues;     /* offsets in the estimator vector */
} qmc2d_rmc_estimators;
/* mstar_setup, cmass_setup and itc_setup on the system's records for paths
 * of ntau beads with ntauskip skipped at each end (itc names: the scalar
 * properties and rhok_<type>). */
int qmc2d_rmc_estimators_setup(const qmc2d_system *sys, int ntau, int ntauskip,
                               qmc2d_rmc_estimators *est);
/* The estimators of every reptile's current path (after qmc2d_rmc_init or
 * qmc2d_rmc), averaged over the reptiles, into out[est->nvalues]. The
 * reference evaluates them in path_props on each proposed path and
 * accumulates the accepted path's values once per step; calling this once
 * per step after qmc2d_rmc(h, 1) gives the same per-step values (the
 * reference refreshes the itc entries only every 100th path_props call). */
int qmc2d_rmc_path_estimators(qmc2d_handle *h, const qmc2d_rmc_estimators *est, double *out);
/* The estimator files of averages(3) (reptation.f:4377-4428, each in the
 * format of write_nonscalar_props, :4582-4616) from a qmc2d_stats over the
 * estimator vector (n_props = est->nvalues) and the block just added:
 * <runid>.mstar_<type>, <runid>.cmass_<type> and the itc files (named as
 * itc_setup names them) rewritten each block, <runid>.z_cmass_<type> with
 * every block's lines after the previous ones. */
int qmc2d_stats_write_estimators(const qmc2d_stats *st, const qmc2d_system *sys,
                                 const qmc2d_rmc_estimators *est, const double *blk,
                                 double blk_norm, const char *dir, const char *runid);

/* ----------------------------------------------------- streams and timing
 * The reference has no timers; these expose device time per kernel. */
enum qmc2d_kernel {
  QMC2D_KERNEL_MOVE = 0,    /* evaluation after the pair passes + accept (VMC/DMC) */
  QMC2D_KERNEL_BRANCH = 1,  /* branch2 comb */
  QMC2D_KERNEL_GATHER = 2,  /* walker slot copies after branching */
  QMC2D_KERNEL_EVAL = 3,    /* batched compute_properties */
  QMC2D_KERNEL_RMC = 4,     /* reptation moves */
  QMC2D_KERNEL_PAIRS = 5,   /* proposal + pair passes of a VMC/DMC move */
  QMC2D_KERNEL_SINGLE = 6,  /* single-electron VMC sweeps (qmc2d_vmc_single) */
  QMC2D_KERNEL_ORB_INV = 7, /* orbitals and their inversion of a move (orb_inv_kernel) */
  QMC2D_NKERNELS = 8
};
/* The handle's CUDA stream (a cudaStream_t) so callers can order work and
 * events after the library's launches. */
int qmc2d_stream(qmc2d_handle *h, void **stream);
/* enable = 1 starts recording a CUDA event pair around every launch on the
 * handle's stream (and clears the totals); 0 stops. */
int qmc2d_profile(qmc2d_handle *h, int enable);
/* Total device milliseconds and launch count of one kernel since enable. */
int qmc2d_profile_get(qmc2d_handle *h, int kernel, double *ms, long *launches);
/* Phase timers inside the walker kernels: with enable = 1 every CTA adds
 * the SM clock cycles its thread 0 spends in each phase of a move
 * (proposal, pair sums, rho_k, u3, orbitals, inversion, F matrices, drift,
 * cross-term matrix, cross term, assembly, accept) to 16 counters; with
 * enable = 0 the counters are copied to cycles[16] and the timers stop. */
int qmc2d_phase_timers(qmc2d_handle *h, int enable, unsigned long long *cycles);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* QMC2D_H */
