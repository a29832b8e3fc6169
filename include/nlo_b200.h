/*
 * nlo_b200.h -- C ABI of the B200 (sm_100a) NLO BK right-hand side and evolution.
 *
 * Plain pointers and sizes only.  Every array argument marked "device" is a CUDA
 * device pointer owned by the caller; every call is asynchronous on the given
 * stream (a cudaStream_t passed as void*, NULL = legacy default stream) and
 * returns NLO_OK or an error code; nlo_last_error() describes the last failure
 * of the calling thread.  No entry point allocates device memory: kernels that
 * need scratch take a caller-provided workspace whose size the matching
 * *_workspace_bytes() function returns.
 *
 * Each entry point replaces one operator of the reference package
 * (HaowuDuan/nlo_bk_optimized, torch_nlo_clean/src/nlo_torch); the citation is
 * given beside it.  The reference binds its operators through pybind with torch
 * tensors on the current CUDA stream; these take the same data as raw buffers.
 */
#ifndef NLO_B200_H
#define NLO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NLO_OK 0
#define NLO_ERR_INVALID 1   /* argument rejected on the host; nothing launched */
#define NLO_ERR_CUDA 2      /* a CUDA runtime call failed */
#define NLO_ERR_WORKSPACE 3 /* workspace missing or too small */

#define NLO_PRECISION_MIXED 0 /* FP32 integrands, FP64 sums, spline refit and RK update */
#define NLO_PRECISION_FP64 1  /* everything in FP64 */

#define NLO_STEPPER_EULER 0 /* bk/evolution.py:110-122 */
#define NLO_STEPPER_RK3 1   /* Kutta RK3, bk/evolution.py:190-236 (_fixed_rk23_step) */
#define NLO_STEPPER_RK4 2   /* classical RK4 (no reference counterpart) */

/* BKConfig.Order (bk/config.py:36-63).  The zero value is the production order. */
#define NLO_ORDER_NLO_RESUM_DLOG_SLOG 0
#define NLO_ORDER_NLO_RESUM_DLOG 1
#define NLO_ORDER_NLO 2
#define NLO_ORDER_LO_RESUM_DLOG_SLOG 3
#define NLO_ORDER_LO_RESUM_DLOG 4
#define NLO_ORDER_LO 5

/* BKConfig.RC_LO, the form of Kernel_lo (bk_kernels/k1.py:37-94).  FIXED_LO is
 * NLO_RC_LO_BALITSKY with fixed_coupling = 1. */
#define NLO_RC_LO_BALITSKY 0
#define NLO_RC_LO_PARENT 1
#define NLO_RC_LO_SMALLEST 2
#define NLO_RC_LO_FAC 3
#define NLO_RC_LO_BEUF 4

/* BKConfig.RESUM_RC, the coupling of the resummation factors (bk_kernels/k1.py:100-107). */
#define NLO_RESUM_RC_SMALLEST 0
#define NLO_RESUM_RC_PARENT 1
#define NLO_RESUM_RC_FIXED 2

/* BKConfig.RC_NLO, the coupling of K2 and Kf (bk/derivatives.py:615-632).  FIXED_NLO is
 * fixed_coupling = 1. */
#define NLO_RC_NLO_SMALLEST 0
#define NLO_RC_NLO_PARENT 1

/* Physics and numerical switches of BKConfig (bk/config.py:66-124) that the
 * right-hand side depends on.  A zero-initialised tail (order, rc_lo, resum_rc, rc_nlo)
 * selects the production choices.  The coupling is bk_alpha_s (coupling.py:10-46): the
 * smooth freeze for NF <= 3, the heavy-flavour thresholds for NF = 5, a constant when
 * fixed_coupling is set (RC_LO = FIXED_LO or RC_NLO = FIXED_NLO).  Orders without NLO
 * kernels (NLO_ORDER_LO*) skip K2 + Kf. */
typedef struct nlo_bk_params {
    double nc;            /* NC */
    double nf;            /* NF: 0, 3 or 5 */
    double lambda_qcd;    /* LambdaQCD */
    double c2;            /* C2 */
    double minr;          /* MINR (double-log resummation switch r > 1.01 MINR, k1.py:117) */
    double ksub;          /* KSUB */
    double fixed_alpha_s; /* FIXED_AS: the fixed coupling, and the RESUM_RC_FIXED coupling */
    double alpha_cap;     /* > 0: alpha_s = min(alpha_s, alpha_cap) (frozen-coupling variant) */
    int32_t symmetrize;   /* SYMMETRIZE_Z_Z2_INTEGRATION */
    int32_t fixed_coupling;
    int32_t force_positive; /* FORCE_POSITIVE_N */
    int32_t precision;      /* NLO_PRECISION_* */
    int32_t order;          /* NLO_ORDER_* */
    int32_t rc_lo;          /* NLO_RC_LO_* */
    int32_t resum_rc;       /* NLO_RESUM_RC_* */
    int32_t rc_nlo;         /* NLO_RC_NLO_* */
    int32_t kinematical_constraint; /* KINEMATICAL_CONSTRAINT: K1 reads the amplitude history;
                                       only nlo_bk_rhs_history / nlo_bk_evolve_history accept it */
} nlo_bk_params;

/* Scrambled Sobol direction numbers of torch.quasirandom.SobolEngine
 * (sobolstate[d][30] and shift[d]; values < 2^30). */
typedef struct nlo_sobol_dirs {
    int32_t dims; /* <= 8 */
    uint32_t state[8][30];
    uint32_t shift[8];
} nlo_sobol_dirs;

/* The K2+Kf integration box in (log z, log z', theta_z, theta_z'):
 * lower + width * u for u in the unit cube (bk/derivatives.py:424-431). */
typedef struct nlo_bk_box {
    double lower[4];
    double width[4];
} nlo_bk_box;

const char* nlo_last_error(void);
int nlo_abi_version(void);

/* Scrambled Sobol points u[n][dims] of indices offset .. offset+n-1, bit-exact to
 * SobolEngine(dims, scramble=True, seed).draw(...) in float32 (precision 0) or
 * float64 (precision 1).  Replaces the host-side draw and host-to-device copy of
 * dis/fixed_sobol.py:87-92 and the Philox draws of custom_kernels/integration.cu:60-93.
 * out: device float[n*dims] or double[n*dims]. */
int nlo_sobol_draw(const nlo_sobol_dirs* dirs, int64_t offset, int64_t n, int32_t precision, void* out,
                   void* stream);

/* Spline buffer size in doubles for a grid of `points` knots:
 * x[points] (log r) followed by the log N and log S coefficient blocks,
 * each [points-1][4] (a, b, c, d), then 2*points doubles of scratch for the
 * tridiagonal factorisation. */
size_t nlo_bk_spline_doubles(int32_t points);

/* Natural-cubic log N and log S splines of an amplitude row (FP64).
 * Replaces evolution_loglog_splines_mixed (custom_kernels/interpolation.cu:374-450)
 * and LogLogSpline (numerics/interpolation.py:95-121, bk/evolution.py:536-560).
 * r, N: device double[points]; spline: device double[nlo_bk_spline_doubles(points)]. */
int nlo_bk_splines(const double* r, const double* N, int32_t points, int32_t force_positive, double* spline,
                   void* stream);

/* Active parents (index > 0 and N <= 0.99999; bk/evolution.py:501) as a list:
 * active: device int32[points] (slot -> grid index), count: device int32[1]. */
int nlo_bk_active(const double* N, int32_t points, int32_t* active, int32_t* count, void* stream);

/* K1 for every active parent by the fixed rule of 8 Gauss-Legendre nodes in
 * log z per grid interval times 24 nodes in v with theta = pi v^2
 * (custom_kernels/bk/k1/kernel.cu:2040-2092, integrand bk/derivatives.py:434-468).
 * Replaces mixed_fixed_grid_integrals (custom_kernels/bk/k1/kernel.cu:2321-2418).
 * out: device double[points]; entries of inactive parents are set to 0. */
int nlo_bk_k1(const nlo_bk_params* params, const double* r, int32_t points, const double* spline,
              const int32_t* active, const int32_t* count, double* out, void* stream);

/* Workspace bytes for nlo_bk_k2kf with `points` grid points. */
size_t nlo_bk_k2kf_workspace_bytes(int32_t points);

/* K2+Kf sums over `samples` scrambled Sobol points (indices offset ..) for every
 * active parent: out[i][0] = sum w K2, out[i][1] = sum w Kf, out[i][2] = sum w^2 (K2+Kf)^2,
 * with w the box volume (bk/derivatives.py:322-335, 490-612).  Replaces
 * bk_nlo_mixed_vegas_summaries (custom_kernels/bk/k2_kf/kernel.cu:877-1063).
 * out: device double[points*3]; inactive parents get zeros. */
int nlo_bk_k2kf(const nlo_bk_params* params, const double* r, int32_t points, const double* spline,
                const int32_t* active, const int32_t* count, const nlo_sobol_dirs* dirs, int64_t offset,
                int64_t samples, const nlo_bk_box* box, double* out, void* workspace, size_t workspace_bytes,
                void* stream);

/* The same K2+Kf sums as nlo_bk_k2kf for callers that cannot allocate device
 * memory (a plugin inside a framework that owns the GPU's memory pool, a serving
 * loop that must not pay cudaMalloc's latency and synchronisation): there is no
 * workspace argument and nothing is allocated; the per-CTA partial sums live in a
 * fixed device array of 296 x 512 x 3 doubles (3.6 MB) that every GPU loading the
 * library holds until the process exits.  points must be <= 512 (larger grids are
 * rejected with NLO_ERR_INVALID), and the parameters and direction numbers are
 * checked as nlo_bk_k2kf checks them.  The first call on a device looks up the
 * array's address with that device current; make it before any stream capture.
 * The address is cached for the device's context: do not use the library across a
 * cudaDeviceReset.
 * All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  This entry point has no counterpart in the reference. */
int nlo_bk_k2kf_static(const nlo_bk_params* params, const double* r, int32_t points, const double* spline,
                       const int32_t* active, const int32_t* count, const nlo_sobol_dirs* dirs, int64_t offset,
                       int64_t samples, const nlo_bk_box* box, double* out, void* stream);

/* Tabulated initial condition (ICDataFile, bk/initial_conditions.py:38-91) on the device.
 * nlo_ic_spline fits the natural cubic spline through n >= 3 rows (r: device double[n],
 * strictly increasing; N: device double[n]) into spline: device double[nlo_ic_spline_doubles(n)],
 * with the reference's FP64 operations (NaturalCubicSpline, numerics/interpolation.py:13-48,
 * 124-149), so the coefficients equal the reference's.  nlo_ic_evaluate is
 * ICDataFile.dipole_amplitude (:86-90) at m points: 0 below the first r, 1 above the last. */
size_t nlo_ic_spline_doubles(int32_t n);
int nlo_ic_spline(const double* r, const double* N, int32_t n, double* spline, void* stream);
int nlo_ic_evaluate(const double* spline, int32_t n, const double* r, int64_t m, double* out, void* stream);

/* Workspace bytes for nlo_bk_rhs / nlo_bk_evolve. */
size_t nlo_bk_rhs_workspace_bytes(int32_t points);

/* dN/dY = K1 + (K2+Kf) at active parents, 0 elsewhere, non-finite -> 0
 * (_evolve_derivative, bk/evolution.py:329-351 with _derivative_components :354-488).
 * N, dndy: device double[points]; k1, k2kf: optional device double[points] (may be NULL). */
int nlo_bk_rhs(const nlo_bk_params* params, const double* r, const double* N, int32_t points,
               const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box, double* dndy, double* k1,
               double* k2kf, void* workspace, size_t workspace_bytes, void* stream);

/* One shard's part of the right-hand side of nlo_bk_rhs, for evolutions sharded over several
 * GPUs: K1 of the active parents i with i % shards == shard, plus K2+Kf of every active parent
 * summed over this shard's Sobol indices [shard*samples/shards, (shard+1)*samples/shards) and
 * divided by the total `samples`.  The shards' dndy rows add up to nlo_bk_rhs's (to FP64
 * summation order), so the ranks sum them with one all-reduce per stage; every lane of the
 * K2+Kf kernel stays busy on every rank (no counterpart in the reference, which runs on one
 * GPU). */
int nlo_bk_rhs_shard(const nlo_bk_params* params, const double* r, const double* N, int32_t points, int32_t shard,
                     int32_t shards, const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box, double* dndy,
                     void* workspace, size_t workspace_bytes, void* stream);

/* One stepper stage: out = N + sum_j coef[j] k[j] (nk <= 4; k: host array of device
 * pointers, coef: host array), clamped to [0, 1] when clamp != 0; status (optional device
 * uint32[1]) gets bit 0 when a value is not finite.  The stage combinations of
 * nlo_bk_evolve, for callers that drive the stepper themselves (bk/evolution.py:110-236). */
int nlo_bk_stage(const double* N, const double* const* k, const double* coef, int32_t nk, int32_t points,
                 int32_t clamp, double* out, uint32_t* status, void* stream);

/* Rapidity evolution of one amplitude row through `steps` steps of size `step`
 * (_bk_steps, bk/evolution.py:85-159): each step applies the stepper, clamps N to
 * [0,1] when force_positive, and stores the row.  table: device double[(steps+1)*points]
 * with row 0 = the initial condition (input).  status: device uint32[1], bit 0 set if
 * a non-finite amplitude appeared (the host raises FloatingPointError).  On grids of more
 * than 192 points the steps after the first replay a CUDA graph of one step, recorded on a
 * private stream during the call (the rows are the same as launching every step). */
int nlo_bk_evolve(const nlo_bk_params* params, const double* r, int32_t points, int32_t steps, double step,
                  int32_t stepper, const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box,
                  double* table, uint32_t* status, void* workspace, size_t workspace_bytes, void* stream);

/* nlo_bk_rhs with the amplitude history that the kinematical constraint reads
 * (bk/derivatives.py:469-487, 712-758; _derivative_components, bk/evolution.py:354-488):
 * hist_N: device double[rows*points], rows >= 1, the last row the amplitude whose
 * derivative is taken; hist_y: device double[rows], increasing, the last value the current
 * rapidity.  Where min(X, Y) > r, K1 takes the daughters at the rapidity shifted by
 * log(min(X^2, Y^2)/r^2), interpolated from the history (6-point natural splines in r,
 * linear in y); where the shift is negative it contributes nothing.  Without
 * params->kinematical_constraint the history beyond the last row is not read. */
int nlo_bk_rhs_history(const nlo_bk_params* params, const double* r, int32_t points, const double* hist_y,
                       const double* hist_N, int32_t rows, const nlo_sobol_dirs* dirs, int64_t samples,
                       const nlo_bk_box* box, double* dndy, double* k1, double* k2kf, void* workspace,
                       size_t workspace_bytes, void* stream);

/* nlo_bk_evolve continued from a stored history (the loop of _bk_steps, bk/evolution.py:85-159,
 * over a table that already holds rows 0..first): table: device double[(first+steps+1)*points],
 * rows 0..first input (row `first` the current amplitude); y: device double[first+steps+1], the
 * rapidities of all rows (y[k] = y[k-1] + step as the caller accumulates them).  Computes rows
 * first+1..first+steps.  With params->kinematical_constraint each step reads the rows before
 * it, and the stepper must be NLO_STEPPER_EULER (BKConfig requires EULER_METHOD). */
int nlo_bk_evolve_history(const nlo_bk_params* params, const double* r, int32_t points, const double* y,
                          int32_t first, int32_t steps, double step, int32_t stepper, const nlo_sobol_dirs* dirs,
                          int64_t samples, const nlo_bk_box* box, double* table, uint32_t* status, void* workspace,
                          size_t workspace_bytes, void* stream);

/* ------------------------------------------------------- many parameter sets at once
 * nlo_bk_evolve for `sets` initial rows (1..256) on one r grid with one parameter block and
 * per-set budgets and Sobol seeds: every stage runs one launch per kernel for all sets, and
 * one K2+Kf launch takes lanes over (set, parent) pairs -- each CTA stages one tile of sample
 * records per set it holds and its lanes sweep their own set's tile (sets of equal budget
 * share CTAs, so the launch has no idle tail per set).  Set i's result equals nlo_bk_evolve's
 * for that row, budget and seed up to the order of the FP64 sums of the CTA partials (no
 * counterpart in the reference, which evolves one condition per call; the batched solve of
 * many initial conditions with uneven budgets, and the request loop's step-level batching).
 * tables: host array of `sets` device pointers, each a double[(steps+1)*points] table whose
 * row 0 holds the set's initial row.  dirs: host array of `sets` Sobol direction sets (at
 * least 4 dimensions each).  samples: host int64[sets], each 0..2^30.  waves (1..64): K2+Kf
 * CTAs per launch ~ waves x 2 x SM count, spread over the sets' groups.  status: device
 * uint32[sets], reset and then flagged per set as in nlo_bk_evolve.  The kinematical
 * constraint is not accepted. */
size_t nlo_bk_sets_workspace_bytes(int32_t points, int32_t sets, int32_t waves);
int nlo_bk_evolve_sets(const nlo_bk_params* params, const double* r, int32_t points, int32_t sets,
                       double* const* tables, int32_t steps, double step, int32_t stepper,
                       const nlo_sobol_dirs* dirs, const int64_t* samples, const nlo_bk_box* box, int32_t waves,
                       uint32_t* status, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ K2+Kf by Vegas
 * The reference's default integrator of the NLO part (BKConfig.INTMETHOD_NLO = VEGAS;
 * rapidity_derivative_nlo, bk/derivatives.py:389-421, driving vegas(),
 * numerics/integration.py:120-589): one Vegas integral per active parent over the box of
 * nlo_bk_box, on scrambled Sobol points of `dirs` (indices 0, 1, ... across the rounds of one
 * right-hand side, the warm-up first).  Each parent's grid lives in the caller's `state` and,
 * with reuse_grid, carries over to the next right-hand side with a shortened warm-up (the
 * per-parent vegas_states of bk/evolution.py:85-100, 354-424).  Defaults in brackets are
 * the reference's. */
typedef struct nlo_bk_vegas_options {
    int64_t samples_per_iteration; /* [MCINTPOINTS] >= 2 */
    int64_t warmup_samples;        /* [max(2, MCINTPOINTS / 5)] 0 or >= 2: an adaptation-only round first */
    int32_t max_iterations;        /* [4] */
    int32_t min_iterations;        /* [2] 1 <= min <= max */
    int32_t bins;                  /* [32] bins per dimension, 2..256 */
    int32_t reuse_grid;            /* [1] VEGAS_REUSE_GRID: keep each parent's grid for the next right-hand side */
    double reuse_warmup_fraction;  /* [0.25] VEGAS_REUSE_WARMUP_FRACTION: warm-up of a kept grid =
                                      max(2, warmup_samples x fraction), none when either is 0 */
    double epsrel;                 /* [0.2] converged after min_iterations once error <= max(epsabs, epsrel |value|) */
    double epsabs;                 /* [0] */
    int32_t replicas;              /* [6 in the reference's CUDA evolution with kept grids and a seed, else 0]
                                      replica refinement (bk/evolution.py:411-456): a parent with
                                      (|K1| + |K2| + |Kf|) / max(|K1 + K2 + Kf|, 0.05 (|K1| + |K2| + |Kf|)) >= 4
                                      or N > 0.9 gets `replicas` more integrals on fresh grids, Sobol points
                                      of dirs[1..replicas] (the reference's seeds seed + 1000 k), and takes
                                      the mean; 0..16 */
} nlo_bk_vegas_options;

/* Per-parent Vegas state in doubles for a grid of `points` parents: per parent the grid
 * edges [4][bins+1] and 16 scalars.  A zero-filled state holds no grid yet (each parent then
 * starts from the uniform grid with the full warm-up). */
size_t nlo_bk_vegas_state_doubles(int32_t points, int32_t bins);

/* Workspace bytes of nlo_bk_rhs_vegas / nlo_bk_evolve_vegas (at least nlo_bk_rhs_workspace_bytes). */
size_t nlo_bk_vegas_workspace_bytes(int32_t points, const nlo_bk_vegas_options* options);

/* The right-hand side of nlo_bk_rhs_history with K2+Kf by Vegas for the active parents
 * i with i % shards == shard (shard = 0, shards = 1: all of them; K1 takes the same parents,
 * so the shards' rows add up to the whole right-hand side).  hist_y may be NULL without the
 * kinematical constraint; hist_N's last row is the amplitude.  state: device
 * double[nlo_bk_vegas_state_doubles(points, bins)], read and updated.  k2kf (optional)
 * receives the Vegas value of each parent (the combined estimate of its iterations, or the
 * replica mean of a refined parent).  dirs: host array of 1 + options->replicas direction
 * sets, dirs[0] the main integrals', dirs[k] replica k's. */
int nlo_bk_rhs_vegas(const nlo_bk_params* params, const double* r, int32_t points, const double* hist_y,
                     const double* hist_N, int32_t rows, int32_t shard, int32_t shards,
                     const nlo_bk_vegas_options* options, const nlo_sobol_dirs* dirs, const nlo_bk_box* box,
                     double* state, double* dndy, double* k1, double* k2kf, void* workspace, size_t workspace_bytes,
                     void* stream);

/* nlo_bk_evolve_history with K2+Kf by Vegas (the reference's production evolution: the
 * parents' grids carried through every right-hand side of the evolution when
 * options->reuse_grid is set).  y may be NULL without the kinematical constraint. */
int nlo_bk_evolve_vegas(const nlo_bk_params* params, const double* r, int32_t points, const double* y,
                        int32_t first, int32_t steps, double step, int32_t stepper,
                        const nlo_bk_vegas_options* options, const nlo_sobol_dirs* dirs, const nlo_bk_box* box,
                        double* state, double* table, uint32_t* status, void* workspace, size_t workspace_bytes,
                        void* stream);

/* --------------------------------------------------- Vegas for a caller's integrand
 * The vegas() integrator (numerics/integration.py:120-589) for any integrand the caller
 * evaluates itself (the reference integrates arbitrary torch functions with it).  The library
 * does the sampling and the bookkeeping on the device; per round (the warm-up, then each
 * iteration): nlo_vegas_sample for a batch of Sobol points, the caller's f at the batch's box
 * points, nlo_vegas_accumulate; after the round's last batch nlo_vegas_end_round re-bins the
 * grid (:804-866) and, for an iteration, updates the inverse-variance-weighted value, error and
 * convergence flag (:510-582).  The state holds the grid edges [dims][bins+1] (the unit cube)
 * and then value, error, n_eval, iterations and converged at NLO_VEGAS_VALUE.. after them. */
size_t nlo_vegas_state_doubles(int32_t dims, int32_t bins);     /* dims 1..8, bins 2..256 */
size_t nlo_vegas_workspace_bytes(int32_t dims, int32_t bins);
/* Clear the sums; a uniform grid unless keep_edges (the edges already in `state`, a kept VegasState). */
int nlo_vegas_begin(int32_t dims, int32_t bins, int32_t keep_edges, double* state, void* workspace,
                    size_t workspace_bytes, void* stream);
/* Points offset..offset+n-1 of the scrambled Sobol sequence `dirs` mapped through the grid:
 * x[n][dims] = lower + width * grid(u), factor[n] = prod(width) * prod(bins * bin width), bin[n][dims].
 * lower, width: host double[dims]; x, factor, bin: device. */
int nlo_vegas_sample(const nlo_sobol_dirs* dirs, int64_t offset, int64_t n, int32_t dims, int32_t bins,
                     const double* state, const double* lower, const double* width, double* x, double* factor,
                     int32_t* bin, void* stream);
/* Add the weights w = f * factor of a batch (f: device double[n], the integrand at the batch's
 * points) to the round's sums and |w| histograms, in a fixed order. */
int nlo_vegas_accumulate(const double* f, const double* factor, const int32_t* bin, int64_t n, int32_t dims,
                         int32_t bins, void* workspace, size_t workspace_bytes, void* stream);
/* Close a round of `samples` points: re-bin the grid; unless warmup, fold the round's estimate
 * into the combination and set converged once iterations >= min_iterations and
 * error <= max(epsabs, epsrel |value|). */
int nlo_vegas_end_round(int32_t dims, int32_t bins, double* state, int64_t samples, int32_t warmup,
                        int32_t min_iterations, double epsrel, double epsabs, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ======================================================================== NLO DIS
 * The NLO DIS cross-section integrands (dis/observables.py, dis/lo.py, dis/transverse.py,
 * dis/longitudinal.py) with the GBW or BK-table dipole, their tensor Gauss-Legendre rule and
 * the device Vegas integrator.  One "job" is one integral: a (Q^2, x_Bj) point, a quark, a
 * polarisation and one term. */

/* Integrand terms (the `contribution` strings of dis/observables.py:107-331). */
#define NLO_DIS_TERM_LO 0   /* LO |Psi|^2 N 2 pi r maxr over (z, r/maxr), all LO quarks; dis/observables.py:352-359 */
#define NLO_DIS_TERM_DIP0 1 /* T0 / Omega_L_const, 2D; dis/observables.py:107-172 */
#define NLO_DIS_TERM_DIP1 2 /* T1 / ab, 3D */
#define NLO_DIS_TERM_DIP2 3 /* T2 / cd, 4D */
#define NLO_DIS_TERM_I1 4   /* qqbar-g I1, 5D; dis/observables.py:175-250 */
#define NLO_DIS_TERM_I2 5   /* qqbar-g I2 with y_t explicit, 6D */
#define NLO_DIS_TERM_I3 6   /* qqbar-g I3 with y_t1, y_t2 explicit, 7D */
#define NLO_DIS_TERM_I2_NESTED 7 /* I2 with the inner rule, 5D; dis/observables.py:253-331 */
#define NLO_DIS_TERM_I3_NESTED 8 /* I3 with the inner rule, 5D */

#define NLO_DIPOLE_GBW 0   /* dipole/amplitude.py:23-45 */
#define NLO_DIPOLE_TABLE 1 /* BKDipole, dipole/amplitude.py:48-252 */

#define NLO_DIS_MAX_QUARKS 8

/* Physics of one job: DISConfig (dis/config.py:103-145), the kinematic point and the quark. */
typedef struct nlo_dis_kinematics {
    double Q2;
    double xbj;
    double mf;                  /* quark mass of the dipole and qqbar-g terms */
    int32_t n_quarks;           /* LO term: sum over these quarks */
    double lo_mass[NLO_DIS_MAX_QUARKS];
    double lo_charge2[NLO_DIS_MAX_QUARKS];
    double maxr;                /* DISConfig.maxr */
    int32_t transverse;         /* 1: Polarization.T, 0: Polarization.L */
    int32_t finite_nc;          /* NcScheme.FiniteNC */
    int32_t parent_coupling;    /* RunningCouplingScheme.PARENT (else SMALLEST) */
    int32_t smooth_coupling;    /* RunningCouplingIRScheme.SMOOTH (else FREEZE) */
    int32_t mass_dependent_x;   /* HeavyQuarkX.MassDependentX */
    double c2_alpha;            /* DISConfig.C2_alpha */
    double active_flavors;      /* DISConfig.active_flavors */
    double max_alpha;           /* DISConfig.max_alpha_s_freeze */
} nlo_dis_kinematics;

/* The dipole amplitude: GBW parameters, or a BK table prepared by nlo_dis_table_prepare. */
typedef struct nlo_dipole {
    int32_t kind;               /* NLO_DIPOLE_* */
    double qs0sqr, lambda, gamma, x0;  /* GBW(Qs0sqr, lambda_, gamma, x0) */
    const double* table;        /* NLO_DIPOLE_TABLE: device buffer of nlo_dis_table_doubles(nr, ny) */
    int32_t nr, ny;
} nlo_dipole;

/* Size in doubles of a prepared BK table with nr r points and ny rapidities. */
size_t nlo_dis_table_doubles(int32_t nr, int32_t ny);

/* Prepare a BK table for the device amplitude (BKDipole.__init__, dipole/amplitude.py:48-83):
 * r: device double[nr] (increasing, nr >= 9; BKDipole requires the reference's logarithmic
 * spacing, the device lookup itself takes any increasing grid), y: device double[ny] (increasing),
 * N: device double[ny*nr] (row y), x0: DipoleTable.x0; table: device double[nlo_dis_table_doubles].
 * The rapidities are stored as y + max(0, ln(1/x0)) like BKDipole.Y. */
int nlo_dis_table_prepare(const double* r, const double* y, const double* N, int32_t nr, int32_t ny, double x0,
                          double* table, void* stream);

/* The same with the reference's interpolation choice (AmplitudeInterpolation,
 * dipole/amplitude.py:15-17): NLO_INTERP_SPLINE_LINEAR (the default of BKDipole, what
 * nlo_dis_table_prepare selects) or NLO_INTERP_LINEAR_LINEAR (bilinear in r and Y,
 * dipole/amplitude.py:188-212; the reference's nlo-dis command line uses it). */
#define NLO_INTERP_SPLINE_LINEAR 0
#define NLO_INTERP_LINEAR_LINEAR 1
int nlo_dis_table_prepare_interpolated(const double* r, const double* y, const double* N, int32_t nr, int32_t ny,
                                       double x0, int32_t interpolation, double* table, void* stream);

/* BKDipole.initialize_interpolation(Y) (dipole/amplitude.py:105-133, 254-272): fit the global
 * spline at rapidity Y, which later evaluations at a matching Y use, and find maxr_interpolate.
 * The caller checks 0 <= Y <= max rapidity of the table (the reference raises ValueError). */
int nlo_dis_table_initialize(double* table, int32_t nr, int32_t ny, double Y, void* stream);

/* dipole_amplitude(r, Y) of GBW (dipole/amplitude.py:37-42) or BKDipole (:135-170) at n points:
 * r, Y, out: device double[n].  A BK table answers from its initialised global spline where Y
 * matches the initialisation rapidity, from the local splines elsewhere. */
int nlo_dis_dipole_amplitude(const nlo_dipole* dipole, const double* r, const double* Y, int64_t n, int32_t precision,
                             double* out, void* stream);

/* Evaluate one term at n unit-cube points (the reference's integrand_* functions and the
 * dis_lo_integrand / dis_dipole_integrand operators, custom_kernels/dis/lo_dipole/kernel.cu):
 * x: device double[n*dims(term)], out: device double[n].  inner_points: the inner rule of the
 * nested terms (8..128, 48 in the reference).  precision: NLO_PRECISION_*. */
int nlo_dis_integrand(const nlo_dis_kinematics* kin, int32_t term, const nlo_dipole* dipole, int32_t inner_points,
                      int32_t precision, const double* x, int64_t n, double* out, void* stream);

/* Tensor Gauss-Legendre integral of a 2D term (LO or DIP0) on the unit square for `jobs`
 * kinematic points at once: out[2*j] = value with `points` nodes per axis, out[2*j+1] =
 * |value - value with points/2 nodes| (numerics/integration.py:94-117,
 * custom_kernels/quadrature.py:38-55).  kin: host array [jobs]; out: device double[2*jobs]. */
int nlo_dis_gauss_legendre(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipole,
                           int32_t points, int32_t precision, double* out, void* workspace, size_t workspace_bytes,
                           void* stream);
size_t nlo_dis_gauss_legendre_workspace_bytes(int32_t jobs);
/* nlo_dis_gauss_legendre with a dipole per job (dipoles: host array [jobs]), so that one launch
 * serves kinematic points of different BK tables -- the requests of a batch or of the
 * serving loop (no counterpart in the reference, which evaluates one dipole at a time). */
int nlo_dis_gauss_legendre_dipoles(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term,
                                   const nlo_dipole* dipoles, int32_t points, int32_t precision, double* out,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* Vegas options (numerics/integration.py:120-138). */
typedef struct nlo_vegas_options {
    int32_t bins;               /* bins per dimension (<= 256) */
    int32_t max_iterations;
    int32_t min_iterations;
    int64_t samples_per_iteration;
    int64_t warmup_samples;     /* 0 or >= 2: one extra adaptation-only round first */
    double epsrel, epsabs;
    int32_t inner_points;       /* nested terms */
    int32_t precision;          /* NLO_PRECISION_* */
    int32_t keep_edges;         /* 1: start from the edges already in `state` (VegasState reuse) */
} nlo_vegas_options;

/* Per-job Vegas state in doubles: edges[dims][bins+1], then value, error, n_eval, iterations,
 * converged at offsets NLO_VEGAS_VALUE.. from the end of the edges. */
#define NLO_VEGAS_VALUE 2
#define NLO_VEGAS_ERROR 3
#define NLO_VEGAS_EVALS 4
#define NLO_VEGAS_ITERATIONS 5
#define NLO_VEGAS_CONVERGED 6
size_t nlo_dis_vegas_state_doubles(int32_t term, int32_t bins);
size_t nlo_dis_vegas_workspace_bytes(int32_t jobs, int32_t term, const nlo_vegas_options* options);

/* Vegas integration of one term for `jobs` kinematic points at once, all iterations on the
 * device without host synchronisation (vegas, numerics/integration.py:120-589, with the grid
 * re-binning of :804-866).  Samples are the scrambled Sobol points of dirs[j] (indices
 * 0, 1, ... across the rounds), split into a bin and a fraction per dimension.
 * kin, dirs: host arrays [jobs]; state: device double[jobs * nlo_dis_vegas_state_doubles]. */
int nlo_dis_vegas(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipole,
                  const nlo_vegas_options* options, const nlo_sobol_dirs* dirs, double* state, void* workspace,
                  size_t workspace_bytes, void* stream);

/* nlo_dis_vegas with a dipole per job (dipoles: host array [jobs]): the integrals of many
 * parameter sets or requests, each with its own BK table, in one sequence of launches (no
 * counterpart in the reference, which evaluates one dipole at a time).  Workspace and state
 * sizes are those of nlo_dis_vegas. */
int nlo_dis_vegas_dipoles(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipoles,
                          const nlo_vegas_options* options, const nlo_sobol_dirs* dirs, double* state,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Fixed-Sobol options (dis/fixed_sobol.py:30-37 defaults in brackets). */
typedef struct nlo_fixed_sobol_options {
    int64_t training_samples;      /* [65536] power of two */
    int32_t training_rounds;       /* [3] */
    int64_t samples_per_replicate; /* [32768] power of two */
    int32_t replicates;            /* [7] >= 2 */
    int32_t bins;                  /* [32] */
    int32_t fold_angle;            /* [1] fold the gluon angle onto [0, pi] */
    double i1_weight;              /* [1.0] weight of I1 in the grid-training score */
    int32_t inner_points;          /* [48] inner rule of I2 / I3 */
    int32_t precision;             /* NLO_PRECISION_* */
} nlo_fixed_sobol_options;

/* Grid buffer of nlo_dis_fixed_sobol in doubles: edges[5][bins+1] then 16 scalars. */
size_t nlo_dis_fixed_sobol_grid_doubles(int32_t bins);
size_t nlo_dis_fixed_sobol_workspace_bytes(const nlo_fixed_sobol_options* options);

/* The fixed-Sobol qqbar-g integration of one quark and polarisation (gbw_qg_fixed_sobol,
 * dis/fixed_sobol.py:273-368): training rounds learn one importance grid from the score
 * |I1|/<|I1|> + |I2|/<|I2|> + |I3|/<|I3|> over Sobol points split by the nearer dipole end
 * (custom_kernels/dis/sampling/kernel.cu:15-84; learn_triple_importance_grid :161-211),
 * then each replicate's means of I1, I2, I3 through the frozen grid
 * (integrate_triple_fixed_sobol :214-270).  dirs: host array [training_rounds + replicates]
 * of the direction numbers for seeds seed + r and seed + 10000 + j.  grid: device
 * double[nlo_dis_fixed_sobol_grid_doubles(bins)] (out); estimates: device
 * double[replicates][3] (out).  The caller forms the replicate mean and standard error.
 * The reference runs this path for GBW only; the device accepts a BK table as well. */
int nlo_dis_fixed_sobol(const nlo_dis_kinematics* kin, const nlo_dipole* dipole, const nlo_fixed_sobol_options* options,
                        const nlo_sobol_dirs* dirs, double* grid, double* estimates, void* workspace,
                        size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NLO_B200_H */
