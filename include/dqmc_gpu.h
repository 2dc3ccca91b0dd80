/*
 * dqmc_gpu.h -- C ABI of the B200 determinant-QMC engine (libdqmc_b200.so).
 *
 * The engine replaces the reference's sweep engine seam, the `Dqmc` API that
 * dqmc_run_replica consumes (SAI-QMC src/dqmc.h:91-108, used at
 * src/replica_run.c:124-126, 184-186, 284-453), with a batched engine: many
 * independent chains (replicas x temperatures, uneven n and L) advance
 * together on one GPU.  Plain pointers and sizes only; every matrix is
 * n x n column-major (the reference's layout, src/linalg.h:4).
 *
 * Return convention (as the reference's dqmc_init_modes, src/dqmc.c:418):
 * 0 = ok, nonzero = failure; dqmc_last_error() describes the last failure
 * of the calling thread.  A chain whose numerics break is frozen with a
 * nonzero status (src/dqmc.h:79-81 semantics: later sweeps are no-ops) and
 * the other chains continue.  Calls on one engine are not thread-safe.
 */
#ifndef DQMC_GPU_H
#define DQMC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DQMC_GPU_ABI_VERSION 1

typedef struct dqmc_engine dqmc_engine;

/* FP64: every product in FP64 (DMMA tensor cores).  MIXED: the wrap
 * (src/green.c:509-548) and the delayed-update flush (src/green.c:462-475)
 * as FP64-emulated int8 split products on the tcgen05 tensor cores (8
 * balanced base-256 digits per line, exact int32 accumulation); QR, G from
 * UDV, B-block products, ratios and sign stay FP64.  Chain status bit 16
 * (DQMC_ST_TIMEOUT) reports an abandoned split product. */
enum { DQMC_PREC_FP64 = 0, DQMC_PREC_MIXED = 1 };
/* Sweep order (DqmcSweepMode, src/dqmc.h:45-48): forward sweeps only, or
 * alternating forward / backward sweeps carrying the prefix and suffix UDV
 * stacks between them (src/dqmc.c:609-963). */
enum { DQMC_SWEEP_FORWARD = 0, DQMC_SWEEP_ALTERNATING = 1 };
/* G rebuild at a stabilization boundary (GreenRebuildMode, src/green.h):
 * COMBINE = one UDV from the two factors, then (1+UDT)^-1 (udv_combine +
 * udv_inv_one_plus_work, src/linalg.c:796-1115); TWO_SIDED = (1+LR)^-1 from
 * the two factors directly (udv_inv_one_plus_two_sided_work,
 * src/linalg.c:1117-1389).  CENTERED (the reference's recentred-D variant of
 * two-sided) is the same computation here: D is always held as log D. */
enum { DQMC_REBUILD_COMBINE = 0, DQMC_REBUILD_TWO_SIDED = 1, DQMC_REBUILD_CENTERED = 2 };
enum { DQMC_DRIFT_STAB = 1, DQMC_DRIFT_SCRATCH = 2 };
/* Delayed-update flush grouping: AUTO pairs site blocks when n >= 128 (the
 * G read-modify-write is bound by G traffic there), OFF flushes after every
 * block of k sites (src/green.c:462-475 with k sites), ON always pairs.
 * The proposals and their order are the same in all three. */
enum { DQMC_PAIRS_AUTO = 0, DQMC_PAIRS_OFF = 1, DQMC_PAIRS_ON = 2 };

/* UDV scale records (src/dqmc.c:100-378): where a factor was observed, as
 * the reference's direction strings, and the record layout returned by
 * dqmc_read_udv_records.  Per factor: min and max of log|D| over the finite
 * nonzero entries, and the counts of finite nonzero, zero and non-finite
 * entries (udv_scale_stats, src/dqmc.c:108-142). */
enum {
    DQMC_UDV_STACK_SUFFIX_PRE_RMUL = 0,  /* "stack_suffix_pre_rmul" (green.c:214) */
    DQMC_UDV_STACK_PREFIX_PRE_LMUL = 1,  /* "stack_prefix_pre_lmul" (green.c:238) */
    DQMC_UDV_FORWARD = 2,                /* "forward" boundary pair (dqmc.c:707)    */
    DQMC_UDV_BACKWARD = 3,               /* "backward" boundary pair (dqmc.c:831)   */
    DQMC_UDV_LEFT_FORWARD = 4,           /* "left_udv_forward" (dqmc.c:772)         */
    DQMC_UDV_LEFT_BACKWARD = 5           /* "left_udv_backward" (dqmc.c:926)        */
};
enum {
    DQMC_UDV_R_KIND = 0, DQMC_UDV_R_TAU, DQMC_UDV_R_BOUNDARY, DQMC_UDV_R_SWEEP,
    DQMC_UDV_R_LEFT = 4,    /* min, max, finite, zero, nonfinite of the (left) factor */
    DQMC_UDV_R_RIGHT = 9,   /* the same for the right factor of a boundary pair      */
    DQMC_UDV_R_HAS_RIGHT = 14,
    DQMC_UDV_R_SPIN = 15,   /* 0: G_up ("u"), 1: G_down ("d") of the two-spin path */
    DQMC_UDV_RECORD_DOUBLES = 16
};

/* Per-bin scalar layout returned by dqmc_read_bins (src/replica.h:6-16). */
enum {
    DQMC_BIN_SUM_SIGN_EHUB = 0,
    DQMC_BIN_SUM_SIGN_EGC,
    DQMC_BIN_SUM_SIGN_EPH,
    DQMC_BIN_SUM_SIGN_N,
    DQMC_BIN_SUM_SIGN_D,
    DQMC_BIN_SUM_SIGN,
    DQMC_BIN_COUNT_F,
    DQMC_BIN_ACCEPTED_F,
    DQMC_BIN_ATTEMPTS_F,
    DQMC_BIN_NFIELDS
};

typedef struct {
    int device;      /* CUDA device ordinal                                  */
    int precision;   /* DQMC_PREC_*                                          */
    int delay_rank;  /* delay rank k of the delayed update (0 = 32): site
                        blocks of k <= 32 sites; 32 < k <= 64 runs blocks
                        of ceil(k/2) sites with paired G updates (one rank
                        <= k update per k sites); k > 64 is rejected     */
    int drift;       /* bit-or of DQMC_DRIFT_*: STAB = max|G_wrap - G_stab|
                        at every stabilization (on by default); SCRATCH =
                        also the reference's rebuild-from-scratch drift
                        (src/dqmc.c:64-98, costly)                            */
    int ctas_per_sm; /* sweep kernel residency: 0 = auto (two chains per SM
                        when there are more chains than SMs), 1 or 2      */
    int sweep_order; /* DQMC_SWEEP_*                                        */
    int green_rebuild; /* DQMC_REBUILD_*                                    */
    int flush_pairs; /* DQMC_PAIRS_*: stage two consecutive site blocks and
                        update G once for both (rank <= 2k)               */
    int udv_diag;    /* 1: record the UDV scale statistics of every factor
                        the reference's udv_scale_file / udv_centered_file
                        diagnostics report (dqmc_read_udv_records); the
                        sweeps then run one launch per sweep             */
    int green_log;   /* > 0: keep up to this many snapshots per chain of G as
                        wrapped just before each stabilization point (the
                        matrix the reference's drift diagnostic compares,
                        src/dqmc.c:64-98), read with dqmc_read_green_log --
                        e.g. two engines run in lock step from the same
                        seeds give max|G_mixed - G_FP64| at every
                        stabilization.  No counterpart in the reference.   */
    int chain_ctas;  /* CTAs that advance one chain together as a thread-block
                        cluster, 2..16 (above 8 where the device allows a
                        non-portable cluster size); 1 = one CTA per chain;
                        0 = automatic: for batches of fewer chains than
                        SMs with a lattice of n >= 128, the largest
                        size at which all the batch's clusters are resident
                        at once, else 1.  Rank 0 runs the sweep; every rank
                        forms its share of the output tiles of the wrap,
                        the B-block products and the delayed-update G
                        update (FP64 or split products), so the trajectory
                        equals the one-CTA run bit for bit.  For batches of
                        fewer chains than SMs (one chain, a few large
                        lattices); one CTA per SM.  No counterpart in the
                        reference, whose sweep runs on one host thread.     */
    int cluster_chains; /* with chain_ctas > 1: how many of the most
                        expensive chains get a cluster each (0 = all); the
                        other chains run one per CTA inside clusters of the
                        same launch.  The automatic choice (chain_ctas = 0)
                        sets both from a cost model of the batch.          */
} dqmc_engine_desc;

typedef struct {
    unsigned long long attempts;   /* src/dqmc.h:84-86 counters */
    unsigned long long accepted;
    unsigned long long sweeps;
    int status;                    /* 0 healthy, else DQMC_ST_* bits */
    int pad;
    double sign;
    double drift_max, drift_mean;  /* max|G_wrapped - G_stabilized|  */
    unsigned long long drift_samples;
    double scratch_drift_max, scratch_drift_mean;  /* reference drift */
    unsigned long long scratch_drift_samples;
    int scratch_drift_max_tau;     /* tau and sweep of the maximum   */
    int pad2;
    unsigned long long scratch_drift_max_sweep;
    uint64_t rng[4];               /* xoshiro256** state (src/rng.h:6-8) */
} dqmc_chain_counters;

/* Fills a descriptor with the defaults (device 0, FP64, k by n, STAB drift). */
void dqmc_desc_default(dqmc_engine_desc *desc);

/* Creates an engine on desc->device.  Replaces the per-chain allocation of
 * dqmc_init_modes (src/dqmc.c:418-483) for a whole batch. */
dqmc_engine *dqmc_engine_create(const dqmc_engine_desc *desc);
void dqmc_engine_destroy(dqmc_engine *e);              /* src/dqmc.c:525-542 */
const char *dqmc_last_error(void);

/* Registers a Hubbard model on a lattice: hopping t (n x n), bipartite signs
 * (+/-1), U, dtau, mu = U/2.  expK = exp(-dtau (t - mu)) and its inverse are
 * computed on the host (model_init, src/model.c:8-31).  Lx, Ly give site
 * coordinates i = x + Lx*y for the spin structure factors (0 if none).
 * Returns the model id (>= 0) or -1. */
int dqmc_model_add(dqmc_engine *e, int n, int Lx, int Ly, const double *thop,
                   const int *bipart, double U, double dtau);
/* dqmc_model_add with a chemical potential (model_init, src/model.c:8-31):
 * half_filling = 1 sets mu = U/2 (mu ignored), else K = t - mu I.  Chains of
 * a model that is not particle-hole symmetric -- not at half filling, or
 * bipart NULL for a non-bipartite lattice -- evolve G_up and G_down
 * separately (the reference's use_ph = 0 path, src/dqmc.c:418-483,
 * 641-813): joint acceptance R = R_up R_down, a running sign reset to
 * det_up * det_down at every stabilization.  two_spin = 1 takes that path
 * also at the PH point (the reference's ph_symmetric = 0 override in
 * tests/test_dqmc_stack.c:81).  The two-spin path runs forward sweeps in
 * FP64, one chain per SM.  Returns the model id or -1. */
int dqmc_model_add_mu(dqmc_engine *e, int n, int Lx, int Ly, const double *t,
                      const int *bipart, double U, double dtau, int half_filling,
                      double mu, int two_spin);

/* Enables Szz(q) / Sperp(q) on a model for the q lists (mx, my), the
 * structure_factor_plan_init selectors of src/structure_factor.c:107-206.
 * nq = 0 disables a channel. */
int dqmc_model_set_spin(dqmc_engine *e, int model, int nq_zz, const int *mx_zz,
                        const int *my_zz, int nq_perp, const int *mx_perp,
                        const int *my_perp);

/* Adds a chain: L time slices, stabilization interval stab, seed of its
 * xoshiro256** stream.  field == NULL draws the field from the stream
 * exactly as field_init (src/field.c:18-23), consuming n*L uniforms; a
 * non-NULL field (L x n, +/-1, slice-major s[l*n+i]) is used as given (the
 * stream still advances by n*L).  Returns the chain id or -1. */
int dqmc_chain_add(dqmc_engine *e, int model, int L, int stab, uint64_t seed,
                   const signed char *field);

/* Sets one chain's delay rank and flush grouping (dqmc_engine_desc's
 * delay_rank and flush_pairs apply to every chain otherwise), before
 * dqmc_engine_prepare: an autotuner gives each size class of a batch its
 * own.  The accept/reject sequence is the same for every setting.  No
 * counterpart in the reference (its delay rank is fixed at 16,
 * src/green.c:10). */
int dqmc_chain_tune(dqmc_engine *e, int chain, int delay_rank, int flush_pairs);

/* Allocates device state for all chains, uploads models and fields and
 * builds each chain's G from scratch (green_from_scratch, src/green.c:262).
 * nbin measurement bins are reserved per chain.  Sweeps launch the chains
 * most expensive first (cost n^3 L). */
int dqmc_engine_prepare(dqmc_engine *e, int nbin);

/* Advances every healthy chain by nsweeps forward sweeps (dqmc_sweep,
 * src/dqmc.c:952-963).  Asynchronous; see dqmc_synchronize. */
int dqmc_sweep(dqmc_engine *e, int nsweeps);

/* As dqmc_sweep, and after each sweep measures every chain (measure_sample,
 * src/measure.c:6-39; measure_szz_sperp_sample, src/structure_factor.c:
 * 328-400) and accumulates the sign-weighted sample into bin `bin`
 * (replica_result_add_sample, src/replica.c:240-269). */
int dqmc_sweep_measure(dqmc_engine *e, int nsweeps, int bin);

/* CUDA-event timing on the engine's stream (the stream every kernel of
 * the engine runs on).  dqmc_kernel_timing(e, 1) records an event pair
 * around every later sweep-kernel and measurement-kernel launch;
 * dqmc_kernel_times waits and returns the summed milliseconds and launch
 * counts since.  dqmc_timer_mark(e, 0|1) records a start/stop event;
 * dqmc_timer_elapsed waits for the stop event and returns the interval. */
int dqmc_kernel_timing(dqmc_engine *e, int enable);
int dqmc_kernel_times(dqmc_engine *e, double *sweep_ms, int *sweep_launches,
                      double *measure_ms, int *measure_launches);
int dqmc_timer_mark(dqmc_engine *e, int which);
int dqmc_timer_elapsed(dqmc_engine *e, double *ms);

/* Waits for queued work; returns nonzero on a CUDA error. */
int dqmc_synchronize(dqmc_engine *e);

int dqmc_chain_count(const dqmc_engine *e);
int dqmc_chain_dims(const dqmc_engine *e, int chain, int *n, int *L);
/* The sweep kernel's residency chosen at dqmc_engine_prepare: chains per
 * SM (1 or 2), the cluster size (1: no clusters) and how many chains, the
 * most expensive ones, run on a cluster each.  No counterpart in the
 * reference. */
int dqmc_engine_residency(const dqmc_engine *e, int *ctas_per_sm, int *chain_ctas,
                          int *cluster_chains);

/* Copies back the up-spin G (n x n) at the chain's current slice (0 after a
 * sweep).  G_down = I - P G_up^T P (src/green.c:372-382). */
int dqmc_read_green(dqmc_engine *e, int chain, double *G);
/* G_down of a chain: the evolved matrix on the two-spin path, else the PH
 * map of G_up (dqmc_map_ph_down, src/dqmc.c:9-17). */
int dqmc_read_green_down(dqmc_engine *e, int chain, double *G);
int dqmc_read_field(dqmc_engine *e, int chain, signed char *field);
/* Replaces a chain's field and rebuilds its G from scratch. */
int dqmc_write_field(dqmc_engine *e, int chain, const signed char *field);
int dqmc_read_counters(dqmc_engine *e, int chain, dqmc_chain_counters *out);
/* Overwrites a chain's G (n x n, column-major host array) without rebuilding
 * it -- the reference's callers own D.Gu.g and its tests corrupt it to check
 * the failure path (tests/test_dqmc.c); a G that is no longer finite stops
 * the chain at its next stabilization point with DQMC_ST_NONFINITE. */
int dqmc_write_green(dqmc_engine *e, int chain, const double *G);
/* Sets a chain's xoshiro256** state (src/rng.h:6-8), e.g. to resume a run
 * from a saved field (dqmc_write_field) and RNG state (read back with
 * dqmc_read_counters).  No counterpart in the reference (no checkpointing). */
int dqmc_write_rng(dqmc_engine *e, int chain, const uint64_t rng[4]);

/* Copies back the bin accumulators: scalars nbin x DQMC_BIN_NFIELDS,
 * szz nbin x nq_zz, sperp nbin x nq_perp (either may be NULL). */
int dqmc_read_bins(dqmc_engine *e, int chain, double *scalars, double *szz,
                   double *sperp);
/* Per-phase SM cycle counters of a chain (the reference's PROF regions,
 * src/profiler.h:6-39, as device clocks): bcache, stack, propose, flush,
 * wrap, bblock, lmul, combine, green, scratch-drift, adopt, measure.
 * Copies min(count, 12) values. */
int dqmc_read_profile(dqmc_engine *e, int chain, unsigned long long *cycles,
                      int count);
/* Calls counted with the same phases: stack builds (bcache), suffix-stack
 * rmuls (stack), accepted flips (propose), G updates (flush), wraps,
 * B-block products, boundary UDV updates, combines, G from UDV, rebuilds
 * from scratch, adoptions, measurements.  Copies min(count, 12) values. */
int dqmc_read_profile_calls(dqmc_engine *e, int chain, unsigned long long *calls,
                            int count);
/* SM clock of the engine's device in Hz (its maximum), to turn the cycle
 * counters into seconds; 0 on error. */
double dqmc_clock_hz(dqmc_engine *e);
/* Clears all bins of all chains. */
int dqmc_clear_bins(dqmc_engine *e);

/* Test entry points (oracle parity).  They return nonzero only on an API or
 * CUDA error; a numerical breakdown is reported as *det_sign == 0. */
/* G from scratch at slice l0 for a chain's current field, without touching
 * the chain (green_from_scratch, src/green.c:262-306). */
int dqmc_green_from_scratch(dqmc_engine *e, int chain, int l0, double *G,
                            int *det_sign);
/* One wrap G <- B_l G B_l^{-1} of a caller G with the chain's field
 * (green_wrap, src/green.c:509-527). */
int dqmc_wrap_green(dqmc_engine *e, int chain, int l, double *G);
/* G = (1 + U diag(D) T)^{-1} and sign det(1 + U D T) on the device for a
 * caller UDV (udv_inv_one_plus_work, src/linalg.c:911-1115; D signed as in
 * the reference). */
int dqmc_udv_green(int device, int n, const double *U, const double *D,
                   const double *T, double *G, int *det_sign);

/* G = (1 + U_L D_L T_L U_R D_R T_R)^-1 and the sign of its determinant from
 * two caller UDV factors (host arrays, column-major n x n; D values signed;
 * the factors are scaled by exp(off_L), exp(off_R) as the reference's
 * log_offset; T_R must be unit upper triangular), by the two-sided
 * reconstruction.  Replaces udv_inv_one_plus_two_sided_work
 * (src/linalg.c:1117-1389).  n <= DQMC_MAX_N. */
int dqmc_udv_green2(int device, int n, const double *UL, const double *DL, const double *TL,
                    double off_L, const double *UR, const double *DR, const double *TR,
                    double off_R, double *G, int *det_sign);

/* Host helper: out = exp(scale * A) for symmetric A (la_expm_sym,
 * src/linalg.c:319-346). */
int dqmc_expm_sym(int n, const double *A, double scale, double *out);

/* No counterpart in the reference.  dqmc_udv_green for callers that must
 * not allocate device memory (their device memory is owned by their own
 * allocator, e.g. a framework's caching pool that has reserved the GPU):
 * the same arguments and result, computed with a fixed scratch array inside
 * the library (about 1.1 MB) instead of allocations.  n is limited to
 * DQMC_NOALLOC_MAX_N; larger n is rejected with an error.  The array and
 * the kernel are placed on a device by the first call on that device (CUDA
 * loads modules lazily), so that first call takes device memory and can
 * fail for lack of it: make it before your allocator reserves the device,
 * and before any stream capture on the device.  Later calls take no device
 * memory; the array is held until the process exits.  A call selects
 * `device`, runs on its legacy default stream, returns after the result is
 * copied back, and restores the caller's current device.  All calls share
 * the array: calls that overlap on the GPU race and must be serialized by
 * the caller. */
#define DQMC_NOALLOC_MAX_N 128
int dqmc_udv_green_noalloc(int device, int n, const double *U, const double *D,
                           const double *T, double *G, int *det_sign);

/* Copies up to max_snapshots of a chain's G snapshots (n x n column-major
 * each, in the order taken; see dqmc_engine_desc.green_log) to out and
 * returns how many, or -1 on error; the log then restarts empty (snapshots
 * beyond its capacity were not kept).  No counterpart in the reference. */
int dqmc_read_green_log(dqmc_engine *e, int chain, double *out, int max_snapshots);

/* Moves up to max_records of a chain's UDV scale records (in the order
 * they were taken, DQMC_UDV_RECORD_DOUBLES each) to out and returns how
 * many, or -1 on error; records beyond max_records stay for the next call.
 * Needs dqmc_engine_desc.udv_diag. */
int dqmc_read_udv_records(dqmc_engine *e, int chain, double *out, int max_records);

#ifdef __cplusplus
}
#endif
#endif
