/*
 * dqmc_host_run: the dqmc_gpu program.  Same input, validation order and
 * output formats as the reference program (SAI-QMC src/main.c:603-2099),
 * but every (beta, replica) chain of the input is one chain of a single
 * batched GPU engine (chains of different L advance in the same launches),
 * instead of one CPU process/thread per replica and beta after beta.
 */
#define _XOPEN_SOURCE 700
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "dqmc_gpu.h"
#include "dqmc_host.h"

/* output_paths_equal (src/scalar_output.c:10-60): same string, same inode,
 * or the same resolved path of the (possibly not yet existing) file. */
static char *resolve(const char *path)
{
    char *r = realpath(path, NULL);
    if (r) return r;
    char *copy = strdup(path);
    if (!copy) return NULL;
    char *slash = strrchr(copy, '/');
    const char *leaf = path, *parent = ".";
    if (slash) {
        *slash = '\0';
        leaf = slash + 1;
        parent = slash == copy ? "/" : copy;
    }
    char *dir = realpath(parent, NULL);
    if (dir) {
        const size_t sz = strlen(dir) + strlen(leaf) + 2;
        r = malloc(sz);
        if (r) snprintf(r, sz, "%s/%s", dir, leaf);
        free(dir);
    }
    free(copy);
    return r;
}

static int same_path(const char *a, const char *b)
{
    if (!strcmp(a, b)) return 1;
    struct stat sa, sb;
    if (stat(a, &sa) == 0 && stat(b, &sb) == 0 && sa.st_dev == sb.st_dev && sa.st_ino == sb.st_ino)
        return 1;
    char *ra = resolve(a), *rb = resolve(b);
    const int same = ra && rb && !strcmp(ra, rb);
    free(ra);
    free(rb);
    return same;
}

/* scalar rows go to stdout and to output_file (src/scalar_output.c:62-109) */
static int scalar_open(FILE **f, const char *path)
{
    *f = NULL;
    if (!strcmp(path, "none")) return 0;
    struct stat so, ss;
    if (stat(path, &so) == 0 && fstat(STDOUT_FILENO, &ss) == 0 && so.st_dev == ss.st_dev &&
        so.st_ino == ss.st_ino)
        return 0;
    *f = fopen(path, "w");
    if (!*f) {
        fprintf(stderr, "ERROR: failed to open output_file %s\n", path);
        return 1;
    }
    return 0;
}

static int sprint(FILE *f, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int failed = vfprintf(stdout, fmt, ap) < 0;
    va_end(ap);
    if (f) {
        va_start(ap, fmt);
        if (vfprintf(f, fmt, ap) < 0) failed = 1;
        va_end(ap);
    }
    return failed;
}

static int sflush(FILE *f)
{
    int failed = fflush(stdout) != 0 || ferror(stdout);
    if (f && (fflush(f) != 0 || ferror(f))) failed = 1;
    if (failed) fprintf(stderr, "ERROR: failed to write scalar output\n");
    return failed;
}

/* write_q_beta / write_spin_consistency_beta (src/main.c:267-377) */
static int write_q(FILE *fp, const DqmcSpinPlan *plan, double breq, double beta, double T,
                   const double *qmajor, const double *qminus, int total)
{
    double *tmp = malloc(sizeof(double) * (size_t)total);
    if (!tmp) return 1;
    for (int q = 0; q < plan->nq; q++) {
        for (int b = 0; b < total; b++) {
            tmp[b] = qminus ? 0.5 * qmajor[q * total + b] - qminus[q * total + b]
                            : qmajor[q * total + b];
            if (!isfinite(tmp[b])) {
                free(tmp);
                return 1;
            }
        }
        double mean, err;
        dqmc_jackknife(tmp, total, &mean, &err);
        const int fmx = plan->Lx > 1 && plan->mx[q] > plan->Lx / 2 ? plan->mx[q] - plan->Lx : plan->mx[q];
        const int fmy = plan->Ly > 1 && plan->my[q] > plan->Ly / 2 ? plan->my[q] - plan->Ly : plan->my[q];
        const double qx = plan->Lx > 1 ? 2.0 * (double)plan->mx[q] / plan->Lx : 0.0;
        const double qy = plan->Ly > 1 ? 2.0 * (double)plan->my[q] / plan->Ly : 0.0;
        const double qxf = plan->Lx > 1 ? 2.0 * (double)fmx / plan->Lx : 0.0;
        const double qyf = plan->Ly > 1 ? 2.0 * (double)fmy / plan->Ly : 0.0;
        fprintf(fp, "%.17g %.17g %.17g %d %d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", breq,
                beta, T, q, plan->mx[q], plan->my[q], qx, qy, qxf, qyf, mean, err);
    }
    free(tmp);
    return (fflush(fp) != 0 || ferror(fp)) ? 1 : 0;
}

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* ---- profile.dat (src/profiler.c) ----------------------------------------
 * Regions and phases in the reference's order (src/profiler.c:10-29).  The
 * sweep work is timed on the device: each chain's SM cycle counters and
 * call counters (include/dqmc_gpu.h) become seconds at the SM clock and are
 * summed over the beta's replicas like the reference's merged per-replica
 * profilers (thread time; with many chains in flight frac_beta exceeds 1,
 * as thread time does under OpenMP).  Device phases map onto regions:
 * dqmc_sweep = every sweep phase, green_stack_build = B-block cache +
 * stack, green_update = proposals + G updates (calls: accepted flips + G
 * updates), green_wrap, udv_lmul (boundary UDV updates, rmuls of backward
 * sweeps included), udv_rmul (suffix-stack rmuls), udv_combine, udv_inv_one_plus (G from UDV),
 * green_from_stack (combine + G from UDV + adoption), green_from_scratch
 * (reference drift rebuilds), measure_sample (the fused measurement,
 * spin correlations included).  Setup regions are host wall time shared by
 * the batch (model_init: the shared model's set-up, counted once per
 * replica as the reference calls it; field_init and dqmc_init in proportion
 * to the beta's chains), finalize = the beta's jackknife and outputs (one
 * call); beta_total = the whole batched run up to this beta's outputs. */
enum { R_BETA_TOTAL, R_MODEL_INIT, R_FIELD_INIT, R_DQMC_INIT, R_DQMC_SWEEP,
       R_GREEN_FROM_SCRATCH, R_GREEN_WRAP, R_GREEN_UPDATE, R_MEASURE_SAMPLE, R_MEASURE_SZZ,
       R_MEASURE_SPERP, R_MEASURE_SPIN, R_JACKKNIFE, R_UDV_LMUL, R_UDV_RMUL, R_UDV_COMBINE,
       R_UDV_INV, R_STACK_BUILD, R_FROM_STACK, R_LA_GEMM, R_LA_INVERSE, R_LA_EXPM, R_COUNT };
static const char *region_names[R_COUNT] = {
    "beta_total", "model_init", "field_init", "dqmc_init", "dqmc_sweep", "green_from_scratch",
    "green_wrap", "green_update", "measure_sample", "measure_szz", "measure_sperp",
    "measure_spin", "jackknife", "udv_lmul", "udv_rmul", "udv_combine", "udv_inv_one_plus",
    "green_stack_build", "green_from_stack", "la_gemm", "la_inverse", "la_expm_sym"};
static const char *prof_phase_names[5] = {"setup", "warmup", "measurement", "finalize", "all"};

typedef struct {
    unsigned long long calls;
    double sec;
} PStat;

typedef struct {
    unsigned long long cy[12], ca[12], sweeps;
} ProfSnap;

/* counters of every chain, beta-major (b * nrep + r) */
static int prof_snapshot(dqmc_engine **engs, int neng, int nrep, int nb, ProfSnap *out)
{
    if (!out) return 1;
    for (int b = 0; b < nb; b++)
        for (int r = 0; r < nrep; r++) {
            const int k = dqmc_replica_rank_for_replica(nrep, neng, r);
            int first, count;
            dqmc_replica_rank_range(nrep, neng, k, &first, &count);
            const int lc = b * count + (r - first);
            ProfSnap *o = out + (size_t)b * nrep + r;
            dqmc_chain_counters cnt;
            if (dqmc_read_profile(engs[k], lc, o->cy, 12) ||
                dqmc_read_profile_calls(engs[k], lc, o->ca, 12) ||
                dqmc_read_counters(engs[k], lc, &cnt))
                return 1;
            o->sweeps = cnt.sweeps;
        }
    return 0;
}

static void padd(PStat *st, unsigned long long calls, double sec)
{
    st->calls += calls;
    st->sec += sec;
}

/* regions of the device counters between two snapshots of one chain */
static void prof_device(PStat *st, const ProfSnap *a, const ProfSnap *b, double hz)
{
    double sec[12];
    unsigned long long ca[12];
    for (int k = 0; k < 12; k++) {
        sec[k] = (double)(b->cy[k] - (a ? a->cy[k] : 0)) / hz;
        ca[k] = b->ca[k] - (a ? a->ca[k] : 0);
    }
    double sweep = 0.0;
    for (int k = 0; k < 11; k++) sweep += sec[k];
    padd(&st[R_DQMC_SWEEP], b->sweeps - (a ? a->sweeps : 0), sweep);
    padd(&st[R_GREEN_FROM_SCRATCH], ca[9], sec[9]);
    padd(&st[R_GREEN_WRAP], ca[4], sec[4]);
    padd(&st[R_GREEN_UPDATE], ca[2] + ca[3], sec[2] + sec[3]);
    padd(&st[R_MEASURE_SAMPLE], ca[11], sec[11]);
    padd(&st[R_UDV_LMUL], ca[6], sec[6]);
    padd(&st[R_UDV_RMUL], ca[1], sec[1]);
    padd(&st[R_UDV_COMBINE], ca[7], sec[7]);
    padd(&st[R_UDV_INV], ca[8], sec[8]);
    padd(&st[R_STACK_BUILD], ca[0], sec[0] + sec[1]);
    padd(&st[R_FROM_STACK], ca[10], sec[7] + sec[8] + sec[10]);
}

/* profiler_beta_end (src/profiler.c:188-223) */
static void prof_rows(FILE *f, double beta, double T, double dtau, int Ltr, int nrep,
                      const char *parallel, int nranks, PStat st[5][R_COUNT])
{
    for (int r = 0; r < R_COUNT; r++)
        for (int ph = 0; ph < 4; ph++) padd(&st[4][r], st[ph][r].calls, st[ph][r].sec);
    const double bt = st[4][R_BETA_TOTAL].sec;
    for (int ph = 0; ph < 5; ph++)
        for (int r = 0; r < R_COUNT; r++) {
            const PStat x = st[ph][r];
            if (x.calls == 0) continue;
            fprintf(f, "%.17g %.17g %.17g %d %s %s %llu %.17g %.17g %.17g %.17g %.17g %d %s", beta,
                    T, dtau, Ltr, prof_phase_names[ph], region_names[r], x.calls, x.sec,
                    x.sec / (double)x.calls, bt > 0.0 ? x.sec / bt : 0.0,
                    r == R_BETA_TOTAL ? bt : 0.0, x.sec, nrep, parallel);
            if (nranks > 1) fprintf(f, " %d", nranks);
            fprintf(f, "\n");
        }
    fflush(f);
}

static int udv_header(const char *path, const char *what, const char *header)
{
    FILE *f = fopen(path, "w");
    if (!f) {
        fprintf(stderr, "ERROR: failed to open %s %s\n", what, path);
        return 1;
    }
    fputs(header, f);
    if (fclose(f)) {
        fprintf(stderr, "ERROR: failed to close %s %s\n", what, path);
        return 1;
    }
    return 0;
}

static const char *udv_direction(int kind)
{
    static const char *names[] = {"stack_suffix_pre_rmul", "stack_prefix_pre_lmul", "forward",
                                  "backward", "left_udv_forward", "left_udv_backward"};
    return kind >= 0 && kind < 6 ? names[kind] : "?";
}

/* One replica's UDV scale records as the reference's diagnostic lines:
 * udv_scale_file rows of dqmc_write_udv_scale_diag (src/dqmc.c:158-194) and
 * udv_centered_file rows of dqmc_record_udv_centered_diag (src/dqmc.c:
 * 287-340).  The engine holds log|D| itself, so effective log D, radius and
 * margin are its own; the stored/offset split of the reference's centered
 * representation is taken as recentered at the record (offset = midpoint of
 * the log D range).  A centered factor that is invalid (zero or non-finite
 * D) or within 8 of the log(DBL_MAX) margin fails the run, as the
 * reference's diagnostic failure stops the replica. */
static int write_udv_records(const DqmcParams *p, dqmc_engine *e, int chain, int b, int Ltr,
                             int r, unsigned long long seed, int n)
{
    FILE *fs = p->udv_scale_file[0] ? fopen(p->udv_scale_file, "a") : NULL;
    FILE *fc = p->udv_centered_file[0] ? fopen(p->udv_centered_file, "a") : NULL;
    int rc = 0;
    if ((p->udv_scale_file[0] && !fs) || (p->udv_centered_file[0] && !fc)) {
        fprintf(stderr, "ERROR: failed to open %s %s\n",
                fs ? "udv_centered_file" : "udv_scale_file",
                fs ? p->udv_centered_file : p->udv_scale_file);
        rc = 1;
    }
    double rec[64 * DQMC_UDV_RECORD_DOUBLES];
    int k;
    while (!rc && (k = dqmc_read_udv_records(e, chain, rec, 64)) > 0) {
        for (int i = 0; i < k; i++) {
            const double *x = rec + (size_t)i * DQMC_UDV_RECORD_DOUBLES;
            const int kind = (int)x[DQMC_UDV_R_KIND], tau = (int)x[DQMC_UDV_R_TAU];
            const int bnd = (int)x[DQMC_UDV_R_BOUNDARY];
            const unsigned long long sw = (unsigned long long)x[DQMC_UDV_R_SWEEP];
            const double *lf = x + DQMC_UDV_R_LEFT, *rt = x + DQMC_UDV_R_RIGHT;
            const int pair = x[DQMC_UDV_R_HAS_RIGHT] != 0.0;
            const char *spin = x[DQMC_UDV_R_SPIN] != 0.0 ? "d" : "u";
            if (fs) {
                const double lsp = lf[2] > 0 ? lf[1] - lf[0] : NAN;
                const double rsp = rt[2] > 0 ? rt[1] - rt[0] : NAN;
                const double cross =
                    pair && isfinite(lf[1]) && isfinite(rt[1]) ? lf[1] + rt[1] : NAN;
                fprintf(fs,
                        "%d %d %d %llu %.17g %.17g %d %llu %d %d %s %s %.17g %.17g %.17g %d %d "
                        "%d %.17g %.17g %.17g %d %d %d %.17g\n",
                        b, Ltr, r, seed, p->U, p->dtau, p->stab_interval, sw, tau, bnd, spin,
                        udv_direction(kind), lf[0], lf[1], lsp, (int)lf[2], (int)lf[3],
                        (int)lf[4], rt[0], rt[1], rsp, (int)rt[2], (int)rt[3], (int)rt[4],
                        cross);
            }
            if (fc) {
                /* the centered factor: left_u, i.e. the right one of a
                 * backward pair (src/dqmc.c:707-709, 831-833) */
                const double *c = kind == DQMC_UDV_BACKWARD ? rt : lf;
                const int valid = (int)c[2] == n && c[3] == 0 && c[4] == 0;
                double smin = NAN, smax = NAN, rad = NAN, off = NAN, emin = NAN, emax = NAN,
                       margin = NAN;
                if (valid) {
                    emin = c[0];
                    emax = c[1];
                    rad = 0.5 * (emax - emin);
                    off = emin + rad;
                    smin = emin - off;
                    smax = emax - off;
                    margin = log(DBL_MAX) - rad;
                }
                int warning = valid && margin <= 32.0;
                const char *status = "ok";
                int fail = 0;
                if (!valid) {
                    status = "invalid_factor";
                    fail = 1;
                } else if (margin <= 8.0) {
                    status = "hard_fail_centered_radius";
                    warning = 1;
                    fail = 1;
                } else if (warning) {
                    status = "warning";
                }
                fprintf(fc,
                        "%d %d %d %llu %llu %d %d %s %s %.17g %.17g %.17g %.17g %.17g %.17g "
                        "%.17g %d %s\n",
                        b, Ltr, r, seed, sw, tau, bnd, spin, udv_direction(kind), smin, smax, rad,
                        off, emin, emax, margin, warning, status);
                if (fail) {
                    fprintf(stderr, "ERROR: centered UDV diagnostic failed (beta_index=%d "
                                    "replica=%d sweep_count=%llu tau=%d status=%s)\n",
                            b, r, sw, tau, status);
                    rc = 1;
                    break;
                }
            }
        }
    }
    if (!rc && k < 0) {
        fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
        rc = 1;
    }
    if (fs && fclose(fs)) rc = 1;
    if (fc && fclose(fc)) rc = 1;
    return rc;
}

/* Engine and local chain index of replica r of beta index b: engine k holds
 * its replica range of every beta, beta-major. */
static dqmc_engine *owner_of(dqmc_engine **engs, int neng, int nrep, int b, int r, int *local)
{
    const int k = dqmc_replica_rank_for_replica(nrep, neng, r);
    int first, count;
    dqmc_replica_rank_range(nrep, neng, k, &first, &count);
    *local = b * count + (r - first);
    return engs[k];
}

int dqmc_host_run(const char *input)
{
    DqmcParams p;
    if (dqmc_params_read(&p, input)) return 1;
    /* validate_scalar_output_path (src/main.c:64-92) */
    if (strcmp(p.output_file, "none")) {
        const char *occ[][2] = {
            {"input", input},
            {"latfile", !strcmp(p.lattice, "file") ? p.latfile : NULL},
            {"hopping matrix", "hopping_used.txt"},
            {"profile_file", p.profile ? (p.profile_file[0] ? p.profile_file : "profile.dat") : NULL},
            {"replica_log", strcmp(p.replica_log, "none") && (p.replica_log[0] || p.nrep > 1)
                                ? (p.replica_log[0] ? p.replica_log : "replicas.dat")
                                : NULL},
            {"szz_file", strcmp(p.szz_q, "none") ? p.szz_file : NULL},
            {"sperp_file", strcmp(p.sperp_q, "none") ? p.sperp_file : NULL},
            {"spin_consistency_file",
             strcmp(p.spin_consistency_file, "none") ? p.spin_consistency_file : NULL},
            {"stab_drift_file", p.stab_drift_file[0] ? p.stab_drift_file : NULL},
            {"udv_scale_file", p.udv_scale_file[0] ? p.udv_scale_file : NULL},
            {"udv_centered_file", p.udv_centered_file[0] ? p.udv_centered_file : NULL}};
        for (size_t i = 0; i < sizeof occ / sizeof occ[0]; i++)
            if (occ[i][1] && occ[i][1][0] && same_path(p.output_file, occ[i][1])) {
                fprintf(stderr, "ERROR: output_file %s collides with %s %s\n", p.output_file,
                        occ[i][0], occ[i][1]);
                return 1;
            }
    }
    DqmcLattice L;
    if (!strcmp(p.lattice, "file")) {
        if (!p.latfile[0]) {
            fprintf(stderr, "ERROR: lattice=file requires latfile\n");
            return 1;
        }
        if (dqmc_lattice_file(&L, p.latfile)) {
            fprintf(stderr, "ERROR: failed to read latfile %s\n", p.latfile);
            return 1;
        }
    } else if (!strcmp(p.lattice, "square")) {
        dqmc_lattice_square(&L, p.Lx, p.Ly, p.thop, p.pbc);
    } else {
        dqmc_lattice_chain(&L, p.Lx, p.thop, p.pbc);
    }
    (void)dqmc_lattice_dump(&L, "hopping_used.txt");
    int rc = 1;
    FILE *scalar = NULL, *replica_fp = NULL, *szz_fp = NULL, *sperp_fp = NULL, *cons_fp = NULL;
    FILE *prof_fp = NULL;
    DqmcSpinPlan zplan = {0}, pplan = {0};
    dqmc_engine *engs[DQMC_MAX_GPUS] = {0};
    int neng = 1, devs[DQMC_MAX_GPUS];
    double *scal = NULL, *zz = NULL, *pp = NULL, *series = NULL, *zbins = NULL, *pbins = NULL;
    unsigned long long *seeds = NULL;
    double tm[5] = {0, 0, 0, 0, 0};   /* model, field, init, warm-up, measurement walls */
    ProfSnap *snap = NULL;
    double t0s = 0.0;
    int *Ltrs = NULL;
    int shared = 0, cons = 0, write_rlog = 0, nb_ok = 0;
    const DqmcSpinPlan *sp = &pplan;
    const char *rlog = NULL, *ppath = NULL;
    if (!L.is_bipartite) {
        fprintf(stderr,
                "ERROR: non-bipartite lattice is outside v1 scope; sign column would be only "
                "relative without determinant-sign initialization\n");
        goto out;
    }
    const double mu = p.U / 2.0;
    if (!strcmp(p.parallel, "mpi") || !strcmp(p.parallel, "hybrid")) {
        fprintf(stderr, "ERROR: parallel=%s requires MPI-enabled build\n", p.parallel);
        goto out;
    }
    if (p.stab_drift_file[0] && strcmp(p.parallel, "serial")) {
        fprintf(stderr, "ERROR: stab_drift_file currently supports parallel=serial only\n");
        goto out;
    }
    /* src/main.c:733-762 */
    if (p.udv_scale_file[0] && strcmp(p.parallel, "serial")) {
        fprintf(stderr, "ERROR: udv_scale_file currently supports parallel=serial only\n");
        goto out;
    }
    if (p.udv_centered_file[0] && strcmp(p.parallel, "serial")) {
        fprintf(stderr, "ERROR: udv_centered_file currently supports parallel=serial only\n");
        goto out;
    }
    if (p.udv_centered_file[0] && strcmp(p.green_rebuild, "centered")) {
        fprintf(stderr, "ERROR: udv_centered_file requires green_rebuild=centered\n");
        goto out;
    }
    /* init_udv_scale_file / init_udv_centered_file (src/main.c:474-515) */
    if (p.udv_scale_file[0] &&
        udv_header(p.udv_scale_file, "udv_scale_file",
                   "# beta_index Ltr replica_id seed U dtau stab_interval sweep_count tau "
                   "boundary spin direction left_min_logD left_max_logD left_spread_logD "
                   "left_finite_count left_zero_count left_nonfinite_count right_min_logD "
                   "right_max_logD right_spread_logD right_finite_count right_zero_count "
                   "right_nonfinite_count cross_max_logD\n"))
        goto out;
    if (p.udv_centered_file[0] &&
        udv_header(p.udv_centered_file, "udv_centered_file",
                   "# beta_index Ltr replica_id seed sweep_count tau boundary spin direction "
                   "stored_min_logD stored_max_logD stored_radius log_offset "
                   "effective_min_logD effective_max_logD remaining_margin warning status\n"))
        goto out;
    if (p.stab_drift_file[0]) {
        FILE *f = fopen(p.stab_drift_file, "w");
        if (!f) {
            fprintf(stderr, "ERROR: failed to open stab_drift_file %s\n", p.stab_drift_file);
            goto out;
        }
        fprintf(f, "# beta_index Ltr replica_id seed U dtau stab use_ph samples max_inf mean_inf "
                   "max_tau max_sweep failed\n");
        fclose(f);
    }
    if (p.nbin > 0 && p.nrep > INT_MAX / p.nbin) {
        fprintf(stderr, "ERROR: nrep*nbin exceeds INT_MAX\n");
        goto out;
    }
    /* spin plans (src/main.c:788-830) */
    int fail = dqmc_spin_plan(&zplan, &L, p.szz_q) != 0;
    shared = !fail && !strcmp(p.szz_q, p.sperp_q);
    if (!fail && !shared && dqmc_spin_plan(&pplan, &L, p.sperp_q)) fail = 1;
    sp = shared ? &zplan : &pplan;
    if (!fail && ((zplan.enabled && !strcmp(p.szz_file, "none")) ||
                  (sp->enabled && !strcmp(p.sperp_file, "none"))))
        fail = 1;
    cons = strcmp(p.spin_consistency_file, "none") != 0;
    if (!fail && cons) {
        if (!zplan.enabled || !sp->enabled || zplan.nq != sp->nq)
            fail = 1;
        else
            for (int q = 0; q < zplan.nq; q++)
                if (zplan.mx[q] != sp->mx[q] || zplan.my[q] != sp->my[q]) fail = 1;
    }
    if (fail) {
        fprintf(stderr,
                "ERROR: invalid spin structure-factor setup szz_selector=%s szz_file=%s "
                "sperp_selector=%s sperp_file=%s consistency_file=%s lattice=%s Lx=%d Ly=%d\n",
                p.szz_q, p.szz_file, p.sperp_q, p.sperp_file, p.spin_consistency_file, p.lattice,
                L.Lx, L.Ly);
        goto out;
    }
    write_rlog = strcmp(p.replica_log, "none") && (p.replica_log[0] || p.nrep > 1);
    rlog = p.replica_log[0] ? p.replica_log : "replicas.dat";
    ppath = p.profile_file[0] ? p.profile_file : "profile.dat";
    {
        const char *act[5][2];
        int na = 0;
        if (p.profile) { act[na][0] = "profile_file"; act[na++][1] = ppath; }
        if (write_rlog) { act[na][0] = "replica_log"; act[na++][1] = rlog; }
        if (zplan.enabled) { act[na][0] = "szz_file"; act[na++][1] = p.szz_file; }
        if (sp->enabled) { act[na][0] = "sperp_file"; act[na++][1] = p.sperp_file; }
        if (cons) { act[na][0] = "spin_consistency_file"; act[na++][1] = p.spin_consistency_file; }
        for (int i = 0; i < na; i++)
            for (int j = i + 1; j < na; j++)
                if (!strcmp(act[i][1], act[j][1])) {
                    fprintf(stderr, "ERROR: output path collision: %s and %s both use %s\n",
                            act[i][0], act[j][0], act[i][1]);
                    goto out;
                }
    }
    if (scalar_open(&scalar, p.output_file)) goto out;
    int sf = sprint(scalar,
                    "# lattice=%s n=%d U=%g mu=%g dtau=%g bipartite=%d green_rebuild=%s "
                    "parallel=%s nrep=%d bins=%d",
                    p.lattice, L.n, p.U, mu, p.dtau, L.is_bipartite, p.green_rebuild, p.parallel,
                    p.nrep, p.nrep * p.nbin);
    if (zplan.enabled) sf |= sprint(scalar, " szz_file=%s szz_nq=%d", p.szz_file, zplan.nq);
    if (sp->enabled) sf |= sprint(scalar, " sperp_file=%s sperp_nq=%d", p.sperp_file, sp->nq);
    if (cons) sf |= sprint(scalar, " spin_consistency_file=%s", p.spin_consistency_file);
    sf |= sprint(scalar, "\n");
    sf |= sprint(scalar, "# T  E_hub dE_hub  E_gc dE_gc  E_ph dE_ph  ntot dN  doublon dD  sign  "
                         "acceptance dAcceptance\n");
    if (sf | sflush(scalar)) goto out;
    if (write_rlog) {
        replica_fp = fopen(rlog, "w");
        if (!replica_fp) {
            fprintf(stderr, "ERROR: failed to open replica_log %s\n", rlog);
            goto out;
        }
        fprintf(replica_fp, "# beta T replica_id seed nwarm nmeas nbin status\n");
    }
    if (zplan.enabled) {
        szz_fp = fopen(p.szz_file, "w");
        if (!szz_fp) {
            fprintf(stderr, "ERROR: failed to open szz_file %s\n", p.szz_file);
            goto out;
        }
        fprintf(szz_fp, "# definition=Szz(q)=N^-1 sum_ij exp[-iq.(ri-rj)] <Szi Szj>\n");
        fprintf(szz_fp, "# spin_operator=Szi=(n_up-n_down)/2 factor3_applied=0\n");
        fprintf(szz_fp, "# lattice=%s Lx=%d Ly=%d n=%d pbc=%d t=%.17g U=%.17g mu=%.17g dtau=%.17g\n",
                p.lattice, L.Lx, L.Ly, L.n, p.pbc, p.thop, p.U, mu, p.dtau);
        fprintf(szz_fp, "# szz_q=%s seed=%llu parallel=%s nrep=%d bins=%d nbeta=%d\n", p.szz_q,
                p.seed, p.parallel, p.nrep, p.nrep * p.nbin, p.nbeta);
        fprintf(szz_fp, "# beta_requested beta T q_index mx my qx_over_pi qy_over_pi "
                        "qx_folded_over_pi qy_folded_over_pi Szz dSzz\n");
    }
    if (sp->enabled) {
        sperp_fp = fopen(p.sperp_file, "w");
        if (!sperp_fp) {
            fprintf(stderr, "ERROR: failed to open sperp_file %s\n", p.sperp_file);
            goto out;
        }
        fprintf(sperp_fp, "# definition=Sperp(q)=N^-1 sum_ij exp[-iq.(ri-rj)] <Sxi Sxj + Syi Syj>\n");
        fprintf(sperp_fp, "# ladder_definition=Sperp(q)=0.5*(S+-(q)+S-+(q)); Splus=Sx+iSy\n");
        fprintf(sperp_fp, "# su2_relation=ensemble Sperp(q)=2*Szz(q) at any dtau for the current "
                          "SU(2)-invariant model\n");
        fprintf(sperp_fp, "# hs_caveat=individual spin-channel-HS samples select the z axis; "
                          "equality is restored by ensemble averaging\n");
        fprintf(sperp_fp, "# lattice=%s Lx=%d Ly=%d n=%d pbc=%d t=%.17g U=%.17g mu=%.17g dtau=%.17g\n",
                p.lattice, L.Lx, L.Ly, L.n, p.pbc, p.thop, p.U, mu, p.dtau);
        fprintf(sperp_fp, "# sperp_q=%s seed=%llu parallel=%s nrep=%d bins=%d nbeta=%d\n", p.sperp_q,
                p.seed, p.parallel, p.nrep, p.nrep * p.nbin, p.nbeta);
        fprintf(sperp_fp, "# beta_requested beta T q_index mx my qx_over_pi qy_over_pi "
                          "qx_folded_over_pi qy_folded_over_pi Sperp dSperp\n");
    }
    if (cons) {
        cons_fp = fopen(p.spin_consistency_file, "w");
        if (!cons_fp) {
            fprintf(stderr, "ERROR: failed to open spin_consistency_file %s\n",
                    p.spin_consistency_file);
            goto out;
        }
        fprintf(cons_fp, "# definition=DeltaSU2(q)=0.5*Sperp(q)-Szz(q)\n");
        fprintf(cons_fp, "# error=paired jackknife over the same sign-reweighted replica/bin samples\n");
        fprintf(cons_fp, "# lattice=%s Lx=%d Ly=%d n=%d pbc=%d t=%.17g U=%.17g mu=%.17g dtau=%.17g\n",
                p.lattice, L.Lx, L.Ly, L.n, p.pbc, p.thop, p.U, mu, p.dtau);
        fprintf(cons_fp, "# szz_q=%s sperp_q=%s seed=%llu parallel=%s nrep=%d bins=%d nbeta=%d\n",
                p.szz_q, p.sperp_q, p.seed, p.parallel, p.nrep, p.nrep * p.nbin, p.nbeta);
        fprintf(cons_fp, "# beta_requested beta T q_index mx my qx_over_pi qy_over_pi "
                         "qx_folded_over_pi qy_folded_over_pi DeltaSU2 dDeltaSU2\n");
    }
    if (p.profile) {
        prof_fp = fopen(ppath, "w");
        if (!prof_fp) {
            fprintf(stderr, "ERROR: failed to initialize profiler output\n");
            goto out;
        }
        /* profiler_init (src/profiler.c:56-76); the MPI build's header when
         * the replicas are split over devices */
        fprintf(prof_fp, "# beta T dtau Ltr phase region calls total_sec avg_sec frac_beta "
                         "wall_sec thread_total_sec nrep parallel%s\n",
                p.ngpu > 1 ? " nranks" : "");
    }
    /* betas run together; the first beta that is not a multiple of dtau
     * ends the run after the betas before it, as the reference does */
    nb_ok = p.nbeta;
    Ltrs = calloc((size_t)p.nbeta, sizeof(int));
    for (int b = 0; b < p.nbeta; b++) {
        const int Ltr = (int)lround(p.beta_list[b] / p.dtau);
        if (fabs(p.beta_list[b] / p.dtau - (double)Ltr) > 1e-9) {
            nb_ok = b;
            break;
        }
        Ltrs[b] = Ltr;
    }
    const int nrep = p.nrep, nbin = p.nbin, total = nrep * nbin;
    seeds = calloc((size_t)(nb_ok * nrep + 1), sizeof(unsigned long long));
    for (int b = 0; b < nb_ok; b++) {
        for (int r = 0; r < nrep; r++) seeds[b * nrep + r] = dqmc_replica_seed(p.seed, b, r);
        for (int i = 0; i < nrep; i++)
            for (int j = i + 1; j < nrep; j++)
                if (seeds[b * nrep + i] == seeds[b * nrep + j]) {
                    fprintf(stderr, "ERROR: duplicate replica seed at beta=%g\n", p.beta_list[b]);
                    goto out;
                }
    }
    t0s = now_s();
    if (p.ngpu > 0) {
        neng = p.ngpu;
        for (int k = 0; k < neng; k++) devs[k] = p.gpu_devices[k];
    } else {
        devs[0] = p.gpu_device;
    }
    if (nb_ok > 0) {
        dqmc_engine_desc d;
        dqmc_desc_default(&d);
        d.precision = !strcmp(p.precision, "mixed") ? DQMC_PREC_MIXED : DQMC_PREC_FP64;
        d.delay_rank = p.delay_rank;
        d.sweep_order = !strcmp(p.sweep_order, "alternating") ? DQMC_SWEEP_ALTERNATING
                                                              : DQMC_SWEEP_FORWARD;
        d.green_rebuild = !strcmp(p.green_rebuild, "two_sided")  ? DQMC_REBUILD_TWO_SIDED
                          : !strcmp(p.green_rebuild, "centered") ? DQMC_REBUILD_CENTERED
                                                                 : DQMC_REBUILD_COMBINE;
        d.drift = DQMC_DRIFT_STAB | (p.stab_drift_file[0] ? DQMC_DRIFT_SCRATCH : 0);
        d.udv_diag = p.udv_scale_file[0] || p.udv_centered_file[0];
        /* one engine per device; device k owns replicas [first_k, first_k +
         * count_k) of every beta (src/replica_mpi.c:13-37 with devices as
         * ranks); all engines advance together (asynchronous launches) */
        for (int k = 0; k < neng; k++) {
            int first, count;
            dqmc_replica_rank_range(nrep, neng, k, &first, &count);
            if (count == 0) continue;
            d.device = devs[k];
            engs[k] = dqmc_engine_create(&d);
            if (!engs[k]) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
            double ts = now_s();
            const int model =
                dqmc_model_add(engs[k], L.n, L.has_coordinates ? L.Lx : 0,
                               L.has_coordinates ? L.Ly : 0, L.t, L.bipart, p.U, p.dtau);
            if (model < 0 ||
                dqmc_model_set_spin(engs[k], model, zplan.enabled ? zplan.nq : 0, zplan.mx,
                                    zplan.my, sp->enabled ? sp->nq : 0, sp->mx, sp->my)) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
            tm[0] += now_s() - ts;
            ts = now_s();
            for (int b = 0; b < nb_ok; b++)
                for (int r = first; r < first + count; r++)
                    if (dqmc_chain_add(engs[k], model, Ltrs[b], p.stab_interval,
                                       seeds[b * nrep + r], NULL) < 0) {
                        fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                        goto out;
                    }
            tm[1] += now_s() - ts;
        }
        const int per = p.nmeas / nbin;
        double ts = now_s();
        for (int k = 0; k < neng; k++)
            if (engs[k] && (dqmc_engine_prepare(engs[k], nbin) || dqmc_synchronize(engs[k]))) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
        tm[2] = now_s() - ts;
        ts = now_s();
        for (int k = 0; k < neng; k++)
            if (engs[k] && dqmc_sweep(engs[k], p.nwarm)) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
        if (prof_fp) {   /* profiler phase boundary (src/replica_run.c:183-200) */
            for (int k = 0; k < neng; k++)
                if (engs[k] && dqmc_synchronize(engs[k])) {
                    fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                    goto out;
                }
            tm[3] = now_s() - ts;
            if (prof_snapshot(engs, neng, nrep, nb_ok, snap = calloc((size_t)nb_ok * nrep * 2,
                                                                        sizeof(ProfSnap)))) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
            ts = now_s();
        }
        for (int bi = 0; bi < nbin; bi++)
            for (int k = 0; k < neng; k++)
                if (engs[k] && dqmc_sweep_measure(engs[k], per, bi)) {
                    fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                    goto out;
                }
        for (int k = 0; k < neng; k++)
            if (engs[k] && dqmc_synchronize(engs[k])) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
        if (prof_fp) {
            tm[4] = now_s() - ts;
            if (prof_snapshot(engs, neng, nrep, nb_ok, snap + (size_t)nb_ok * nrep)) {
                fprintf(stderr, "ERROR: %s\n", dqmc_last_error());
                goto out;
            }
        }
    }
    scal = malloc(sizeof(double) * (size_t)nbin * DQMC_BIN_NFIELDS);
    zz = malloc(sizeof(double) * (size_t)nbin * (zplan.nq + 1));
    pp = malloc(sizeof(double) * (size_t)nbin * (sp->nq + 1));
    series = malloc(sizeof(double) * (size_t)total * 7);
    zbins = malloc(sizeof(double) * (size_t)total * (zplan.nq + 1));
    pbins = malloc(sizeof(double) * (size_t)total * (sp->nq + 1));
    if (!scal || !zz || !pp || !series || !zbins || !pbins) goto out;
    for (int b = 0; b < nb_ok; b++) {
        const double beta = p.beta_list[b], beta_eff = Ltrs[b] * p.dtau, T = 1.0 / beta_eff;
        int any_failed = 0;
        const double tfin = now_s();
        for (int r = 0; r < nrep; r++) {
            const int c = b * nrep + r;
            int lc;
            dqmc_engine *e = owner_of(engs, neng, nrep, b, r, &lc);
            dqmc_chain_counters cnt;
            dqmc_read_counters(e, lc, &cnt);
            if (cnt.status) {
                fprintf(stderr,
                        "ERROR: dqmc numerical breakdown (beta_index=%d beta=%.17g T=%.17g "
                        "replica=%d seed=%llu U=%g dtau=%g Ltr=%d stab=%d sweep_count=%llu "
                        "status=%d)\n",
                        b, beta_eff, T, r, seeds[c], p.U, p.dtau, Ltrs[b], p.stab_interval,
                        cnt.sweeps, cnt.status);
                fprintf(stderr, "ERROR: replica %d failed\n", r);
                any_failed = 1;
            }
            if (p.stab_drift_file[0]) {
                FILE *f = fopen(p.stab_drift_file, "a");
                if (!f) {
                    fprintf(stderr, "ERROR: failed to open stab_drift_file %s\n", p.stab_drift_file);
                    goto out;
                }
                fprintf(f, "%d %d %d %llu %.17g %.17g %d %d %llu %.17g %.17g %d %llu %d\n", b,
                        Ltrs[b], r, seeds[c], p.U, p.dtau, p.stab_interval, 1,
                        cnt.scratch_drift_samples, cnt.scratch_drift_max, cnt.scratch_drift_mean,
                        cnt.scratch_drift_max_tau, cnt.scratch_drift_max_sweep, cnt.status ? 1 : 0);
                fclose(f);
            }
            if ((p.udv_scale_file[0] || p.udv_centered_file[0]) &&
                write_udv_records(&p, e, lc, b, Ltrs[b], r, seeds[c], L.n))
                goto out;
        }
        if (replica_fp) {
            for (int r = 0; r < nrep; r++) {
                int lc;
                dqmc_engine *e = owner_of(engs, neng, nrep, b, r, &lc);
                dqmc_chain_counters cnt;
                dqmc_read_counters(e, lc, &cnt);
                if (neng > 1) /* the owner column of the MPI runner (src/main.c:1216-1232) */
                    fprintf(replica_fp, "%.17g %.17g %d %llu %d %d %d %s %d\n", beta, T, r,
                            seeds[b * nrep + r], p.nwarm, p.nmeas, nbin,
                            cnt.status ? "error" : "ok",
                            dqmc_replica_rank_for_replica(nrep, neng, r));
                else
                    fprintf(replica_fp, "%.17g %.17g %d %llu %d %d %d %s\n", beta, T, r,
                            seeds[b * nrep + r], p.nwarm, p.nmeas, nbin,
                            cnt.status ? "error" : "ok");
            }
            fflush(replica_fp);
        }
        if (any_failed) goto out;
        double *Eh = series, *Eg = Eh + total, *Ep = Eg + total, *Nn = Ep + total,
               *Dd = Nn + total, *Ss = Dd + total, *Ac = Ss + total;
        for (int r = 0; r < nrep; r++) {
            int lc;
            dqmc_engine *e = owner_of(engs, neng, nrep, b, r, &lc);
            dqmc_read_bins(e, lc, scal, zz, pp);
            for (int bi = 0; bi < nbin; bi++) {
                const int o = r * nbin + bi;
                const double *bf = scal + (size_t)bi * DQMC_BIN_NFIELDS;
                double v[6];
                if (dqmc_bin_values(bf, v)) {
                    fprintf(stderr,
                            "ERROR: invalid bin at beta=%.17g replica=%d bin=%d count=%d "
                            "sum_sign=%.17g\n",
                            beta, r, bi, (int)bf[DQMC_BIN_COUNT_F], bf[DQMC_BIN_SUM_SIGN]);
                    goto out;
                }
                Eh[o] = v[0];
                Eg[o] = v[1];
                Ep[o] = v[2];
                Nn[o] = v[3];
                Dd[o] = v[4];
                Ss[o] = v[5];
                Ac[o] = bf[DQMC_BIN_ATTEMPTS_F] > 0 ? bf[DQMC_BIN_ACCEPTED_F] / bf[DQMC_BIN_ATTEMPTS_F]
                                                    : 0.0;
                const double ss = bf[DQMC_BIN_SUM_SIGN];
                if (zplan.enabled) {
                    double *vals = zz + (size_t)bi * zplan.nq;
                    for (int q = 0; q < zplan.nq; q++) vals[q] /= ss;
                    double lhs = 0, rhs = 0;
                    if (dqmc_sum_rule(&zplan, vals, v[3], v[4], 0.25, &lhs, &rhs)) {
                        fprintf(stderr,
                                "ERROR: Szz sum rule failed at beta=%.17g replica=%d bin=%d "
                                "lhs=%.17g rhs=%.17g diff=%.17g sum_sign=%.17g\n",
                                beta, r, bi, lhs, rhs, lhs - rhs, ss);
                        goto out;
                    }
                    for (int q = 0; q < zplan.nq; q++) zbins[q * total + o] = vals[q];
                }
                if (sp->enabled) {
                    double *vals = pp + (size_t)bi * sp->nq;
                    for (int q = 0; q < sp->nq; q++) vals[q] /= ss;
                    double lhs = 0, rhs = 0;
                    if (dqmc_sum_rule(sp, vals, v[3], v[4], 0.5, &lhs, &rhs)) {
                        fprintf(stderr,
                                "ERROR: Sperp sum rule failed at beta=%.17g replica=%d bin=%d "
                                "lhs=%.17g rhs=%.17g diff=%.17g sum_sign=%.17g\n",
                                beta, r, bi, lhs, rhs, lhs - rhs, ss);
                        goto out;
                    }
                    for (int q = 0; q < sp->nq; q++) pbins[q * total + o] = vals[q];
                }
            }
        }
        char row[512];
        if (dqmc_format_row(row, sizeof row, T, Eh, Eg, Ep, Nn, Dd, Ss, Ac, total)) {
            fprintf(stderr, "ERROR: non-finite or empty jackknife input at T=%.17g total_bins=%d\n",
                    T, total);
            goto out;
        }
        if (sprint(scalar, "%s", row) | sflush(scalar)) goto out;
        if (zplan.enabled && write_q(szz_fp, &zplan, beta, beta_eff, T, zbins, NULL, total)) {
            fprintf(stderr, "ERROR: failed to finalize Szz at beta=%.17g\n", beta);
            goto out;
        }
        if (sp->enabled && write_q(sperp_fp, sp, beta, beta_eff, T, pbins, NULL, total)) {
            fprintf(stderr, "ERROR: failed to finalize Sperp at beta=%.17g\n", beta);
            goto out;
        }
        if (cons && write_q(cons_fp, &zplan, beta, beta_eff, T, pbins, zbins, total)) {
            fprintf(stderr, "ERROR: failed to finalize spin consistency at beta=%.17g\n", beta);
            goto out;
        }
        if (prof_fp) {
            PStat st[5][R_COUNT];
            memset(st, 0, sizeof st);
            const double hz = dqmc_clock_hz(engs[dqmc_replica_rank_for_replica(nrep, neng, 0)]);
            const double share = (double)nrep / (double)(nrep * nb_ok);
            padd(&st[0][R_MODEL_INIT], nrep, tm[0]);   /* one model_init per replica */
            padd(&st[0][R_FIELD_INIT], nrep, tm[1] * share);
            padd(&st[0][R_DQMC_INIT], nrep, tm[2] * share);
            for (int r = 0; r < nrep; r++) {
                const ProfSnap *w = snap + (size_t)b * nrep + r;
                const ProfSnap *m = snap + (size_t)(nb_ok + b) * nrep + r;
                if (hz > 0) {
                    prof_device(st[1], NULL, w, hz);
                    prof_device(st[2], w, m, hz);
                }
            }
            const double tend = now_s();
            padd(&st[3][R_JACKKNIFE], 1, tend - tfin);   /* one finalize per beta */
            st[4][R_BETA_TOTAL].calls = 1;
            st[4][R_BETA_TOTAL].sec = (tfin - t0s) + (tend - tfin);
            prof_rows(prof_fp, beta, T, p.dtau, Ltrs[b], nrep, p.parallel, neng, st);
        }
    }
    if (nb_ok < p.nbeta) {
        const double beta = p.beta_list[nb_ok];
        fprintf(stderr, "ERROR: beta=%g not a multiple of dtau=%g (beta/dtau=%g)\n", beta, p.dtau,
                beta / p.dtau);
        goto out;
    }
    rc = 0;
out:
    for (int k = 0; k < DQMC_MAX_GPUS; k++)
        if (engs[k]) dqmc_engine_destroy(engs[k]);
    if (scalar) fclose(scalar);
    if (replica_fp) fclose(replica_fp);
    if (szz_fp) fclose(szz_fp);
    if (sperp_fp) fclose(sperp_fp);
    if (cons_fp) fclose(cons_fp);
    if (prof_fp) fclose(prof_fp);
    if (!shared) dqmc_spin_plan_free(&pplan);
    dqmc_spin_plan_free(&zplan);
    dqmc_lattice_free(&L);
    free(scal);
    free(zz);
    free(pp);
    free(series);
    free(zbins);
    free(pbins);
    free(seeds);
    free(Ltrs);
    free(snap);
    return rc;
}
