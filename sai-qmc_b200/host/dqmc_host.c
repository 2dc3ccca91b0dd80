/*
 * Host side of the dqmc_gpu driver: input, lattices, spin plans, binning,
 * jackknife and output writers, plus dqmc_host_run, which replaces the
 * reference's main() (SAI-QMC src/main.c:603-2099) with one batched GPU
 * engine: every (beta, replica) chain of the input advances together.
 * Formats and validation messages follow the reference so that outputs are
 * interchangeable; engine-specific keys are delay_rank, precision,
 * gpu_device and gpu_devices.
 */
#define _XOPEN_SOURCE 700
#include "dqmc_host.h"

#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include "dqmc_gpu.h"

/* ------------------------------------------------------------- parser */
static int parse_int(const char *s, int *out)
{
    char *end = NULL;
    errno = 0;
    const long v = strtol(s, &end, 10);
    if (errno || end == s || *end != '\0' || v < INT_MIN || v > INT_MAX) return 1;
    *out = (int)v;
    return 0;
}

static int parse_ull(const char *s, unsigned long long *out)
{
    char *end = NULL;
    errno = 0;
    if (s[0] == '-') return 1;
    const unsigned long long v = strtoull(s, &end, 10);
    if (errno || end == s || *end != '\0') return 1;
    *out = v;
    return 0;
}

static int parse_dbl(const char *s, double *out)
{
    char *end = NULL;
    errno = 0;
    const double v = strtod(s, &end);
    if (errno || end == s || *end != '\0' || !isfinite(v)) return 1;
    *out = v;
    return 0;
}

static void copy_str(char *dst, size_t cap, const char *src)
{
    size_t n = strlen(src);
    if (n >= cap) n = cap - 1;
    memcpy(dst, src, n);
    dst[n] = '\0';
}

/* io.c:71-103 defaults */
static void params_defaults(DqmcParams *p)
{
    memset(p, 0, sizeof *p);
    strcpy(p->lattice, "chain");
    p->Lx = 4;
    p->Ly = 1;
    p->pbc = 1;
    p->thop = -1.0;
    p->U = 4.0;
    p->dtau = 0.1;
    p->nwarm = 200;
    p->nmeas = 2000;
    p->nbin = 20;
    p->stab_interval = 8;
    strcpy(p->output_file, "observables.dat");
    strcpy(p->sweep_order, "forward");
    strcpy(p->green_rebuild, "combine");
    strcpy(p->parallel, "serial");
    p->nrep = 1;
    strcpy(p->szz_q, "none");
    strcpy(p->szz_file, "szz.dat");
    strcpy(p->sperp_q, "none");
    strcpy(p->sperp_file, "sperp.dat");
    strcpy(p->spin_consistency_file, "none");
    p->seed = 12345ULL;
    strcpy(p->precision, "fp64");
}

static int strict_key(const char *k)
{
    return !strcmp(k, "output_file") || !strcmp(k, "szz_q") || !strcmp(k, "szz_file") ||
           !strcmp(k, "sperp_q") || !strcmp(k, "sperp_file") ||
           !strcmp(k, "spin_consistency_file");
}

/* io.c:105-145: the value is the whole trimmed remainder, no inner space */
static int strict_value(const char *line, const char *key, char out[256])
{
    const char *eq = strchr(line, '=');
    if (!eq) return 1;
    const char *kb = line;
    while (isspace((unsigned char)*kb)) kb++;
    const char *ke = eq;
    while (ke > kb && isspace((unsigned char)ke[-1])) ke--;
    if ((size_t)(ke - kb) != strlen(key) || strncmp(kb, key, strlen(key))) return 1;
    const char *vb = eq + 1;
    while (isspace((unsigned char)*vb)) vb++;
    const char *ve = vb + strlen(vb);
    while (ve > vb && isspace((unsigned char)ve[-1])) ve--;
    const size_t len = (size_t)(ve - vb);
    if (len == 0 || len >= 256) return 1;
    for (const char *q = vb; q < ve; q++)
        if (isspace((unsigned char)*q)) return 1;
    memcpy(out, vb, len);
    out[len] = '\0';
    return 0;
}

int dqmc_params_read(DqmcParams *p, const char *path)
{
    params_defaults(p);
    FILE *fp = fopen(path, "r");
    if (!fp) {
        perror(path);
        return 1;
    }
#define FAIL(...)                     \
    do {                              \
        fprintf(stderr, __VA_ARGS__); \
        fclose(fp);                   \
        return 1;                     \
    } while (0)
    char line[512];
    int lineno = 0;
    while (fgets(line, sizeof line, fp)) {
        lineno++;
        if (!strchr(line, '\n') && !feof(fp))
            FAIL("ERROR: input line %d exceeds %zu bytes\n", lineno, sizeof line - 1);
        char *hash = strchr(line, '#');
        if (hash) *hash = '\0';
        char key[64], val[256];
        if (sscanf(line, "%63[^= \t]=%255s", key, val) != 2) {
            char probe[64];
            if (sscanf(line, " %63[^= \t]", probe) == 1 && strict_key(probe))
                FAIL("ERROR: invalid %s value on line %d\n", probe, lineno);
            continue;
        }
        if (strict_key(key) && strict_value(line, key, val))
            FAIL("ERROR: invalid %s value on line %d\n", key, lineno);
        if (!strcmp(key, "lattice")) {
            copy_str(p->lattice, sizeof p->lattice, val);
        } else if (!strcmp(key, "latfile")) {
            copy_str(p->latfile, sizeof p->latfile, val);
        } else if (!strcmp(key, "Lx")) {
            if (parse_int(val, &p->Lx)) FAIL("ERROR: Lx must be integer (got %s)\n", val);
        } else if (!strcmp(key, "Ly")) {
            if (parse_int(val, &p->Ly)) FAIL("ERROR: Ly must be integer (got %s)\n", val);
        } else if (!strcmp(key, "pbc")) {
            if (parse_int(val, &p->pbc)) FAIL("ERROR: pbc must be 0 or 1 (got %s)\n", val);
        } else if (!strcmp(key, "bc")) {
            if (!strcmp(val, "periodic") || !strcmp(val, "pbc") || !strcmp(val, "1"))
                p->pbc = 1;
            else if (!strcmp(val, "open") || !strcmp(val, "obc") || !strcmp(val, "0"))
                p->pbc = 0;
            else
                FAIL("ERROR: bc must be periodic/open/pbc/obc/1/0 (got %s)\n", val);
        } else if (!strcmp(key, "t")) {
            if (parse_dbl(val, &p->thop)) FAIL("ERROR: t must be numeric (got %s)\n", val);
        } else if (!strcmp(key, "U")) {
            if (parse_dbl(val, &p->U)) FAIL("ERROR: U must be numeric (got %s)\n", val);
        } else if (!strcmp(key, "dtau")) {
            if (parse_dbl(val, &p->dtau)) FAIL("ERROR: dtau must be numeric (got %s)\n", val);
        } else if (!strcmp(key, "nwarm")) {
            if (parse_int(val, &p->nwarm)) FAIL("ERROR: nwarm must be integer (got %s)\n", val);
        } else if (!strcmp(key, "nmeas")) {
            if (parse_int(val, &p->nmeas)) FAIL("ERROR: nmeas must be integer (got %s)\n", val);
        } else if (!strcmp(key, "nbin")) {
            if (parse_int(val, &p->nbin)) FAIL("ERROR: nbin must be integer (got %s)\n", val);
        } else if (!strcmp(key, "stab") || !strcmp(key, "stabilize_interval")) {
            if (parse_int(val, &p->stab_interval))
                FAIL("ERROR: stab must be integer (got %s)\n", val);
        } else if (!strcmp(key, "output_file")) {
            copy_str(p->output_file, sizeof p->output_file, val);
        } else if (!strcmp(key, "profile")) {
            if (parse_int(val, &p->profile))
                FAIL("ERROR: profile must be 0 or 1 (got %s)\n", val);
        } else if (!strcmp(key, "profile_file")) {
            copy_str(p->profile_file, sizeof p->profile_file, val);
        } else if (!strcmp(key, "stab_drift_file") ||
                   !strcmp(key, "stabilization_drift_file")) {
            copy_str(p->stab_drift_file, sizeof p->stab_drift_file, val);
        } else if (!strcmp(key, "udv_scale_file") ||
                   !strcmp(key, "udv_scale_diagnostics_file")) {
            copy_str(p->udv_scale_file, sizeof p->udv_scale_file, val);
        } else if (!strcmp(key, "udv_centered_file") ||
                   !strcmp(key, "udv_centered_diagnostics_file")) {
            copy_str(p->udv_centered_file, sizeof p->udv_centered_file, val);
        } else if (!strcmp(key, "sweep_order")) {
            copy_str(p->sweep_order, sizeof p->sweep_order, val);
        } else if (!strcmp(key, "green_rebuild")) {
            copy_str(p->green_rebuild, sizeof p->green_rebuild, val);
        } else if (!strcmp(key, "parallel")) {
            copy_str(p->parallel, sizeof p->parallel, val);
        } else if (!strcmp(key, "nrep")) {
            if (parse_int(val, &p->nrep)) FAIL("ERROR: nrep must be integer (got %s)\n", val);
        } else if (!strcmp(key, "replica_log")) {
            copy_str(p->replica_log, sizeof p->replica_log, val);
        } else if (!strcmp(key, "szz_q")) {
            copy_str(p->szz_q, sizeof p->szz_q, val);
        } else if (!strcmp(key, "szz_file")) {
            copy_str(p->szz_file, sizeof p->szz_file, val);
        } else if (!strcmp(key, "sperp_q")) {
            copy_str(p->sperp_q, sizeof p->sperp_q, val);
        } else if (!strcmp(key, "sperp_file")) {
            copy_str(p->sperp_file, sizeof p->sperp_file, val);
        } else if (!strcmp(key, "spin_consistency_file")) {
            copy_str(p->spin_consistency_file, sizeof p->spin_consistency_file, val);
        } else if (!strcmp(key, "seed")) {
            if (parse_ull(val, &p->seed))
                FAIL("ERROR: seed must be unsigned integer (got %s)\n", val);
        } else if (!strcmp(key, "beta_list")) {
            p->nbeta = 0;
            char *tok = strtok(val, ",");
            if (!tok) FAIL("ERROR: beta_list must contain positive numeric values\n");
            while (tok) {
                if (p->nbeta >= DQMC_MAX_BETA)
                    FAIL("ERROR: beta_list has too many entries (max 64)\n");
                if (parse_dbl(tok, &p->beta_list[p->nbeta]) || p->beta_list[p->nbeta] <= 0.0)
                    FAIL("ERROR: beta_list must contain positive numeric values\n");
                p->nbeta++;
                tok = strtok(NULL, ",");
            }
        } else if (!strcmp(key, "delay_rank")) {
            if (parse_int(val, &p->delay_rank) || p->delay_rank < 0 || p->delay_rank > 64)
                FAIL("ERROR: delay_rank must be an integer in 0..64 (got %s)\n", val);
        } else if (!strcmp(key, "precision")) {
            if (strcmp(val, "fp64") && strcmp(val, "mixed"))
                FAIL("ERROR: precision must be fp64 or mixed (got %s)\n", val);
            copy_str(p->precision, sizeof p->precision, val);
        } else if (!strcmp(key, "gpu_device")) {
            if (parse_int(val, &p->gpu_device) || p->gpu_device < 0)
                FAIL("ERROR: gpu_device must be a non-negative integer (got %s)\n", val);
        } else if (!strcmp(key, "gpu_devices")) {
            p->ngpu = 0;
            char *tok = strtok(val, ",");
            if (!tok) FAIL("ERROR: gpu_devices must list non-negative device ordinals\n");
            while (tok) {
                if (p->ngpu >= DQMC_MAX_GPUS)
                    FAIL("ERROR: gpu_devices has too many entries (max %d)\n", DQMC_MAX_GPUS);
                if (parse_int(tok, &p->gpu_devices[p->ngpu]) || p->gpu_devices[p->ngpu] < 0)
                    FAIL("ERROR: gpu_devices must list non-negative device ordinals\n");
                p->ngpu++;
                tok = strtok(NULL, ",");
            }
        } else {
            FAIL("ERROR: unknown key %s\n", key);
        }
    }
    fclose(fp);
#undef FAIL
    if (p->nbeta == 0) {
        p->beta_list[0] = 2.0;
        p->nbeta = 1;
    }
    /* io.c:345-417 */
    if (strcmp(p->lattice, "chain") && strcmp(p->lattice, "square") && strcmp(p->lattice, "file")) {
        fprintf(stderr, "ERROR: lattice must be chain, square, or file (got %s)\n", p->lattice);
        return 1;
    }
    if (p->Lx <= 0) { fprintf(stderr, "ERROR: Lx must be > 0\n"); return 1; }
    if (p->Ly <= 0) { fprintf(stderr, "ERROR: Ly must be > 0\n"); return 1; }
    if (p->pbc != 0 && p->pbc != 1) { fprintf(stderr, "ERROR: pbc must be 0 or 1\n"); return 1; }
    if (p->U < 0.0) { fprintf(stderr, "ERROR: U must be >= 0\n"); return 1; }
    if (p->dtau <= 0.0) { fprintf(stderr, "ERROR: dtau must be > 0\n"); return 1; }
    if (p->nwarm < 0) { fprintf(stderr, "ERROR: nwarm must be >= 0\n"); return 1; }
    if (p->stab_interval <= 0) { fprintf(stderr, "ERROR: stab must be > 0\n"); return 1; }
    if (p->profile != 0 && p->profile != 1) {
        fprintf(stderr, "ERROR: profile must be 0 or 1 (got %d)\n", p->profile);
        return 1;
    }
    if (strcmp(p->sweep_order, "forward") && strcmp(p->sweep_order, "alternating")) {
        fprintf(stderr, "ERROR: sweep_order must be forward or alternating (got %s)\n",
                p->sweep_order);
        return 1;
    }
    if (strcmp(p->green_rebuild, "combine") && strcmp(p->green_rebuild, "two_sided") &&
        strcmp(p->green_rebuild, "centered")) {
        fprintf(stderr,
                "ERROR: green_rebuild must be combine, two_sided, or centered (got %s)\n",
                p->green_rebuild);
        return 1;
    }
    if (strcmp(p->parallel, "serial") && strcmp(p->parallel, "omp") &&
        strcmp(p->parallel, "mpi") && strcmp(p->parallel, "hybrid")) {
        fprintf(stderr, "ERROR: parallel must be serial, omp, mpi, or hybrid (got %s)\n",
                p->parallel);
        return 1;
    }
    if (p->nrep < 1) { fprintf(stderr, "ERROR: nrep must be >= 1 (got %d)\n", p->nrep); return 1; }
    if (p->nbin < 2) { fprintf(stderr, "ERROR: nbin must be >= 2 (got %d)\n", p->nbin); return 1; }
    if (p->nmeas < p->nbin) {
        fprintf(stderr, "ERROR: nmeas (%d) must be >= nbin (%d)\n", p->nmeas, p->nbin);
        return 1;
    }
    if (p->nmeas % p->nbin != 0) {
        fprintf(stderr, "ERROR: nmeas (%d) must be divisible by nbin (%d)\n", p->nmeas, p->nbin);
        return 1;
    }
    return 0;
}

/* ------------------------------------------------------------ lattices */
static int lat_alloc(DqmcLattice *L, int n)
{
    memset(L, 0, sizeof *L);
    L->n = n;
    L->t = calloc((size_t)n * n, sizeof(double));
    L->bipart = calloc((size_t)n, sizeof(int));
    L->is_bipartite = 1;
    return (L->t && L->bipart) ? 0 : 1;
}

static void bond(DqmcLattice *L, int i, int j, double t)
{
    L->t[i + (size_t)j * L->n] += t;
    L->t[j + (size_t)i * L->n] += t;
}

/* lattice_chain (src/lattice.c:26-44) */
int dqmc_lattice_chain(DqmcLattice *L, int Lx, double t, int pbc)
{
    if (Lx <= 0 || lat_alloc(L, Lx)) return 1;
    L->type = 1;
    L->Lx = Lx;
    L->Ly = 1;
    L->has_coordinates = 1;
    for (int x = 0; x < Lx; x++) {
        if (x + 1 < Lx) bond(L, x, x + 1, t);
        else if (pbc && Lx > 1) bond(L, x, 0, t);
        L->bipart[x] = (x % 2 == 0) ? 1 : -1;
    }
    L->is_bipartite = (pbc && Lx > 1 && Lx % 2 != 0) ? 0 : 1;
    return 0;
}

/* lattice_square (src/lattice.c:46-82) */
int dqmc_lattice_square(DqmcLattice *L, int Lx, int Ly, double t, int pbc)
{
    if (Lx <= 0 || Ly <= 0 || lat_alloc(L, Lx * Ly)) return 1;
    L->type = 2;
    L->Lx = Lx;
    L->Ly = Ly;
    L->has_coordinates = 1;
    for (int y = 0; y < Ly; y++)
        for (int x = 0; x < Lx; x++) {
            const int i = x + y * Lx;
            if (x + 1 < Lx) bond(L, i, (x + 1) + y * Lx, t);
            else if (pbc && Lx > 1) bond(L, i, y * Lx, t);
            if (y + 1 < Ly) bond(L, i, x + (y + 1) * Lx, t);
            else if (pbc && Ly > 1) bond(L, i, x, t);
            L->bipart[i] = ((x + y) % 2 == 0) ? 1 : -1;
        }
    const int odd = (pbc && Lx > 1 && Lx % 2 != 0) || (pbc && Ly > 1 && Ly % 2 != 0);
    L->is_bipartite = odd ? 0 : 1;
    return 0;
}

/* lattice_from_file (src/lattice.c:84-182): n, then the n x n hopping
 * matrix row by row; two-colouring by breadth-first search. */
int dqmc_lattice_file(DqmcLattice *L, const char *path)
{
    FILE *fp = fopen(path, "r");
    if (!fp) {
        perror(path);
        return 1;
    }
    int n = 0;
    if (fscanf(fp, "%d", &n) != 1 || n <= 0) {
        fprintf(stderr, "ERROR: hopping matrix size must be positive\n");
        fclose(fp);
        return 1;
    }
    if (lat_alloc(L, n)) {
        fclose(fp);
        return 1;
    }
    L->type = 3;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double v = 0.0;
            if (fscanf(fp, "%lf", &v) != 1) {
                fclose(fp);
                dqmc_lattice_free(L);
                return 1;
            }
            L->t[i + (size_t)j * n] = v;
        }
    fclose(fp);
    for (int i = 0; i < n; i++)
        if (fabs(L->t[i + (size_t)i * n]) > 1e-12) {
            fprintf(stderr, "ERROR: hopping matrix diagonal must be zero at (%d,%d)\n", i, i);
            dqmc_lattice_free(L);
            return 1;
        }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (fabs(L->t[i + (size_t)j * n] - L->t[j + (size_t)i * n]) > 1e-12) {
                fprintf(stderr, "ERROR: hopping matrix not symmetric at (%d,%d)\n", i, j);
                dqmc_lattice_free(L);
                return 1;
            }
    int *q = malloc(sizeof(int) * (size_t)n);
    L->is_bipartite = 1;
    for (int s = 0; s < n && L->is_bipartite; s++) {
        if (L->bipart[s] != 0) continue;
        L->bipart[s] = 1;
        int head = 0, tail = 0;
        q[tail++] = s;
        while (head < tail && L->is_bipartite) {
            const int i = q[head++];
            for (int j = 0; j < n; j++) {
                if (i == j || fabs(L->t[i + (size_t)j * n]) <= 1e-12) continue;
                const int want = -L->bipart[i];
                if (L->bipart[j] == 0) {
                    L->bipart[j] = want;
                    q[tail++] = j;
                } else if (L->bipart[j] != want) {
                    L->is_bipartite = 0;
                    break;
                }
            }
        }
    }
    if (!L->is_bipartite)
        for (int i = 0; i < n; i++) L->bipart[i] = 0;
    free(q);
    return 0;
}

int dqmc_lattice_dump(const DqmcLattice *L, const char *path)
{
    FILE *fp = fopen(path, "w");
    if (!fp) {
        perror(path);
        return 1;
    }
    const int n = L->n;
    fprintf(fp, "%d\n", n);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            fprintf(fp, "%.17g%c", L->t[i + (size_t)j * n], (j == n - 1) ? '\n' : ' ');
    fclose(fp);
    return 0;
}

void dqmc_lattice_free(DqmcLattice *L)
{
    free(L->t);
    free(L->bipart);
    memset(L, 0, sizeof *L);
}

/* ---------------------------------------------------------- spin plans */
void dqmc_spin_plan_free(DqmcSpinPlan *plan)
{
    if (!plan) return;
    free(plan->mx);
    free(plan->my);
    memset(plan, 0, sizeof *plan);
}

/* structure_factor_plan_init (src/structure_factor.c:107-206) */
int dqmc_spin_plan(DqmcSpinPlan *plan, const DqmcLattice *L, const char *sel)
{
    memset(plan, 0, sizeof *plan);
    if (!L || !sel || !sel[0]) return 1;
    for (const char *c = sel; *c; c++)
        if (isspace((unsigned char)*c)) return 1;
    if (!strcmp(sel, "none")) return 0;
    if (!L->has_coordinates || (L->type != 1 && L->type != 2) || L->n <= 0 ||
        L->Lx * L->Ly != L->n)
        return 1;
    plan->enabled = 1;
    plan->n = L->n;
    plan->Lx = L->Lx;
    plan->Ly = L->Ly;
    if (!strcmp(sel, "af")) {
        if ((L->Lx > 1 && L->Lx % 2) || (L->Ly > 1 && L->Ly % 2)) goto fail;
        plan->nq = 1;
        plan->mx = malloc(sizeof(int));
        plan->my = malloc(sizeof(int));
        plan->mx[0] = L->Lx > 1 ? L->Lx / 2 : 0;
        plan->my[0] = L->Ly > 1 ? L->Ly / 2 : 0;
    } else if (!strcmp(sel, "all")) {
        plan->is_all = 1;
        plan->nq = L->n;
        plan->mx = malloc(sizeof(int) * (size_t)L->n);
        plan->my = malloc(sizeof(int) * (size_t)L->n);
        int q = 0;
        for (int y = 0; y < L->Ly; y++)
            for (int x = 0; x < L->Lx; x++) {
                plan->mx[q] = x;
                plan->my[q] = y;
                q++;
            }
    } else {
        int nq = 1;
        for (const char *c = sel; *c; c++) nq += (*c == ',');
        plan->mx = malloc(sizeof(int) * (size_t)nq);
        plan->my = malloc(sizeof(int) * (size_t)nq);
        const char *p = sel;
        for (int q = 0; q < nq; q++) {
            char *end = NULL;
            errno = 0;
            long v = strtol(p, &end, 10);
            if (errno || end == p || v < 0 || v > INT_MAX || *end != ':') goto fail;
            plan->mx[q] = (int)v;
            p = end + 1;
            errno = 0;
            v = strtol(p, &end, 10);
            if (errno || end == p || v < 0 || v > INT_MAX) goto fail;
            plan->my[q] = (int)v;
            if ((q + 1 < nq && *end != ',') || (q + 1 == nq && *end != '\0')) goto fail;
            if (plan->mx[q] >= L->Lx || plan->my[q] >= L->Ly || (L->type == 1 && plan->my[q] != 0))
                goto fail;
            for (int r = 0; r < q; r++)
                if (plan->mx[r] == plan->mx[q] && plan->my[r] == plan->my[q]) goto fail;
            p = end + (q + 1 < nq ? 1 : 0);
        }
        plan->nq = nq;
    }
    return 0;
fail:
    dqmc_spin_plan_free(plan);
    return 1;
}

/* ------------------------------------------------- replica ownership */
void dqmc_replica_rank_range(int nrep, int nranks, int rank, int *first_replica,
                             int *local_nrep)
{
    int first = 0, count = 0;
    if (nrep >= 0 && nranks > 0 && rank >= 0 && rank < nranks) {
        const int base = nrep / nranks, rem = nrep % nranks;
        count = base + (rank < rem);
        first = rank * base + (rank < rem ? rank : rem);
    }
    if (first_replica) *first_replica = first;
    if (local_nrep) *local_nrep = count;
}

int dqmc_replica_rank_for_replica(int nrep, int nranks, int replica_id)
{
    if (nrep <= 0 || nranks <= 0 || replica_id < 0 || replica_id >= nrep) return -1;
    for (int r = 0; r < nranks; r++) {
        int first, count;
        dqmc_replica_rank_range(nrep, nranks, r, &first, &count);
        if (replica_id >= first && replica_id < first + count) return r;
    }
    return -1;
}

int dqmc_replica_gather_layout(int nrep, int nbin, int nranks, int item_width,
                               int *recvcounts, int *displs)
{
    if (!recvcounts || !displs || nrep < 0 || nranks <= 0 || nbin < 0 || item_width < 0)
        return 1;
    for (int r = 0; r < nranks; r++) {
        int first, count;
        dqmc_replica_rank_range(nrep, nranks, r, &first, &count);
        const long long per = (long long)nbin * item_width;
        const long long recv = per ? (long long)count * per : 0;
        const long long disp = per ? (long long)first * per : 0;
        if (recv > INT_MAX || disp > INT_MAX) return 1;
        recvcounts[r] = (int)recv;
        displs[r] = (int)disp;
    }
    return 0;
}

/* ------------------------------------------------------- bins, errors */
unsigned long long dqmc_replica_seed(unsigned long long base, int b, int r)
{
    const unsigned long long legacy = base + 1000ULL * (unsigned long long)b;
    if (r == 0) return legacy;
    uint64_t x = base;
    x ^= 0xD1B54A32D192ED03ULL * (uint64_t)(unsigned)(b + 1);
    x ^= 0xABC98388FB8FAC03ULL * (uint64_t)(unsigned)(r + 1);
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    if (z == legacy) {
        uint64_t y = z + 0x9E3779B97F4A7C15ULL;
        y = (y ^ (y >> 30)) * 0xBF58476D1CE4E5B9ULL;
        y = (y ^ (y >> 27)) * 0x94D049BB133111EBULL;
        z = y ^ (y >> 31);
    }
    return z;
}

void dqmc_jackknife(const double *x, int N, double *mean, double *err)
{
    double sum = 0.0;
    for (int i = 0; i < N; i++) sum += x[i];
    const double mu = N > 0 ? sum / (double)N : 0.0;
    *mean = mu;
    if (N < 2) {
        *err = 0.0;
        return;
    }
    double var = 0.0;
    for (int i = 0; i < N; i++) {
        const double d = (sum - x[i]) / (double)(N - 1) - mu;
        var += d * d;
    }
    *err = sqrt(var * (double)(N - 1) / (double)N);
}

int dqmc_bin_values(const double *b, double *out)
{
    const double count = b[DQMC_BIN_COUNT_F], ss = b[DQMC_BIN_SUM_SIGN];
    for (int k = 0; k < 6; k++)
        if (!isfinite(b[k])) return 1;
    if (count <= 0.0 || !isfinite(ss) || fabs(ss) == 0.0) return 1;
    out[0] = b[DQMC_BIN_SUM_SIGN_EHUB] / ss;
    out[1] = b[DQMC_BIN_SUM_SIGN_EGC] / ss;
    out[2] = b[DQMC_BIN_SUM_SIGN_EPH] / ss;
    out[3] = b[DQMC_BIN_SUM_SIGN_N] / ss;
    out[4] = b[DQMC_BIN_SUM_SIGN_D] / ss;
    out[5] = ss / count;
    for (int k = 0; k < 6; k++)
        if (!isfinite(out[k])) return 1;
    return 0;
}

int dqmc_sum_rule(const DqmcSpinPlan *plan, const double *v, double ntot, double doublon,
                  double prefactor, double *lhs_out, double *rhs_out)
{
    if (!plan || !plan->is_all) return 0;
    if (!plan->enabled || !v || plan->nq != plan->n || !isfinite(ntot) || !isfinite(doublon))
        return 1;
    const double rhs = prefactor * (ntot - 2.0 * (double)plan->n * doublon);
    const double tol = 1e-12 + 1e-10 * fmax(1.0, fabs(rhs));
    double lhs = 0.0;
    for (int q = 0; q < plan->nq; q++) {
        if (!isfinite(v[q])) return 1;
        lhs += v[q];
    }
    if (lhs_out) *lhs_out = lhs;
    if (rhs_out) *rhs_out = rhs;
    return (!isfinite(lhs - rhs) || fabs(lhs - rhs) > tol) ? 1 : 0;
}

int dqmc_format_row(char *buf, size_t len, double T, const double *Ehub, const double *Egc,
                    const double *Eph, const double *N, const double *D, const double *S,
                    const double *Acc, int nb)
{
    double m[7], e[7];
    const double *series[7] = {Ehub, Egc, Eph, N, D, S, Acc};
    for (int k = 0; k < 7; k++) {
        for (int i = 0; i < nb; i++)
            if (!isfinite(series[k][i])) return 1;
        dqmc_jackknife(series[k], nb, &m[k], &e[k]);
        if (!isfinite(m[k]) || !isfinite(e[k])) return 1;
    }
    /* src/main.c:259-262 */
    snprintf(buf, len,
             "%.6g %.8g %.3g %.8g %.3g %.8g %.3g %.6g %.2g %.8g %.2g %.6g %.8g %.3g\n", T, m[0],
             e[0], m[1], e[1], m[2], e[2], m[3], e[3], m[4], e[4], m[5], m[6], e[6]);
    return 0;
}
