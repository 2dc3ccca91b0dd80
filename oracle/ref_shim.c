/*
 * Test-only shim over the UNMODIFIED SAI-QMC reference engine.
 *
 * This file is test infrastructure: it is compiled together with the
 * reference's own src/*.c (minus main.c) into oracle/_ref/libdqmcref.so by
 * oracle/build.py, and only tests/, tests/golden/make_golden.py and the CPU
 * baseline use it.  It adds no algorithm of its own; every entry point calls
 * the reference functions named beside it so that golden vectors can be
 * produced from the reference itself:
 *
 *   ref_chain_new      lattice_chain/lattice_square (lattice.c:26-82),
 *                      model_init (model.c:8-31), rng_seed (rng.c:17-22),
 *                      field_init (field.c:6-24), dqmc_init_modes
 *                      (dqmc.c:418-483)
 *   ref_chain_new_mode the same with sweep_order and green_rebuild
 *   ref_chain_new_mu   the same with model_init's half/mu arguments and the
 *                      ph_symmetric = 0 override of tests/test_dqmc_stack.c:81
 *                      (the reference's two-spin path, dqmc.c:418-483)
 *   ref_chain_sweep    dqmc_sweep (dqmc.c:952-963)
 *   ref_chain_measure  measure_sample (measure.c:6-39) and
 *                      measure_szz_sperp_sample (structure_factor.c:328-400)
 *   ref_green_scratch  green_from_scratch (green.c:262-306)
 *   ref_udv_inv        udv_inv_one_plus_work (linalg.c:911-1115)
 *   ref_expm_sym       la_expm_sym (linalg.c:319-346)
 */
#include "dqmc.h"
#include "field.h"
#include "green.h"
#include "lattice.h"
#include "linalg.h"
#include "measure.h"
#include "model.h"
#include "replica.h"
#include "rng.h"
#include "structure_factor.h"

#include <stdlib.h>
#include <string.h>

typedef struct {
    Lattice lat;
    Model m;
    Rng r;
    Field f;
    Dqmc D;
    int stab;
} RefChain;

void *ref_chain_new_mode(int kind, int Lx, int Ly, int pbc, double t, double U,
                         double dtau, int L, int stab, unsigned long long seed,
                         const signed char *field, int enable_drift, int sweep_mode,
                         int rebuild_mode);

void *ref_chain_new(int kind, int Lx, int Ly, int pbc, double t, double U,
                    double dtau, int L, int stab, unsigned long long seed,
                    const signed char *field, int enable_drift)
{
    return ref_chain_new_mode(kind, Lx, Ly, pbc, t, U, dtau, L, stab, seed, field,
                              enable_drift, 0, 0);
}

/* As ref_chain_new with the reference's sweep order (DqmcSweepMode:
 * 0 forward, 1 alternating forward/backward, dqmc.h:45-48) and G rebuild
 * (GreenRebuildMode: 0 combine, 1 two-sided, 2 centered, green.h). */
void *ref_chain_new_mode(int kind, int Lx, int Ly, int pbc, double t, double U,
                         double dtau, int L, int stab, unsigned long long seed,
                         const signed char *field, int enable_drift, int sweep_mode,
                         int rebuild_mode)
{
    RefChain *c = calloc(1, sizeof(RefChain));
    if (c == NULL) {
        return NULL;
    }
    if (kind == 0) {
        lattice_chain(&c->lat, Lx, t, pbc);
    } else {
        lattice_square(&c->lat, Lx, Ly, t, pbc);
    }
    model_init(&c->m, &c->lat, U, dtau, 1, 0.0);
    rng_seed(&c->r, seed);
    field_init(&c->f, c->lat.n, L, U, dtau, &c->r);
    if (field != NULL) {
        memcpy(c->f.s, field, (size_t)L * (size_t)c->lat.n);
    }
    c->stab = stab;
    if (dqmc_init_modes(&c->D, &c->m, &c->f, &c->r, stab, NULL,
                        sweep_mode ? DQMC_SWEEP_ALTERNATING : DQMC_SWEEP_FORWARD,
                        rebuild_mode == 1   ? GREEN_REBUILD_TWO_SIDED
                        : rebuild_mode == 2 ? GREEN_REBUILD_CENTERED
                                            : GREEN_REBUILD_COMBINE) != 0) {
        c->D.status = 1;
    }
    if (enable_drift) {
        dqmc_enable_stab_drift(&c->D, 1);
    }
    return c;
}

/* As ref_chain_new on a model_init(half, mu) model; force_two_spin sets
 * ph_symmetric = 0 before dqmc_init so the two-spin path runs even at the
 * particle-hole point. */
void *ref_chain_new_mu(int kind, int Lx, int Ly, int pbc, double t, double U, double dtau,
                       int L, int stab, unsigned long long seed, int half, double mu,
                       int force_two_spin)
{
    RefChain *c = calloc(1, sizeof(RefChain));
    if (c == NULL) {
        return NULL;
    }
    if (kind == 0) {
        lattice_chain(&c->lat, Lx, t, pbc);
    } else {
        lattice_square(&c->lat, Lx, Ly, t, pbc);
    }
    model_init(&c->m, &c->lat, U, dtau, half, mu);
    if (force_two_spin) {
        c->m.ph_symmetric = 0;
    }
    rng_seed(&c->r, seed);
    field_init(&c->f, c->lat.n, L, U, dtau, &c->r);
    c->stab = stab;
    dqmc_init(&c->D, &c->m, &c->f, &c->r, stab, NULL);
    return c;
}

int ref_chain_n(void *h) { return ((RefChain *)h)->lat.n; }

void ref_chain_model(void *h, double *expK, double *expKinv, double *thop,
                     int *bipart)
{
    RefChain *c = h;
    const size_t nn = (size_t)c->lat.n * (size_t)c->lat.n;
    if (expK) memcpy(expK, c->m.expK, nn * sizeof(double));
    if (expKinv) memcpy(expKinv, c->m.expKinv, nn * sizeof(double));
    if (thop) memcpy(thop, c->lat.t, nn * sizeof(double));
    if (bipart) memcpy(bipart, c->lat.bipart, (size_t)c->lat.n * sizeof(int));
}

int ref_chain_sweep(void *h, int nsweeps)
{
    RefChain *c = h;
    for (int s = 0; s < nsweeps; s++) {
        dqmc_sweep(&c->D);
    }
    return c->D.status;
}

void ref_chain_state(void *h, double *Gu, double *Gd, signed char *field,
                     unsigned long long *counters, double *sign, int *status,
                     unsigned long long *rng_state)
{
    RefChain *c = h;
    const int n = c->lat.n;
    const size_t nn = (size_t)n * (size_t)n;
    if (Gu) memcpy(Gu, c->D.Gu.g, nn * sizeof(double));
    if (Gd) memcpy(Gd, c->D.Gd.g, nn * sizeof(double));
    if (field) memcpy(field, c->f.s, (size_t)c->f.L * (size_t)n);
    if (counters) {
        counters[0] = c->D.accept_attempts;
        counters[1] = c->D.accept_accepted;
        counters[2] = c->D.sweep_count;
    }
    if (sign) *sign = c->D.sign;
    if (status) *status = c->D.status;
    if (rng_state) {
        for (int i = 0; i < 4; i++) rng_state[i] = c->r.s[i];
    }
}

void ref_chain_drift(void *h, double *out)
{
    RefChain *c = h;
    out[0] = (double)c->D.stab_drift.samples;
    out[1] = c->D.stab_drift.max_inf;
    out[2] = c->D.stab_drift.sum_inf;
    out[3] = (double)c->D.stab_drift.max_tau;
    out[4] = (double)c->D.stab_drift.failed;
}

/* out = {E, ekin, eint, ntot, doublon}; szz/sperp may be NULL. */
int ref_chain_measure(void *h, double *out, const char *selector,
                      double *szz, double *sperp)
{
    RefChain *c = h;
    MeasSample s =
        measure_sample(c->lat.n, c->lat.t, c->m.U, c->D.Gu.g, c->D.Gd.g);
    out[0] = s.E;
    out[1] = s.ekin;
    out[2] = s.eint;
    out[3] = s.ntot;
    out[4] = s.doublon;
    if (selector == NULL || szz == NULL || sperp == NULL) {
        return 0;
    }
    StructureFactorPlan plan;
    if (structure_factor_plan_init(&plan, &c->lat, selector) != 0) {
        return 1;
    }
    StructureFactorWorkspace w1, w2;
    structure_factor_workspace_init(&w1, &plan);
    structure_factor_workspace_init(&w2, &plan);
    const int rc = measure_szz_sperp_sample(&plan, &w1, szz, &plan, &w2,
                                            sperp, c->D.Gu.g, c->D.Gd.g);
    structure_factor_workspace_free(&w1);
    structure_factor_workspace_free(&w2);
    structure_factor_plan_free(&plan);
    return rc;
}

int ref_green_scratch(void *h, int l0, double *G, int *det_sign)
{
    RefChain *c = h;
    Green g;
    green_alloc(&g, &c->m, &c->f, 1.0);
    const int rc = green_from_scratch(&g, l0);
    memcpy(G, g.g, (size_t)c->lat.n * (size_t)c->lat.n * sizeof(double));
    *det_sign = g.det_sign;
    green_free(&g);
    return rc;
}

/* One forward wrap G <- B_l G B_l^{-1} of an arbitrary G at slice l. */
void ref_wrap(void *h, int l, double *G)
{
    RefChain *c = h;
    Green g;
    green_alloc(&g, &c->m, &c->f, 1.0);
    memcpy(g.g, G, (size_t)c->lat.n * (size_t)c->lat.n * sizeof(double));
    g.cur_l = l;
    green_wrap(&g);
    memcpy(G, g.g, (size_t)c->lat.n * (size_t)c->lat.n * sizeof(double));
    green_free(&g);
}

void ref_chain_free(void *h)
{
    RefChain *c = h;
    if (c == NULL) return;
    dqmc_free(&c->D);
    field_free(&c->f);
    model_free(&c->m);
    lattice_free(&c->lat);
    free(c);
}

int ref_udv_inv(int n, const double *U, const double *D, const double *T,
                double log_offset, double *G, int *det_sign)
{
    UDV s;
    udv_init(&s, n);
    memcpy(s.U, U, (size_t)n * (size_t)n * sizeof(double));
    memcpy(s.D, D, (size_t)n * sizeof(double));
    memcpy(s.T, T, (size_t)n * (size_t)n * sizeof(double));
    s.log_offset = log_offset;
    LinalgWork w;
    linalg_work_init(&w, n);
    const int rc = udv_inv_one_plus_work(&s, G, det_sign, &w);
    linalg_work_free(&w);
    udv_free(&s);
    return rc;
}

int ref_udv_recenter(int n, double *D, double *log_offset)
{
    UDV s;
    udv_init(&s, n);
    memcpy(s.D, D, (size_t)n * sizeof(double));
    s.log_offset = *log_offset;
    const int rc = udv_recenter(&s, 8.0, NULL, NULL);
    memcpy(D, s.D, (size_t)n * sizeof(double));
    *log_offset = s.log_offset;
    udv_free(&s);
    return rc;
}

void ref_expm_sym(int n, const double *A, double scale, double *out)
{
    la_expm_sym(n, A, scale, out);
}

unsigned long long ref_replica_seed(unsigned long long base, int b, int r)
{
    return replica_seed(base, b, r);
}

void ref_jackknife(const double *x, int N, double *mean, double *err)
{
    jackknife(x, N, mean, err);
}

double ref_rng_first(unsigned long long seed, int k, double *out)
{
    Rng r;
    rng_seed(&r, seed);
    for (int i = 0; i < k; i++) out[i] = rng_double(&r);
    return out[0];
}
