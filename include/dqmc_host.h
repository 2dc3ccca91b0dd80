/*
 * dqmc_host.h -- host side of the dqmc_gpu driver (libdqmc_b200.so).
 *
 * Mirrors the reference program's outer boundary so an input file of the
 * reference runs unchanged: the key=value parser (SAI-QMC src/io.c), the
 * lattices (src/lattice.c), the spin structure-factor plans
 * (src/structure_factor.c:107-206), replica seeds (src/replica.c:17-34),
 * per-bin ratios and jackknife (src/replica.c:88-120, src/measure.c:48-69),
 * the sum rules (src/structure_factor.c:447-510) and the output formats of
 * src/main.c:221-377, 892-1023.  None of these calls needs a GPU except
 * dqmc_host_run, which drives the engine of dqmc_gpu.h.
 */
#ifndef DQMC_HOST_H
#define DQMC_HOST_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DQMC_MAX_BETA 64
#define DQMC_MAX_GPUS 16

/* Params of src/io.h:4-38 plus the engine's own keys. */
typedef struct {
    char lattice[16];
    char latfile[256];
    int Lx, Ly, pbc;
    double thop, U, dtau;
    double beta_list[DQMC_MAX_BETA];
    int nbeta;
    int nwarm, nmeas, nbin, stab_interval;
    char output_file[256];
    int profile;
    char profile_file[256];
    char stab_drift_file[256];
    char udv_scale_file[256];
    char udv_centered_file[256];
    char sweep_order[16];
    char green_rebuild[16];
    char parallel[16];
    int nrep;
    char replica_log[256];
    char szz_q[256];
    char szz_file[256];
    char sperp_q[256];
    char sperp_file[256];
    char spin_consistency_file[256];
    unsigned long long seed;
    /* engine keys (not in the reference): */
    int delay_rank;       /* delay_rank=k, site-block size (0 = default) */
    char precision[16];   /* precision=fp64|mixed                        */
    int gpu_device;       /* gpu_device=ordinal                          */
    int gpu_devices[DQMC_MAX_GPUS];  /* gpu_devices=0,1,...: replicas of each
                                        beta split over these devices      */
    int ngpu;             /* entries in gpu_devices (0: gpu_device alone) */
} DqmcParams;

/* params_read (src/io.c:156-418): 0 ok, 1 error (message on stderr). */
int dqmc_params_read(DqmcParams *p, const char *path);

typedef struct {
    int n, Lx, Ly, type; /* type: 1 chain, 2 square, 3 file */
    int has_coordinates, is_bipartite;
    double *t;           /* n x n column-major */
    int *bipart;
} DqmcLattice;

int dqmc_lattice_chain(DqmcLattice *L, int Lx, double t, int pbc);
int dqmc_lattice_square(DqmcLattice *L, int Lx, int Ly, double t, int pbc);
int dqmc_lattice_file(DqmcLattice *L, const char *path);
int dqmc_lattice_dump(const DqmcLattice *L, const char *path);
void dqmc_lattice_free(DqmcLattice *L);

typedef struct {
    int enabled, is_all, n, Lx, Ly, nq;
    int *mx, *my;
} DqmcSpinPlan;

/* structure_factor_plan_init selectors: none / af / all / "mx:my,...". */
int dqmc_spin_plan(DqmcSpinPlan *plan, const DqmcLattice *L, const char *selector);
void dqmc_spin_plan_free(DqmcSpinPlan *plan);

unsigned long long dqmc_replica_seed(unsigned long long base, int beta_index,
                                     int replica_id);
void dqmc_jackknife(const double *x, int N, double *mean, double *err);

/* Replica ownership across devices or ranks, as the reference's MPI runner
 * splits the nrep replicas of each beta (src/replica_mpi.c:13-89): rank r
 * owns the contiguous range [first, first + count), the first nrep % nranks
 * ranks one replica more.  rank_for_replica returns the owner (-1 if out of
 * range); gather_layout fills per-rank element counts and displacements of
 * a replica-major (replica, bin, item) gather, 0 ok, 1 on bad arguments or
 * int overflow. */
void dqmc_replica_rank_range(int nrep, int nranks, int rank, int *first_replica,
                             int *local_nrep);
int dqmc_replica_rank_for_replica(int nrep, int nranks, int replica_id);
int dqmc_replica_gather_layout(int nrep, int nbin, int nranks, int item_width,
                               int *recvcounts, int *displs);

/* replica_bin_values (src/replica.c:88-120) on one bin of
 * dqmc_read_bins' scalar layout; out = {Ehub, Egc, Eph, N, D, sign}. */
int dqmc_bin_values(const double *bin_fields, double *out);

/* sum_rule_check (src/structure_factor.c:447-510): prefactor 0.25 (Szz) or
 * 0.5 (Sperp); returns 0 when |sum_q S(q) - rhs| <= tolerance. */
int dqmc_sum_rule(const DqmcSpinPlan *plan, const double *values, double ntot,
                  double doublon, double prefactor, double *lhs, double *rhs);

/* One 14-column observables row (src/main.c:221-265) from the bin series. */
int dqmc_format_row(char *buf, size_t len, double T, const double *Ehub,
                    const double *Egc, const double *Eph, const double *N,
                    const double *D, const double *S, const double *Acc,
                    int total_bins);

/* The whole dqmc_gpu run for an input file (the reference's main()). */
int dqmc_host_run(const char *input_path);

#ifdef __cplusplus
}
#endif
#endif
