/* Device-side data layout shared by the host engine and the kernels.
 *
 * Every matrix is n x n, column-major, leading dimension n (the reference's
 * layout, linalg.h:4).  One chain's device state lives in one contiguous
 * arena (see dqmc_engine.cu, chain_arena_layout) so a chain is one pointer
 * plus offsets; chains of different (n, L) coexist in one launch.
 */
#pragma once
#include <stdint.h>

#define DQMC_NT 256          /* threads per CTA; one CTA owns one chain   */
#define DQMC_MAX_N 1024      /* largest lattice the kernels are laid out for */
#define DQMC_MAX_KB 32       /* largest site block of the delayed update (one lane per column) */
#define DQMC_QNB 16          /* Householder panel width                     */

/* status bits (per chain, sticky; a chain with status != 0 is frozen)     */
#define DQMC_ST_NONFINITE 1  /* non-finite value in a factor or in G        */
#define DQMC_ST_SINGULAR 2   /* zero pivot in a QR                          */
#define DQMC_ST_LOGRANGE 4   /* log-scale D left the representable range   */
#define DQMC_ST_DETSIGN 8    /* det sign came out 0                         */
#define DQMC_ST_TIMEOUT 16   /* a bounded wait on the tensor-core pipeline ran out */

/* per-bin scalar accumulators (replica.h:6-16 ReplicaBin order)           */
enum {
    DQMC_BIN_EHUB = 0,
    DQMC_BIN_EGC,
    DQMC_BIN_EPH,
    DQMC_BIN_N,
    DQMC_BIN_D,
    DQMC_BIN_SIGN,
    DQMC_BIN_COUNT,
    DQMC_BIN_ACCEPTED,
    DQMC_BIN_ATTEMPTS,
    DQMC_BIN_FIELDS
};

/* phase timers (SM clock cycles, thread 0, phases are barrier-separated) */
enum {
    DQMC_PH_BCACHE = 0,   /* B-block products for the suffix stack (first sweep) */
    DQMC_PH_STACK,        /* suffix stack rmuls                                  */
    DQMC_PH_PROPOSE,      /* site-block proposals (warp 0) incl. block loads     */
    DQMC_PH_FLUSH,        /* rank-m flush of the accepted block                  */
    DQMC_PH_WRAP,         /* G <- B G B^-1                                       */
    DQMC_PH_BBLOCK,       /* left B-block products                               */
    DQMC_PH_LMUL,         /* left UDV update                                     */
    DQMC_PH_COMBINE,      /* left x suffix                                       */
    DQMC_PH_GREEN,        /* (1 + UDT)^-1                                        */
    DQMC_PH_SDRIFT,       /* reference drift rebuild (opt-in)                    */
    DQMC_PH_ADOPT,        /* drift + copy of the stabilized G                    */
    DQMC_PH_MEASURE,      /* fused measurement                                   */
    DQMC_PH_COUNT
};

/* int8 digits per operand of a split product (balanced base-256 digits,
 * 8 S - 2 = 62 bits of each line's fixed-point representation) */
#ifndef DQMC_MIX_DIGITS
#define DQMC_MIX_DIGITS 8
#endif
/* pipeline stages of the split GEMM (shared memory: stages x digits x
 * (128 + 128) lines x 32 bytes) */
#ifndef DQMC_SPL_STAGES
#define DQMC_SPL_STAGES 3
#endif

/* A split operand in device memory (dqmc_split.cuh): tiles (line block,
 * k chunk) of DQMC_MIX_DIGITS digit slices in the tensor core's canonical
 * layout, and one power-of-two scale per line. */
typedef struct {
    signed char *t;
    double *sc;
    int nlb, nkc;
} DqmcSplitDev;

typedef struct {
    int n, Lx, Ly;
    double U, dtau, mu;
    double expv[2];     /* exp(+lambda*s - dtau*U/2) for s = -1, +1 (green.c:63-67) */
    double expvinv[2];  /* 1/expv                                           */
    /* the same for sigma = -1 (G_down of the two-spin path, green.c:63-67) */
    double expvd[2], expvinvd[2];
    int ph;             /* 1: particle-hole path (G_down mapped from G_up)  */
    double Nup[2];      /* N_cache[sigma=+1][s] = exp(-2 lambda s) - 1 (field.c:11-17) */
    double Ndn[2];      /* N_cache[sigma=-1][s] = exp(+2 lambda s) - 1      */
    const double *expK, *expKinv, *thop;
    const int *bipart;
    int nq_zz, nq_perp;
    const double *cos_zz, *cos_perp;   /* n x nq phase tables (structure_factor.c:182-199) */
    /* split-product (mixed precision) operands, precomputed per model:
     * expK and expK^-1 by rows (A operands, 128-line blocks) and by
     * columns (B operands, 64-line blocks) */
    DqmcSplitDev spK_r, spK_c, spKi_r, spKi_c;
} DqmcModelDev;

/* Command block of a chain advanced by a thread-block cluster: rank 0
 * writes the product the cluster forms next (op, operands, sizes, scalars);
 * the other ranks read it after the cluster barrier. */
typedef struct {
    int op, i[3];
    int err, pad;              /* a rank's bounded wait ran out during the command */
    const void *p[6];
    double d[4];
} DqmcClCmd;

/* largest cluster that advances one chain (non-portable size above 8)     */
#define DQMC_MAX_CHAIN_CTAS 16
/* per-chain global staging for the other ranks of a chain's cluster: a site
 * block's flush operands (four DQMC_MAX_KB x (DQMC_MAX_KB + 2) blocks, the
 * DQMC_MAX_KB factors and the accepted list), then the pre-pivot's column
 * norms (DQMC_MAX_N), then each rank's reflector count and flags of a QR
 * factorization (two ints per rank)                                      */
#define DQMC_CL_FLUSH_DOUBLES (4 * DQMC_MAX_KB * (DQMC_MAX_KB + 2) + 2 * DQMC_MAX_KB)
#define DQMC_CL_STAGE_DOUBLES (DQMC_CL_FLUSH_DOUBLES + DQMC_MAX_N + DQMC_MAX_CHAIN_CTAS)

typedef struct {
    int model, n, L, stab, M, kb;
    int status, bvalid;        /* bvalid: cached B-block products are current */
    /* alternating sweep order: direction of the next sweep (0 forward, 1
     * backward) and whether the prefix stack P (after a forward sweep) or
     * the suffix stack S (after a backward sweep) carries over */
    int alt, dir, pvalid, svalid;
    int rebuild;               /* 0: combine, 1: two-sided G at boundaries */
    int pair;                  /* flush G after every second site block   */
    int ns;                    /* evolved spins: 1 (PH path) or 2 (G_up, G_down) */
    /* UDV scale records (opt-in): DQMC_UDV_RECORD_DOUBLES each, udv_n of
     * udv_cap used since the host last drained them, udv_lost dropped */
    int udv_cap, udv_n, udv_lost;
    double *udvrec;
    double sign;
    unsigned long long attempts, accepted, sweeps;
    unsigned long long meas_accepted, meas_attempts;  /* counters at last measurement */
    uint64_t rng[4];
    /* drift: max|G_wrapped - G_stabilized| over stabilization points       */
    double drift_max, drift_sum;
    unsigned long long drift_count;
    /* reference-style drift (rebuild from scratch), opt-in                 */
    double sdrift_max, sdrift_sum;
    unsigned long long sdrift_count, sdrift_max_sweep;
    int sdrift_max_tau;
    /* arena pointers */
    signed char *field;        /* L x n */
    double *G;                 /* n x n */
    double *S;                 /* (M+1) UDV slots */
    double *P;                 /* (M+1) UDV slots, prefix stack (alternating) */
    double *left, *comb, *scr; /* UDV slots (scr: rebuilds from scratch) */
    double *bcache;            /* M x n x n block products B(b_{j+1}, b_j) */
    double *w[6];              /* n x n scratch */
    double *Zs, *Ys;           /* n x 2kb / 2kb x n flush operands (two blocks) */
    /* G_down's own state on the two-spin path (else null) */
    double *Gd, *Sd, *leftd, *combd, *bcached, *Zsd, *Ysd;
    double *twall;             /* n x QNB compact-WY factors of the last QR */
    double *bins;              /* nbin x DQMC_BIN_FIELDS */
    double *bins_zz, *bins_perp;   /* nbin x nq */
    int nbin;
    /* mixed precision: the per-chain split buffers of an A operand (128-line
     * blocks) and a B operand (64-line blocks) with K <= n; null in FP64 */
    DqmcSplitDev spA, spB;
    /* G as wrapped, before each rebuild (opt-in diagnostic): up to glog_cap
     * snapshots of n x n, glog_n taken since the host last drained them */
    double *glog;
    int glog_cap, glog_n, glog_lost, glog_pad;
    unsigned long long prof[DQMC_PH_COUNT];
    /* calls of each phase's region as the reference's profiler counts them
     * (src/profiler.c): wraps, accepted flips and G updates, stack builds,
     * B-block products, UDV updates, combines, G from UDV, adoptions,
     * rebuilds from scratch, measurements */
    unsigned long long pcalls[DQMC_PH_COUNT];
    DqmcClCmd cl;
    double *clstage;           /* DQMC_CL_STAGE_DOUBLES */
} DqmcChainDev;

/* UDV slot: U (n*n) | T (n*n) | ell = log D (n) | detU (1) | pad (1)        */
/* UDV slot: U (n x n) | T (n x n) | log D (n) | sign det U | pad | column
 * permutation of an rmul factor, T = R_unit P^T (n, stored as doubles) */
#define DQMC_UDV_SIZE(n) (2 * (size_t)(n) * (n) + 2 * (size_t)(n) + 2)
