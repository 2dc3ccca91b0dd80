/*
 * CPU ORACLE -- test infrastructure, not product code.
 *
 * A plain-C restatement of the SAI-QMC reference's BSS-DQMC forward sweep
 * for the half-filled Hubbard model (particle-hole path, combine rebuild),
 * written from the reference's algorithm; each function names the reference
 * file:line it restates.  It has no dependency on BLAS/LAPACK: the LAPACK
 * routines the reference calls (dgeqrf/dorgqr, dgetrf/dgetri, dtrtri, dsyev)
 * are restated from their published algorithms (LAPACK 3.x dlarfg
 * Householder convention; partial-pivot LU; cyclic Jacobi for the symmetric
 * eigenproblem).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * this library, and only as the checker.  Parity of this restatement itself
 * is pinned in tests/test_oracle_*.py against golden vectors produced by the
 * unmodified reference (tests/golden/, made by tests/golden/make_golden.py)
 * and against the reference's own fixture files.
 *
 * Matrices are n x n column-major, A[i + j*n] (linalg.h:4).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- RNG -- */
/* rng.c:8-37: splitmix64 seeding of xoshiro256**, double = (x>>11)*2^-53 */
typedef struct { uint64_t s[4]; } ORng;

static uint64_t o_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t o_splitmix(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static void o_rng_seed(ORng *r, uint64_t seed)
{
    for (int i = 0; i < 4; i++) r->s[i] = o_splitmix(&seed);
}

static double o_rng_double(ORng *r)
{
    uint64_t *s = r->s;
    const uint64_t res = o_rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = o_rotl(s[3], 45);
    return (double)(res >> 11) * (1.0 / 9007199254740992.0);
}

void orc_rng(unsigned long long seed, int k, double *out)
{
    ORng r;
    o_rng_seed(&r, seed);
    for (int i = 0; i < k; i++) out[i] = o_rng_double(&r);
}

/* replica.c:9-34 */
static uint64_t o_mix(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

unsigned long long orc_replica_seed(unsigned long long base, int b, int r)
{
    const unsigned long long legacy = base + 1000ULL * (unsigned long long)b;
    if (r == 0) return legacy;
    uint64_t x = base;
    x ^= 0xD1B54A32D192ED03ULL * (uint64_t)(unsigned)(b + 1);
    x ^= 0xABC98388FB8FAC03ULL * (uint64_t)(unsigned)(r + 1);
    uint64_t m = o_mix(x);
    if (m == legacy) m = o_mix(m);
    return m;
}

/* measure.c:48-69 */
void orc_jackknife(const double *x, int N, double *mean, double *err)
{
    double sum = 0.0;
    for (int i = 0; i < N; i++) sum += x[i];
    const double mu = N > 0 ? sum / N : 0.0;
    *mean = mu;
    if (N < 2) { *err = 0.0; return; }
    double var = 0.0;
    for (int i = 0; i < N; i++) {
        const double d = (sum - x[i]) / (N - 1) - mu;
        var += d * d;
    }
    *err = sqrt(var * (N - 1) / N);
}

/* ------------------------------------------------------- dense kernels -- */
static void o_eye(int n, double *A)
{
    memset(A, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; i++) A[i + i * n] = 1.0;
}

/* C = op(A) op(B); ta/tb select transposes (dgemm semantics, alpha=1 beta=0) */
static void o_gemm(int n, int ta, int tb, const double *A, const double *B,
                   double *C)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) {
                const double a = ta ? A[k + i * n] : A[i + k * n];
                const double b = tb ? B[j + k * n] : B[k + j * n];
                s += a * b;
            }
            C[i + j * n] = s;
        }
}

static void o_matmul(int n, const double *A, const double *B, double *C)
{
    o_gemm(n, 0, 0, A, B, C);
}

/* Householder QR restating LAPACK dgeqrf (dlarfg convention, v(1)=1):
 * on exit R is in the upper triangle, v below it, tau[j] the scalar. */
static void o_geqrf(int n, double *A, double *tau)
{
    for (int j = 0; j < n; j++) {
        double *x = &A[j + j * n];
        const int m = n - j;
        double xnorm = 0.0;
        for (int i = 1; i < m; i++) xnorm = hypot(xnorm, x[i]);
        const double alpha = x[0];
        if (xnorm == 0.0) {
            tau[j] = 0.0;
            continue;
        }
        const double beta = -copysign(hypot(alpha, xnorm), alpha);
        tau[j] = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        for (int i = 1; i < m; i++) x[i] *= scal;
        x[0] = beta;
        for (int c = j + 1; c < n; c++) {
            double *y = &A[j + c * n];
            double w = y[0];
            for (int i = 1; i < m; i++) w += x[i] * y[i];
            w *= tau[j];
            y[0] -= w;
            for (int i = 1; i < m; i++) y[i] -= w * x[i];
        }
    }
}

/* LAPACK dorgqr restated: Q = H_1 H_2 ... H_n formed in place from the
 * reflectors stored below the diagonal of A. */
static void o_orgqr(int n, double *A, const double *tau)
{
    double *Q = malloc(sizeof(double) * (size_t)n * n);
    o_eye(n, Q);
    for (int j = n - 1; j >= 0; j--) {
        if (tau[j] == 0.0) continue;
        const double *v = &A[j + j * n];
        for (int c = j; c < n; c++) {
            double *y = &Q[j + c * n];
            double w = y[0];
            for (int i = 1; i < n - j; i++) w += v[i] * y[i];
            w *= tau[j];
            y[0] -= w;
            for (int i = 1; i < n - j; i++) y[i] -= w * v[i];
        }
    }
    memcpy(A, Q, sizeof(double) * (size_t)n * n);
    free(Q);
}

/* LU with partial pivoting restating dgetrf; returns info (0 ok). */
static int o_getrf(int n, double *A, int *piv)
{
    for (int j = 0; j < n; j++) {
        int p = j;
        double best = fabs(A[j + j * n]);
        for (int i = j + 1; i < n; i++)
            if (fabs(A[i + j * n]) > best) { best = fabs(A[i + j * n]); p = i; }
        piv[j] = p;
        if (A[p + j * n] == 0.0) return j + 1;
        if (p != j)
            for (int c = 0; c < n; c++) {
                const double t = A[j + c * n];
                A[j + c * n] = A[p + c * n];
                A[p + c * n] = t;
            }
        const double inv = 1.0 / A[j + j * n];
        for (int i = j + 1; i < n; i++) A[i + j * n] *= inv;
        for (int c = j + 1; c < n; c++) {
            const double a = A[j + c * n];
            if (a == 0.0) continue;
            for (int i = j + 1; i < n; i++) A[i + c * n] -= A[i + j * n] * a;
        }
    }
    return 0;
}

/* la_inverse_work (linalg.c:394-409) restated: getrf then solve A X = I. */
static int o_inverse(int n, const double *A, double *Ainv)
{
    double *LU = malloc(sizeof(double) * (size_t)n * n);
    int *piv = malloc(sizeof(int) * (size_t)n);
    memcpy(LU, A, sizeof(double) * (size_t)n * n);
    int info = o_getrf(n, LU, piv);
    if (info == 0) {
        o_eye(n, Ainv);
        for (int j = 0; j < n; j++)
            if (piv[j] != j)
                for (int c = 0; c < n; c++) {
                    const double t = Ainv[j + c * n];
                    Ainv[j + c * n] = Ainv[piv[j] + c * n];
                    Ainv[piv[j] + c * n] = t;
                }
        for (int c = 0; c < n; c++) {
            double *x = &Ainv[c * n];
            for (int i = 0; i < n; i++)
                for (int k = 0; k < i; k++) x[i] -= LU[i + k * n] * x[k];
            for (int i = n - 1; i >= 0; i--) {
                for (int k = i + 1; k < n; k++) x[i] -= LU[i + k * n] * x[k];
                x[i] /= LU[i + i * n];
            }
        }
    }
    free(LU);
    free(piv);
    return info;
}

/* la_logdet_work (linalg.c:287-317) restated: sign of det via getrf. */
static int o_logdet_sign(int n, const double *A, int *sign, double *logabs)
{
    double *LU = malloc(sizeof(double) * (size_t)n * n);
    int *piv = malloc(sizeof(int) * (size_t)n);
    memcpy(LU, A, sizeof(double) * (size_t)n * n);
    const int info = o_getrf(n, LU, piv);
    if (info == 0) {
        int s = 1;
        double la = 0.0;
        for (int i = 0; i < n; i++) {
            const double d = LU[i + i * n];
            if (d < 0.0) s = -s;
            la += log(fabs(d));
            if (piv[i] != i) s = -s;
        }
        *sign = s;
        *logabs = la;
    }
    free(LU);
    free(piv);
    return info;
}

/* dtrtri('U','U') restated: inverse of a unit upper-triangular matrix. */
static void o_trtri_unit_upper(int n, const double *T, double *X)
{
    o_eye(n, X);
    for (int j = 0; j < n; j++)
        for (int i = j - 1; i >= 0; i--) {
            double s = 0.0;
            for (int k = i + 1; k <= j; k++) s += T[i + k * n] * X[k + j * n];
            X[i + j * n] = -s;
        }
}

/* la_expm_sym (linalg.c:319-346) restated with a cyclic Jacobi eigensolver
 * in place of dsyev: expA = V diag(exp(scale*w)) V^T. */
void orc_expm_sym(int n, const double *A, double scale, double *out)
{
    double *a = malloc(sizeof(double) * (size_t)n * n);
    double *V = malloc(sizeof(double) * (size_t)n * n);
    memcpy(a, A, sizeof(double) * (size_t)n * n);
    o_eye(n, V);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < j; i++) off += a[i + j * n] * a[i + j * n];
        if (off < 1e-300) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = a[p + q * n];
                if (apq == 0.0) continue;
                const double theta = (a[q + q * n] - a[p + p * n]) / (2.0 * apq);
                const double t = copysign(1.0, theta) /
                                 (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {
                    const double akp = a[k + p * n], akq = a[k + q * n];
                    a[k + p * n] = c * akp - s * akq;
                    a[k + q * n] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    const double apk = a[p + k * n], aqk = a[q + k * n];
                    a[p + k * n] = c * apk - s * aqk;
                    a[q + k * n] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    const double vkp = V[k + p * n], vkq = V[k + q * n];
                    V[k + p * n] = c * vkp - s * vkq;
                    V[k + q * n] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int k = 0; k < n; k++)
                s += V[i + k * n] * exp(scale * a[k + k * n]) * V[j + k * n];
            out[i + j * n] = s;
        }
    free(a);
    free(V);
}

/* ------------------------------------------------------------- UDV ----- */
/* linalg.h:16-24; combine mode only (log_offset = 0). */
typedef struct { int n; double *U, *D, *T; } OUdv;

static void o_udv_init(OUdv *s, int n)
{
    s->n = n;
    s->U = malloc(sizeof(double) * (size_t)n * n);
    s->T = malloc(sizeof(double) * (size_t)n * n);
    s->D = malloc(sizeof(double) * (size_t)n);
    o_eye(n, s->U);
    o_eye(n, s->T);
    for (int i = 0; i < n; i++) s->D[i] = 1.0;
}

static void o_udv_identity(OUdv *s)
{
    o_eye(s->n, s->U);
    o_eye(s->n, s->T);
    for (int i = 0; i < s->n; i++) s->D[i] = 1.0;
}

static void o_udv_copy(OUdv *d, const OUdv *s)
{
    const size_t nn = (size_t)s->n * s->n;
    memcpy(d->U, s->U, nn * sizeof(double));
    memcpy(d->T, s->T, nn * sizeof(double));
    memcpy(d->D, s->D, (size_t)s->n * sizeof(double));
}

static void o_udv_free(OUdv *s)
{
    free(s->U);
    free(s->T);
    free(s->D);
}

static int o_finite(int m, const double *x)
{
    for (int i = 0; i < m; i++)
        if (!isfinite(x[i])) return 0;
    return 1;
}

/* QR of M in place; R -> out R (upper, zero below), Q -> M. */
static int o_qr_split(int n, double *M, double *R, double *tau)
{
    o_geqrf(n, M, tau);
    memset(R, 0, sizeof(double) * (size_t)n * n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) R[i + j * n] = M[i + j * n];
    o_orgqr(n, M, tau);
    for (int i = 0; i < n; i++)
        if (R[i + i * n] == 0.0) return 1;
    return !o_finite(n * n, M) || !o_finite(n * n, R);
}

/* udv_lmul_impl (linalg.c:515-642), non-centered: U D T <- B U D T. */
static int o_udv_lmul(OUdv *s, const double *B)
{
    const int n = s->n;
    const size_t nn = (size_t)n * n;
    double *M = malloc(nn * sizeof(double)), *R = malloc(nn * sizeof(double));
    double *Tn = malloc(nn * sizeof(double)), *tau = malloc(n * sizeof(double));
    o_matmul(n, B, s->U, M);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) M[i + j * n] *= s->D[j];
    int rc = o_qr_split(n, M, R, tau);
    memcpy(s->U, M, nn * sizeof(double));
    for (int i = 0; i < n; i++) s->D[i] = R[i + i * n];
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            R[i + j * n] = (i <= j) ? R[i + j * n] / s->D[i] : 0.0;
    o_matmul(n, R, s->T, Tn);
    memcpy(s->T, Tn, nn * sizeof(double));
    free(M); free(R); free(Tn); free(tau);
    return rc;
}

/* udv_rmul_impl (linalg.c:662-784), non-centered: U D T <- U D T B. */
static int o_udv_rmul(OUdv *s, const double *B)
{
    const int n = s->n;
    const size_t nn = (size_t)n * n;
    double *M = malloc(nn * sizeof(double)), *R = malloc(nn * sizeof(double));
    double *TP = malloc(nn * sizeof(double)), *Un = malloc(nn * sizeof(double));
    double *tau = malloc(n * sizeof(double));
    o_matmul(n, s->T, B, TP);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) M[i + j * n] = s->D[i] * TP[i + j * n];
    int rc = o_qr_split(n, M, R, tau);
    o_matmul(n, s->U, M, Un);
    memcpy(s->U, Un, nn * sizeof(double));
    for (int i = 0; i < n; i++) s->D[i] = R[i + i * n];
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            s->T[i + j * n] = (i <= j) ? R[i + j * n] / s->D[i] : 0.0;
    free(M); free(R); free(TP); free(Un); free(tau);
    return rc;
}

/* udv_combine (linalg.c:796-909): out = l * r. */
static int o_udv_combine(const OUdv *l, const OUdv *r, OUdv *out)
{
    const int n = l->n;
    const size_t nn = (size_t)n * n;
    double *TLUR = malloc(nn * sizeof(double)), *C = malloc(nn * sizeof(double));
    double *R = malloc(nn * sizeof(double)), *tau = malloc(n * sizeof(double));
    o_matmul(n, l->T, r->U, TLUR);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            C[i + j * n] = l->D[i] * TLUR[i + j * n] * r->D[j];
    int rc = o_qr_split(n, C, R, tau);
    o_matmul(n, l->U, C, out->U);
    for (int i = 0; i < n; i++) out->D[i] = R[i + i * n];
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            TLUR[i + j * n] = (i <= j) ? R[i + j * n] / out->D[i] : 0.0;
    o_matmul(n, TLUR, r->T, out->T);
    free(TLUR); free(C); free(R); free(tau);
    return rc;
}

/* udv_inv_one_plus_work (linalg.c:911-1115), non-centered branch:
 * g = (1 + U D T)^{-1} and sign det(1 + U D T). */
static int o_udv_inv_one_plus(const OUdv *s, double *g, int *det_sign)
{
    const int n = s->n;
    const size_t nn = (size_t)n * n;
    double *Db = malloc(n * sizeof(double)), *Ds = malloc(n * sizeof(double));
    double *Tinv = malloc(nn * sizeof(double)), *UT = malloc(nn * sizeof(double));
    double *M = malloc(nn * sizeof(double)), *Minv = malloc(nn * sizeof(double));
    double *tmp = malloc(nn * sizeof(double)), *gp = malloc(nn * sizeof(double));
    int rc = 0;
    *det_sign = 0;
    for (int i = 0; i < n; i++) {
        if (fabs(s->D[i]) > 1.0) { Db[i] = s->D[i]; Ds[i] = 1.0; }
        else { Db[i] = 1.0; Ds[i] = s->D[i]; }
    }
    o_trtri_unit_upper(n, s->T, Tinv);
    o_gemm(n, 1, 0, s->U, Tinv, UT);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) M[i + j * n] = UT[i + j * n] / Db[i];
    for (int i = 0; i < n; i++) M[i + i * n] += Ds[i];
    if (o_inverse(n, M, Minv) != 0) { rc = 1; goto out; }
    {
        int sgn = 1;
        for (int i = 0; i < n; i++)
            if (fabs(s->D[i]) > 1.0 && s->D[i] < 0.0) sgn = -sgn;
        int su = 0, sm = 0;
        double la = 0.0;
        if (o_logdet_sign(n, s->U, &su, &la) != 0 ||
            o_logdet_sign(n, M, &sm, &la) != 0) { rc = 1; goto out; }
        *det_sign = sgn * su * sm;
    }
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) tmp[i + j * n] = Minv[i + j * n] / Db[j];
    o_gemm(n, 0, 1, tmp, s->U, gp);
    o_matmul(n, Tinv, gp, g);
    if (!o_finite(n * n, g)) { rc = 1; *det_sign = 0; }
out:
    free(Db); free(Ds); free(Tinv); free(UT); free(M); free(Minv);
    free(tmp); free(gp);
    return rc;
}

int orc_udv_inv(int n, const double *U, const double *D, const double *T,
                double *G, int *det_sign)
{
    OUdv s;
    o_udv_init(&s, n);
    memcpy(s.U, U, sizeof(double) * (size_t)n * n);
    memcpy(s.T, T, sizeof(double) * (size_t)n * n);
    memcpy(s.D, D, sizeof(double) * (size_t)n);
    const int rc = o_udv_inv_one_plus(&s, G, det_sign);
    o_udv_free(&s);
    return rc;
}

/* ------------------------------------------------------------ chain ---- */
typedef struct {
    int n, L, stab, M, kind, Lx, Ly, cap;
    double U, dtau, lambda;
    double *thop, *expK, *expKinv;
    int *bipart;
    double N_cache[2][2];    /* field.c:11-17: [sigma<0?0:1][s<0?0:1] */
    double expv[2], expvinv[2];  /* green.c:63-67 for sigma=+1 */
    signed char *s;
    ORng rng;
    double *Gu, *Gd;
    int cur_l, det_sign, status;
    double sign;
    unsigned long long attempts, accepted, sweeps;
    int delay_count;
    double *dc, *dv;
    OUdv *S;   /* suffix stack, M+1 entries (green.h:51-64) */
    int *b;
    OUdv left, combined;
    int drift_on;
    double drift_max, drift_sum;
    unsigned long long drift_samples;
} OChain;

/* lattice.c:26-82 */
static void o_lattice(OChain *c, int pbc, double t)
{
    const int n = c->n;
    c->thop = calloc((size_t)n * n, sizeof(double));
    c->bipart = calloc((size_t)n, sizeof(int));
    const int Lx = c->Lx, Ly = c->Ly;
    for (int y = 0; y < Ly; y++)
        for (int x = 0; x < Lx; x++) {
            const int i = x + y * Lx;
            int nb[2] = {-1, -1};
            if (x + 1 < Lx) nb[0] = (x + 1) + y * Lx;
            else if (pbc && Lx > 1) nb[0] = 0 + y * Lx;
            if (c->kind == 1) {
                if (y + 1 < Ly) nb[1] = x + (y + 1) * Lx;
                else if (pbc && Ly > 1) nb[1] = x;
            }
            for (int k = 0; k < 2; k++)
                if (nb[k] >= 0) {
                    c->thop[i + nb[k] * n] += t;
                    c->thop[nb[k] + i * n] += t;
                }
            c->bipart[i] = ((x + y) % 2 == 0) ? 1 : -1;
        }
}

/* green.c:126-137: B_l = expK diag(expv[s_l]) */
static void o_build_B(const OChain *c, int l, double *out)
{
    const int n = c->n;
    for (int j = 0; j < n; j++) {
        const double d = c->expv[c->s[l * n + j] > 0];
        for (int i = 0; i < n; i++) out[i + j * n] = c->expK[i + j * n] * d;
    }
}

/* green.c:139-149: B_l^{-1} = diag(expvinv[s_l]) expKinv */
static void o_build_Binv(const OChain *c, int l, double *out)
{
    const int n = c->n;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            out[i + j * n] = c->expKinv[i + j * n] * c->expvinv[c->s[l * n + i] > 0];
}

/* green.c:151-166 */
static void o_build_Bblock(const OChain *c, int l0, int len, double *out)
{
    const int n = c->n;
    const size_t nn = (size_t)n * n;
    if (len <= 0) { o_eye(n, out); return; }
    double *B = malloc(nn * sizeof(double)), *tmp = malloc(nn * sizeof(double));
    o_build_B(c, l0, out);
    for (int p = 1; p < len; p++) {
        o_build_B(c, l0 + p, B);
        o_matmul(n, B, out, tmp);
        memcpy(out, tmp, nn * sizeof(double));
    }
    free(B);
    free(tmp);
}

/* green.c:262-306 (into an arbitrary buffer) */
static int o_green_scratch(const OChain *c, int l0, double *g, int *det_sign)
{
    const int n = c->n;
    double *B = malloc(sizeof(double) * (size_t)n * n);
    OUdv u;
    o_udv_init(&u, n);
    int rc = 0;
    for (int k = 0; k < c->L && rc == 0; k++) {
        o_build_B(c, (l0 + k) % c->L, B);
        rc = o_udv_lmul(&u, B);
    }
    if (rc == 0) rc = o_udv_inv_one_plus(&u, g, det_sign);
    else *det_sign = 0;
    o_udv_free(&u);
    free(B);
    return rc;
}

/* green.c:372-382 via dqmc.c:9-17 */
static void o_map_ph(OChain *c)
{
    const int n = c->n;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            c->Gd[i + j * n] = (i == j ? 1.0 : 0.0) -
                               (double)(c->bipart[i] * c->bipart[j]) * c->Gu[j + i * n];
}

/* green.c:462-475: g -= C V^T */
static void o_delay_flush(OChain *c)
{
    const int n = c->n;
    if (c->delay_count == 0) return;
    for (int col = 0; col < n; col++)
        for (int row = 0; row < n; row++) {
            double s = 0.0;
            for (int p = 0; p < c->delay_count; p++)
                s += c->dc[row + p * n] * c->dv[col + p * n];
            c->Gu[row + col * n] -= s;
        }
    c->delay_count = 0;
}

/* green.c:384-392 */
static double o_delay_diag(const OChain *c, int i)
{
    const int n = c->n;
    double g = c->Gu[i + i * n];
    for (int p = 0; p < c->delay_count; p++) g -= c->dc[i + p * n] * c->dv[i + p * n];
    return g;
}

/* green.c:418-460 */
static void o_delay_accept(OChain *c, int i, double N)
{
    const int n = c->n;
    if (c->delay_count >= c->cap) o_delay_flush(c);
    const double denom = 1.0 + (1.0 - o_delay_diag(c, i)) * N;
    const double fac = N / denom;
    const int p = c->delay_count;
    double *u = &c->dc[p * n], *v = &c->dv[p * n];
    for (int j = 0; j < n; j++) {
        double gij = c->Gu[j + i * n];
        for (int q = 0; q < p; q++) gij -= c->dc[j + q * n] * c->dv[i + q * n];
        u[j] = (i == j ? 1.0 : 0.0) - gij;
    }
    for (int k = 0; k < n; k++) {
        double gik = c->Gu[i + k * n];
        for (int q = 0; q < p; q++) gik -= c->dc[i + q * n] * c->dv[k + q * n];
        v[k] = gik;
    }
    for (int j = 0; j < n; j++) u[j] *= fac;
    c->delay_count++;
    if (c->delay_count == c->cap) o_delay_flush(c);
}

/* green.c:509-527 */
static void o_wrap_g(const OChain *c, int l, double *g)
{
    const int n = c->n;
    const size_t nn = (size_t)n * n;
    double *B = malloc(nn * sizeof(double)), *Bi = malloc(nn * sizeof(double));
    double *tmp = malloc(nn * sizeof(double));
    o_build_B(c, l, B);
    o_build_Binv(c, l, Bi);
    o_matmul(n, B, g, tmp);
    o_matmul(n, tmp, Bi, g);
    free(B); free(Bi); free(tmp);
}

static void o_wrap(OChain *c)
{
    o_delay_flush(c);
    o_wrap_g(c, c->cur_l, c->Gu);
    c->cur_l = (c->cur_l + 1) % c->L;
}

/* dqmc.c:64-98 (up spin only: the PH path) */
static int o_drift(OChain *c, int tau)
{
    if (!c->drift_on) return 0;
    const int n = c->n;
    double *gr = malloc(sizeof(double) * (size_t)n * n);
    int ds = 0;
    const int rc = o_green_scratch(c, tau, gr, &ds);
    double m = 0.0;
    for (int i = 0; i < n * n; i++) m = fmax(m, fabs(c->Gu[i] - gr[i]));
    free(gr);
    if (rc != 0 || ds == 0) return 1;
    c->drift_samples++;
    c->drift_sum += m;
    if (m > c->drift_max || c->drift_samples == 1) c->drift_max = m;
    return 0;
}

void *orc_chain_new(int kind, int Lx, int Ly, int pbc, double t, double U,
                    double dtau, int L, int stab, unsigned long long seed,
                    const signed char *field, int delay_capacity, int drift)
{
    OChain *c = calloc(1, sizeof(OChain));
    c->kind = kind;
    c->Lx = Lx;
    c->Ly = kind == 0 ? 1 : Ly;
    c->n = c->Lx * c->Ly;
    c->L = L;
    c->stab = stab > 0 ? stab : 8;
    c->cap = delay_capacity > 0 ? delay_capacity : 16;
    c->U = U;
    c->dtau = dtau;
    const int n = c->n;
    const size_t nn = (size_t)n * n;
    o_lattice(c, pbc, t);
    /* model.c:8-31: K = t - mu I, mu = U/2 */
    double *K = malloc(nn * sizeof(double));
    memcpy(K, c->thop, nn * sizeof(double));
    for (int i = 0; i < n; i++) K[i + i * n] -= U / 2.0;
    c->expK = malloc(nn * sizeof(double));
    c->expKinv = malloc(nn * sizeof(double));
    orc_expm_sym(n, K, -dtau, c->expK);
    orc_expm_sym(n, K, dtau, c->expKinv);
    free(K);
    /* field.c:6-24 */
    c->lambda = acosh(exp(dtau * U / 2.0));
    for (int is = 0; is < 2; is++)
        for (int ss = 0; ss < 2; ss++) {
            const double sg = is ? 1.0 : -1.0, sv = ss ? 1.0 : -1.0;
            c->N_cache[is][ss] = exp(-2.0 * c->lambda * sg * sv) - 1.0;
        }
    const double cc = -dtau * U / 2.0;
    c->expv[0] = exp(-c->lambda + cc);
    c->expv[1] = exp(c->lambda + cc);
    c->expvinv[0] = 1.0 / c->expv[0];
    c->expvinv[1] = 1.0 / c->expv[1];
    o_rng_seed(&c->rng, seed);
    c->s = malloc((size_t)L * n);
    for (int k = 0; k < L * n; k++) c->s[k] = (o_rng_double(&c->rng) < 0.5) ? -1 : 1;
    if (field) memcpy(c->s, field, (size_t)L * n);
    c->Gu = malloc(nn * sizeof(double));
    c->Gd = malloc(nn * sizeof(double));
    c->dc = malloc(nn > 0 ? (size_t)n * c->cap * sizeof(double) : 8);
    c->dv = malloc(nn > 0 ? (size_t)n * c->cap * sizeof(double) : 8);
    /* green.c:168-187 */
    c->M = (L + c->stab - 1) / c->stab;
    c->S = malloc(sizeof(OUdv) * (size_t)(c->M + 1));
    c->b = malloc(sizeof(int) * (size_t)(c->M + 1));
    for (int j = 0; j <= c->M; j++) {
        c->b[j] = j * c->stab > L ? L : j * c->stab;
        o_udv_init(&c->S[j], n);
    }
    o_udv_init(&c->left, n);
    o_udv_init(&c->combined, n);
    c->drift_on = drift;
    /* dqmc.c:466-483: G from scratch at l0 = 0, PH map, sign = +1 */
    if (o_green_scratch(c, 0, c->Gu, &c->det_sign) != 0 || c->det_sign == 0) {
        c->status = 1;
        c->sign = 0.0;
    } else {
        o_map_ph(c);
        c->sign = 1.0;
    }
    c->cur_l = 0;
    return c;
}

/* dqmc.c:609-813, carry_prefix = 0, use_ph = 1, combine rebuild */
static void o_sweep(OChain *c)
{
    if (c->status) return;
    const int n = c->n, L = c->L;
    const size_t nn = (size_t)n * n;
    double *B = malloc(nn * sizeof(double));
    int tau_left = 0;
    /* green.c:203-226 suffix stack */
    o_udv_identity(&c->S[c->M]);
    o_udv_identity(&c->S[0]);
    for (int j = c->M - 1; j >= 1; j--) {
        o_build_Bblock(c, c->b[j], c->b[j + 1] - c->b[j], B);
        o_udv_copy(&c->S[j], &c->S[j + 1]);
        if (o_udv_rmul(&c->S[j], B) != 0) { c->status = 1; goto done; }
    }
    o_udv_identity(&c->left);
    for (int l = 0; l < L; l++) {
        for (int i = 0; i < n; i++) {
            const int si = c->s[l * n + i] > 0;
            const double Nu = c->N_cache[1][si];
            const double Nd = c->N_cache[0][si];
            const double gii = o_delay_diag(c, i);
            const double Ru = 1.0 + (1.0 - gii) * Nu;
            const double Rd = 1.0 + gii * Nd;
            const double R = Ru * Rd;
            c->attempts++;
            if (o_rng_double(&c->rng) < fabs(R)) {
                c->accepted++;
                o_delay_accept(c, i, Nu);
                c->s[l * n + i] *= -1;
                if (R < 0.0) c->sign = -c->sign;
            }
        }
        o_wrap(c);
        if ((l + 1) % c->stab == 0 && l + 1 < L) {
            const int tau = l + 1, j = tau / c->stab, len = tau - tau_left;
            if (o_drift(c, tau)) { c->status = 1; goto done; }
            o_build_Bblock(c, tau_left, len, B);
            if (o_udv_lmul(&c->left, B)) { c->status = 1; goto done; }
            tau_left = tau;
            int ds = 0;
            if (o_udv_combine(&c->left, &c->S[j], &c->combined) ||
                o_udv_inv_one_plus(&c->combined, c->Gu, &ds) || ds == 0) {
                c->status = 1;
                goto done;
            }
            c->det_sign = ds;
            c->cur_l = c->b[j] % L;
            c->delay_count = 0;
            o_map_ph(c);
            c->sign = 1.0;
        }
    }
    {
        const int len = L - tau_left;
        if (o_drift(c, 0)) { c->status = 1; goto done; }
        if (len > 0) {
            o_build_Bblock(c, tau_left, len, B);
            if (o_udv_lmul(&c->left, B)) { c->status = 1; goto done; }
        }
        int ds = 0;
        if (o_udv_inv_one_plus(&c->left, c->Gu, &ds) || ds == 0) {
            c->status = 1;
            goto done;
        }
        c->det_sign = ds;
        c->cur_l = 0;
        c->delay_count = 0;
        o_map_ph(c);
        c->sign = 1.0;
    }
    c->sweeps++;
done:
    free(B);
}

int orc_chain_sweep(void *h, int nsweeps)
{
    OChain *c = h;
    for (int k = 0; k < nsweeps; k++) o_sweep(c);
    return c->status;
}

void orc_chain_state(void *h, double *Gu, double *Gd, signed char *field,
                     unsigned long long *counters, double *sign, int *status,
                     unsigned long long *rng_state)
{
    OChain *c = h;
    const size_t nn = (size_t)c->n * c->n;
    if (Gu) memcpy(Gu, c->Gu, nn * sizeof(double));
    if (Gd) memcpy(Gd, c->Gd, nn * sizeof(double));
    if (field) memcpy(field, c->s, (size_t)c->L * c->n);
    if (counters) {
        counters[0] = c->attempts;
        counters[1] = c->accepted;
        counters[2] = c->sweeps;
    }
    if (sign) *sign = c->sign;
    if (status) *status = c->status;
    if (rng_state)
        for (int i = 0; i < 4; i++) rng_state[i] = c->rng.s[i];
}

void orc_chain_model(void *h, double *expK, double *expKinv, double *thop,
                     int *bipart, double *consts)
{
    OChain *c = h;
    const size_t nn = (size_t)c->n * c->n;
    if (expK) memcpy(expK, c->expK, nn * sizeof(double));
    if (expKinv) memcpy(expKinv, c->expKinv, nn * sizeof(double));
    if (thop) memcpy(thop, c->thop, nn * sizeof(double));
    if (bipart) memcpy(bipart, c->bipart, (size_t)c->n * sizeof(int));
    if (consts) {
        consts[0] = c->lambda;
        consts[1] = c->expv[0];
        consts[2] = c->expv[1];
        consts[3] = c->N_cache[1][0];
        consts[4] = c->N_cache[1][1];
        consts[5] = c->N_cache[0][0];
        consts[6] = c->N_cache[0][1];
    }
}

void orc_chain_drift(void *h, double *out)
{
    OChain *c = h;
    out[0] = (double)c->drift_samples;
    out[1] = c->drift_max;
    out[2] = c->drift_sum;
}

int orc_green_scratch(void *h, int l0, double *G, int *det_sign)
{
    return o_green_scratch((OChain *)h, l0, G, det_sign);
}

void orc_wrap(void *h, int l, double *G)
{
    o_wrap_g((OChain *)h, l, G);
}

/* measure.c:6-39 on (G_up, G_dn); out = {E, ekin, eint, ntot, doublon} */
void orc_measure_g(int n, const double *thop, double U, const double *gu,
                   const double *gd, double *out)
{
    double ekin = 0.0, eint = 0.0, dbl = 0.0, ntot = 0.0;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            const double t = thop[i + j * n], dij = i == j ? 1.0 : 0.0;
            ekin += t * (dij - gu[j + i * n]);
            ekin += t * (dij - gd[j + i * n]);
        }
    for (int i = 0; i < n; i++) {
        const double nu = 1.0 - gu[i + i * n], nd = 1.0 - gd[i + i * n];
        eint += nu * nd;
        dbl += nu * nd;
        ntot += nu + nd;
    }
    out[1] = ekin;
    out[2] = U * eint;
    out[3] = ntot;
    out[4] = dbl / n;
    out[0] = out[1] + out[2];
}

/* structure_factor.c:107-206 (af / all selectors), 258-297, 311-400.
 * sel: 1 = af, 2 = all.  Returns nq. */
int orc_spin_g(int n, int Lx, int Ly, int sel, const double *gu,
               const double *gd, double *szz, double *sperp)
{
    int nq = 0;
    int *mx = malloc(sizeof(int) * (size_t)n), *my = malloc(sizeof(int) * (size_t)n);
    if (sel == 1) {
        nq = 1;
        mx[0] = Lx > 1 ? Lx / 2 : 0;
        my[0] = Ly > 1 ? Ly / 2 : 0;
    } else {
        for (int y = 0; y < Ly; y++)
            for (int x = 0; x < Lx; x++) { mx[nq] = x; my[nq] = y; nq++; }
    }
    double *cz = calloc((size_t)n, sizeof(double)), *cp = calloc((size_t)n, sizeof(double));
    for (int i = 0; i < n; i++) {
        const int xi = i % Lx, yi = i / Lx;
        for (int j = 0; j < n; j++) {
            const double d = i == j ? 1.0 : 0.0;
            const double uii = gu[i + i * n], dii = gd[i + i * n];
            const double ujj = gu[j + j * n], djj = gd[j + j * n];
            const double uij = gu[i + j * n], uji = gu[j + i * n];
            const double dij = gd[i + j * n], dji = gd[j + i * n];
            const double czz = 0.25 * ((dii - uii) * (djj - ujj) + (d - uji) * uij +
                                       (d - dji) * dij);
            const double cpp = 0.5 * ((d - uji) * dij + (d - dji) * uij);
            int dx = xi - j % Lx, dy = yi - j / Lx;
            if (dx < 0) dx += Lx;
            if (dy < 0) dy += Ly;
            cz[dx + dy * Lx] += czz;
            cp[dx + dy * Lx] += cpp;
        }
    }
    const double two_pi = 2.0 * acos(-1.0);
    for (int q = 0; q < nq; q++) {
        double sz = 0.0, sp = 0.0;
        for (int disp = 0; disp < n; disp++) {
            const int dx = disp % Lx, dy = disp / Lx;
            const double ph = cos(two_pi * ((double)mx[q] * dx / Lx +
                                            (double)my[q] * dy / Ly));
            sz += ph * cz[disp];
            sp += ph * cp[disp];
        }
        szz[q] = sz / n;
        sperp[q] = sp / n;
    }
    free(mx); free(my); free(cz); free(cp);
    return nq;
}

int orc_chain_measure(void *h, double *out, int sel, double *szz, double *sperp)
{
    OChain *c = h;
    orc_measure_g(c->n, c->thop, c->U, c->Gu, c->Gd, out);
    if (sel <= 0 || szz == NULL || sperp == NULL) return 0;
    return orc_spin_g(c->n, c->Lx, c->Ly, sel, c->Gu, c->Gd, szz, sperp);
}

void orc_chain_free(void *h)
{
    OChain *c = h;
    if (!c) return;
    for (int j = 0; j <= c->M; j++) o_udv_free(&c->S[j]);
    o_udv_free(&c->left);
    o_udv_free(&c->combined);
    free(c->S); free(c->b); free(c->thop); free(c->bipart); free(c->expK);
    free(c->expKinv); free(c->s); free(c->Gu); free(c->Gd); free(c->dc);
    free(c->dv);
    free(c);
}
