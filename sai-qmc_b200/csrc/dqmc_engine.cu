/* Host side of libdqmc_b200: the C ABI declared in include/dqmc_gpu.h.
 *
 * Owns device memory (one arena per engine: every chain's state is a slice
 * of it), the stream, and the launches.  Setup work that the reference does
 * per replica on the host (model_init's matrix exponential, rng_seed,
 * field_init) stays on the host here too; everything per sweep runs on the
 * device.  There is no CPU fallback: without a CUDA device every call that
 * needs one fails with an error.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dqmc_gpu.h"
#include "dqmc_k2.h"
#include "dqmc_kernels.cuh"

namespace {

thread_local std::string g_err;

int set_err(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return 1;
}

#define CU(call)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess)                                                   \
            return set_err("%s failed: %s", #call, cudaGetErrorString(e_));      \
    } while (0)

/* splitmix64 seeding and xoshiro256** (src/rng.c:8-37), host copy used for
 * field_init before the stream moves to the device. */
uint64_t splitmix(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double host_rng_next(uint64_t *s)
{
    const uint64_t res = ((s[1] * 5) << 7 | (s[1] * 5) >> 57) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return (double)(res >> 11) * (1.0 / 9007199254740992.0);
}

/* Symmetric eigendecomposition A = Z diag(w) Z^T (column-major n x n), as
 * the reference's dsyev call in la_expm_sym (src/linalg.c:319-346) provides
 * it: Householder reduction to tridiagonal form with the reflectors
 * accumulated, then implicit symmetric QR steps with Wilkinson shifts on the
 * tridiagonal (Golub & Van Loan, Matrix Computations, Algorithms 5.1.1,
 * 8.3.1 and 8.3.2-8.3.3).  O(n^3) with a small constant: about 0.1 s at
 * n = 256 where cyclic Jacobi took seconds.  Returns 0, or -1 when the QR
 * iteration has not converged after 64 n shifts (w, Z are then not
 * eigenpairs and must not be used). */
int sym_eig(int n, const double *A, std::vector<double> &w, std::vector<double> &Z)
{
    std::vector<double> a(A, A + (size_t)n * n);
    auto at = [&](int i, int j) -> double & { return a[i + (size_t)j * n]; };
    std::vector<double> vs((size_t)n * n, 0.0), betas(n, 0.0), pv(n), wv(n);
    /* tridiagonalization: H_k = I - beta v v^T on rows / columns k+1 .. n-1 */
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        double *v = &vs[(size_t)k * n];
        double sigma = 0.0;
        for (int i = 1; i < m; ++i) sigma += at(k + 1 + i, k) * at(k + 1 + i, k);
        if (sigma == 0.0) continue;          /* column already tridiagonal */
        const double x0 = at(k + 1, k);
        const double mu = std::sqrt(x0 * x0 + sigma);
        const double v0 = x0 <= 0.0 ? x0 - mu : -sigma / (x0 + mu);
        const double beta = 2.0 * v0 * v0 / (sigma + v0 * v0);
        v[0] = 1.0;
        for (int i = 1; i < m; ++i) v[i] = at(k + 1 + i, k) / v0;
        betas[k] = beta;
        /* p = beta A22 v (column sweeps), w = p - (beta p^T v / 2) v */
        for (int i = 0; i < m; ++i) pv[i] = 0.0;
        for (int j = 0; j < m; ++j) {
            const double vj = beta * v[j];
            const double *col = &at(k + 1, k + 1 + j);
            for (int i = 0; i < m; ++i) pv[i] += col[i] * vj;
        }
        double ptv = 0.0;
        for (int i = 0; i < m; ++i) ptv += pv[i] * v[i];
        const double half = 0.5 * beta * ptv;
        for (int i = 0; i < m; ++i) wv[i] = pv[i] - half * v[i];
        /* A22 -= v w^T + w v^T */
        for (int j = 0; j < m; ++j) {
            double *col = &at(k + 1, k + 1 + j);
            const double wj = wv[j], vj = v[j];
            for (int i = 0; i < m; ++i) col[i] -= v[i] * wj + wv[i] * vj;
        }
        at(k + 1, k) = mu;
        at(k, k + 1) = mu;
        for (int i = 1; i < m; ++i) {
            at(k + 1 + i, k) = 0.0;
            at(k, k + 1 + i) = 0.0;
        }
    }
    /* Q = H_0 ... H_{n-3} by backward accumulation (Golub & Van Loan 5.1.6) */
    Z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Z[i + (size_t)i * n] = 1.0;
    for (int k = n - 3; k >= 0; --k) {
        if (betas[k] == 0.0) continue;
        const int m = n - k - 1;
        const double *v = &vs[(size_t)k * n];
        for (int j = k + 1; j < n; ++j) {
            double *col = &Z[(k + 1) + (size_t)j * n];
            double sdot = 0.0;
            for (int i = 0; i < m; ++i) sdot += v[i] * col[i];
            sdot *= betas[k];
            for (int i = 0; i < m; ++i) col[i] -= sdot * v[i];
        }
    }
    std::vector<double> d(n), e(n > 1 ? n - 1 : 1, 0.0);
    for (int i = 0; i < n; ++i) d[i] = at(i, i);
    for (int i = 0; i + 1 < n; ++i) e[i] = at(i + 1, i);
    /* implicit symmetric QR with Wilkinson shifts; Z <- Z R^T per rotation */
    const double eps = std::numeric_limits<double>::epsilon();
    int q = n - 1, guard = 0;
    while (q > 0 && guard < 64 * n) {
        for (int i = 0; i < q; ++i)
            if (std::fabs(e[i]) <= eps * (std::fabs(d[i]) + std::fabs(d[i + 1]))) e[i] = 0.0;
        if (e[q - 1] == 0.0) {
            --q;
            continue;
        }
        int p = q - 1;
        while (p > 0 && e[p - 1] != 0.0) --p;
        ++guard;
        const double dd = 0.5 * (d[q - 1] - d[q]), ee = e[q - 1];
        const double mu = d[q] - ee * ee / (dd + std::copysign(std::hypot(dd, ee), dd));
        double x = d[p] - mu, z = e[p], bulge = 0.0;
        for (int k = p; k < q; ++k) {
            const double r = std::hypot(x, z);
            const double c = r == 0.0 ? 1.0 : x / r, sn = r == 0.0 ? 0.0 : z / r;
            if (k > p) e[k - 1] = r;
            const double ak = d[k], bk = e[k], ck = d[k + 1];
            d[k] = c * c * ak + 2.0 * c * sn * bk + sn * sn * ck;
            e[k] = c * sn * (ck - ak) + (c * c - sn * sn) * bk;
            d[k + 1] = sn * sn * ak - 2.0 * c * sn * bk + c * c * ck;
            if (k + 1 < q) {
                bulge = sn * e[k + 1];
                e[k + 1] *= c;
            }
            double *zk = &Z[(size_t)k * n], *zk1 = &Z[(size_t)(k + 1) * n];
            for (int i = 0; i < n; ++i) {
                const double u = zk[i], t = zk1[i];
                zk[i] = c * u + sn * t;
                zk1[i] = -sn * u + c * t;
            }
            x = e[k];
            z = bulge;
        }
    }
    w = d;
    return q > 0 ? -1 : 0;
}

/* out_s = Z diag(exp(s_t w)) Z^T for the scales s_0, s_1 of one
 * decomposition (expK and expK^-1 of a model share it). */
void expm_from_eig(int n, const std::vector<double> &w, const std::vector<double> &Z,
                   double scale, double *out)
{
    for (size_t i = 0; i < (size_t)n * n; ++i) out[i] = 0.0;
    for (int k = 0; k < n; ++k) {
        const double f = std::exp(scale * w[k]);
        const double *zk = &Z[(size_t)k * n];
        for (int j = 0; j < n; ++j) {
            const double fj = f * zk[j];
            double *col = out + (size_t)j * n;
            for (int i = 0; i < n; ++i) col[i] += zk[i] * fj;
        }
    }
}

size_t rup(size_t b) { return (b + 255) & ~(size_t)255; }

struct HModel {
    int n, Lx, Ly;
    double U, dtau;
    double mu = 0.0;
    int ph = 1;   /* particle-hole path (half filling on a bipartite lattice) */
    std::vector<double> thop, expK, expKinv, cos_zz, cos_perp;
    std::vector<int> bipart;
    int nq_zz = 0, nq_perp = 0;
};

struct HChain {
    int model, L, stab, M, kb;
    int pair_forced;           /* delay rank > 32: two site blocks per G update */
    int pair_mode;             /* DQMC_PAIRS_* of this chain                   */
    uint64_t rng[4];
    std::vector<signed char> field;
    std::vector<double> udv;   /* drained UDV scale records, oldest first */
};

/* UDV scale records a chain can take in one sweep: M - 1 stack factors,
 * M - 1 boundaries, the final factor, and M prefix factors of a backward
 * sweep that has to build its prefix stack. */
int udv_cap(int M) { return 3 * M + 4; }

}  // namespace

namespace dqmc_internal {
/* lets other translation units of the library report through
 * dqmc_last_error() */
void set_error(const char *msg) { g_err = msg; }
}  // namespace dqmc_internal

struct dqmc_engine {
    dqmc_engine_desc desc;
    std::vector<HModel> models;
    std::vector<HChain> chains;
    cudaStream_t stream = nullptr;
    char *dmod = nullptr, *darena = nullptr;
    DqmcModelDev *dmodels = nullptr;
    DqmcChainDev *dchains = nullptr;
    int *dorder = nullptr;           /* launch order of the sweep kernel */
    std::vector<DqmcChainDev> hdev;  /* host mirror: device pointers */
    int nbin = 0;
    size_t smem = 0, msmem = 0, smem2 = 0;
    int per_sm = 1;           /* CTAs per SM of the sweep kernels (1 or 2) */
    int cl = 1;               /* cluster size of the sweep kernel (1: none)       */
    int ncoop = 0;            /* chains (most expensive first) on a cluster each  */
    int nclus = 0;            /* clusters of the launch                           */
    bool prepared = false;
    /* per-launch CUDA events (kind 0 = sweep kernel, 1 = measurement) */
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_kind;
    cudaEvent_t mark[2] = {nullptr, nullptr};
};

static void ev_begin(dqmc_engine *e, int kind)
{
    if (!e->timing) return;
    cudaEvent_t a;
    cudaEventCreate(&a);
    cudaEventRecord(a, e->stream);
    e->ev.push_back(a);
    e->ev_kind.push_back(kind);
}

static void ev_end(dqmc_engine *e)
{
    if (!e->timing) return;
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, e->stream);
    e->ev.push_back(b);
    e->ev_kind.push_back(-1);
}

extern "C" {

const char *dqmc_last_error(void) { return g_err.c_str(); }

void dqmc_desc_default(dqmc_engine_desc *d)
{
    std::memset(d, 0, sizeof *d);
    d->device = 0;
    d->precision = DQMC_PREC_FP64;
    d->delay_rank = 0;
    d->drift = DQMC_DRIFT_STAB;
}

int dqmc_expm_sym(int n, const double *A, double scale, double *out)
{
    if (n <= 0 || !A || !out) return set_err("dqmc_expm_sym: bad arguments");
    std::vector<double> w, Z;
    if (sym_eig(n, A, w, Z) != 0)
        return set_err("dqmc_expm_sym: the symmetric QR iteration did not converge");
    expm_from_eig(n, w, Z, scale, out);
    return 0;
}

dqmc_engine *dqmc_engine_create(const dqmc_engine_desc *desc)
{
    dqmc_engine_desc d;
    if (desc)
        d = *desc;
    else
        dqmc_desc_default(&d);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_err("no CUDA device available (%s); the engine has no CPU path",
                e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return nullptr;
    }
    if (d.device < 0 || d.device >= ndev) {
        set_err("device %d out of range (%d devices)", d.device, ndev);
        return nullptr;
    }
    if (d.sweep_order != DQMC_SWEEP_FORWARD && d.sweep_order != DQMC_SWEEP_ALTERNATING) {
        set_err("sweep_order %d is neither DQMC_SWEEP_FORWARD nor DQMC_SWEEP_ALTERNATING",
                d.sweep_order);
        return nullptr;
    }
    if (d.flush_pairs < DQMC_PAIRS_AUTO || d.flush_pairs > DQMC_PAIRS_ON) {
        set_err("flush_pairs %d is not a DQMC_PAIRS_* value", d.flush_pairs);
        return nullptr;
    }
    if (d.green_rebuild < DQMC_REBUILD_COMBINE || d.green_rebuild > DQMC_REBUILD_CENTERED) {
        set_err("green_rebuild %d is not a DQMC_REBUILD_* value", d.green_rebuild);
        return nullptr;
    }
    if (d.precision != DQMC_PREC_FP64 && d.precision != DQMC_PREC_MIXED) {
        set_err("precision %d is neither DQMC_PREC_FP64 nor DQMC_PREC_MIXED", d.precision);
        return nullptr;
    }
    if (d.chain_ctas < 0 || d.chain_ctas > DQMC_MAX_CHAIN_CTAS) {
        set_err("chain_ctas %d is outside 0..%d", d.chain_ctas, DQMC_MAX_CHAIN_CTAS);
        return nullptr;
    }
    if (d.chain_ctas > 1 && d.ctas_per_sm == 2) {
        set_err("chain_ctas %d needs one CTA per SM (ctas_per_sm 0 or 1)", d.chain_ctas);
        return nullptr;
    }
    if (cudaSetDevice(d.device) != cudaSuccess) {
        set_err("cudaSetDevice(%d) failed", d.device);
        return nullptr;
    }
    dqmc_engine *eng = new dqmc_engine();
    eng->desc = d;
    if (cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_err("cudaStreamCreate failed");
        delete eng;
        return nullptr;
    }
    return eng;
}

void dqmc_engine_destroy(dqmc_engine *e)
{
    if (!e) return;
    cudaSetDevice(e->desc.device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (cudaEvent_t v : e->ev) cudaEventDestroy(v);
    for (cudaEvent_t v : e->mark)
        if (v) cudaEventDestroy(v);
    cudaFree(e->dmod);
    cudaFree(e->darena);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int dqmc_model_add(dqmc_engine *e, int n, int Lx, int Ly, const double *thop,
                   const int *bipart, double U, double dtau)
{
    if (!bipart) return -set_err("dqmc_model_add: null bipart (see dqmc_model_add_mu)");
    return dqmc_model_add_mu(e, n, Lx, Ly, thop, bipart, U, dtau, 1, 0.0, 0);
}

int dqmc_model_add_mu(dqmc_engine *e, int n, int Lx, int Ly, const double *thop,
                      const int *bipart, double U, double dtau, int half_filling, double mu,
                      int two_spin)
{
    if (!e || e->prepared) return -set_err("dqmc_model_add: engine missing or prepared");
    if (n <= 0 || n > DQMC_MAX_N || !thop)
        return -set_err("dqmc_model_add: n=%d outside 1..%d or null input", n, DQMC_MAX_N);
    if (!(dtau > 0.0) || !(U >= 0.0)) return -set_err("dqmc_model_add: need U>=0, dtau>0");
    if (!half_filling && !std::isfinite(mu)) return -set_err("dqmc_model_add: mu not finite");
    HModel m;
    m.n = n;
    m.Lx = Lx;
    m.Ly = Ly;
    m.U = U;
    m.dtau = dtau;
    m.thop.assign(thop, thop + (size_t)n * n);
    if (bipart) m.bipart.assign(bipart, bipart + n);
    else m.bipart.assign(n, 0);
    /* model_init (src/model.c:8-31): mu = U/2 at half filling, K = t - mu I;
     * the PH path needs half filling on a bipartite lattice (ph_symmetric) */
    m.mu = half_filling ? U / 2.0 : mu;
    m.ph = (half_filling && bipart && !two_spin) ? 1 : 0;
    std::vector<double> K(m.thop);
    for (int i = 0; i < n; ++i) K[i + (size_t)i * n] -= m.mu;
    m.expK.resize((size_t)n * n);
    m.expKinv.resize((size_t)n * n);
    std::vector<double> w, Z;   /* one decomposition for expK and expK^-1 */
    if (sym_eig(n, K.data(), w, Z) != 0)
        return -set_err("dqmc_model_add: the eigensolver of t - mu I did not converge");
    expm_from_eig(n, w, Z, -dtau, m.expK.data());
    expm_from_eig(n, w, Z, dtau, m.expKinv.data());
    e->models.push_back(std::move(m));
    return (int)e->models.size() - 1;
}

int dqmc_model_set_spin(dqmc_engine *e, int model, int nq_zz, const int *mx_zz,
                        const int *my_zz, int nq_perp, const int *mx_perp,
                        const int *my_perp)
{
    if (!e || e->prepared || model < 0 || model >= (int)e->models.size())
        return set_err("dqmc_model_set_spin: bad engine/model");
    HModel &m = e->models[model];
    if ((nq_zz > 0 || nq_perp > 0) && (m.Lx <= 0 || m.Ly <= 0 || m.Lx * m.Ly != m.n))
        return set_err("dqmc_model_set_spin: model has no site coordinates");
    /* phase table of structure_factor_plan_init (src/structure_factor.c:
     * 182-199): cos(2 pi (mx dx / Lx + my dy / Ly)) */
    const double two_pi = 2.0 * std::acos(-1.0);
    auto table = [&](int nq, const int *mx, const int *my, std::vector<double> &out) {
        out.assign((size_t)m.n * nq, 0.0);
        for (int q = 0; q < nq; ++q)
            for (int d = 0; d < m.n; ++d) {
                const int dx = d % m.Lx, dy = d / m.Lx;
                const double ang = two_pi * ((double)mx[q] * (double)dx / (double)m.Lx +
                                             (double)my[q] * (double)dy / (double)m.Ly);
                out[d + (size_t)q * m.n] = std::cos(ang);
            }
    };
    m.nq_zz = nq_zz > 0 ? nq_zz : 0;
    m.nq_perp = nq_perp > 0 ? nq_perp : 0;
    if (m.nq_zz) table(nq_zz, mx_zz, my_zz, m.cos_zz);
    if (m.nq_perp) table(nq_perp, mx_perp, my_perp, m.cos_perp);
    return 0;
}

/* Delay rank k of one chain: site blocks of k <= 32 sites (one register
 * lane per column); 32 < k <= 64 runs blocks of ceil(k/2) sites whose G
 * updates are paired, one rank <= k update per k sites. */
static int set_delay(dqmc_engine *e, HChain &c, int n, int model, int delay_rank, int pairs,
                     const char *who)
{
    int kb = delay_rank;
    c.pair_forced = 0;
    if (pairs < DQMC_PAIRS_AUTO || pairs > DQMC_PAIRS_ON)
        return set_err("%s: flush_pairs %d is not a DQMC_PAIRS_* value", who, pairs);
    c.pair_mode = pairs;
    if (kb <= 0) kb = 32;
    if (kb > 2 * DQMC_MAX_KB)
        return set_err("%s: delay_rank %d exceeds %d (site blocks of at most %d sites, two per "
                       "G update)", who, kb, 2 * DQMC_MAX_KB, DQMC_MAX_KB);
    if (kb > DQMC_MAX_KB) {
        if (pairs == DQMC_PAIRS_OFF)
            return set_err("%s: delay_rank %d > %d needs paired flushes (flush_pairs is OFF)",
                           who, kb, DQMC_MAX_KB);
        if (!e->models[model].ph)
            return set_err("%s: delay_rank %d > %d is not available on the two-spin path", who,
                           kb, DQMC_MAX_KB);
        kb = (kb + 1) / 2;
        c.pair_forced = 1;
    }
    if (kb > n) kb = n;
    c.kb = kb;
    return 0;
}

int dqmc_chain_tune(dqmc_engine *e, int chain, int delay_rank, int flush_pairs)
{
    if (!e || e->prepared || chain < 0 || chain >= (int)e->chains.size())
        return set_err("dqmc_chain_tune: bad engine/chain, or engine already prepared");
    HChain &c = e->chains[chain];
    return set_delay(e, c, e->models[c.model].n, c.model, delay_rank, flush_pairs,
                     "dqmc_chain_tune");
}

int dqmc_chain_add(dqmc_engine *e, int model, int L, int stab, uint64_t seed,
                   const signed char *field)
{
    if (!e || e->prepared || model < 0 || model >= (int)e->models.size())
        return -set_err("dqmc_chain_add: bad engine/model");
    if (L <= 0) return -set_err("dqmc_chain_add: L must be > 0");
    const int n = e->models[model].n;
    HChain c;
    c.model = model;
    c.L = L;
    c.stab = stab > 0 ? stab : 8;   /* green_stack_alloc default, src/green.c:172 */
    c.M = (L + c.stab - 1) / c.stab;
    if (set_delay(e, c, n, model, e->desc.delay_rank, e->desc.flush_pairs, "dqmc_chain_add"))
        return -1;
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) c.rng[i] = splitmix(&x);
    c.field.resize((size_t)L * n);
    /* field_init (src/field.c:18-23): one uniform per (l, i), always drawn */
    for (size_t k = 0; k < c.field.size(); ++k)
        c.field[k] = host_rng_next(c.rng) < 0.5 ? -1 : 1;
    if (field) {
        for (size_t k = 0; k < c.field.size(); ++k) {
            if (field[k] != 1 && field[k] != -1)
                return -set_err("dqmc_chain_add: field entries must be +/-1");
            c.field[k] = field[k];
        }
    }
    e->chains.push_back(std::move(c));
    return (int)e->chains.size() - 1;
}

/* A split-product operand of a model matrix (the device's spl_split, same
 * arithmetic and block layout, dqmc_split.cuh): line l is row l of M
 * (by_rows, M[l + k*n]) or column l (M[k + l*n]), in blocks of 128 lines;
 * X = round(x 2^(NB - e)) in balanced base-256 digits (top digit first);
 * sc[l] = 2^(e - NB + 4 (S - 1)). */
static void split_host(int n, const double *M, bool by_rows, std::vector<signed char> &tiles,
                       std::vector<double> &sc)
{
    const int S = DQMC_MIX_DIGITS, NB = dq::SPL_NB, nkc = dq::spl_nkc(n);
    tiles.assign(dq::spl_tile_bytes(n, n), 0);
    sc.assign((size_t)dq::spl_nlb(n) * dq::SPL_LB, std::ldexp(1.0, -NB + 4 * (S - 1)));
    for (int l = 0; l < n; ++l) {
        auto val = [&](int k) { return by_rows ? M[l + (size_t)k * n] : M[k + (size_t)l * n]; };
        double m = 0.0;
        for (int k = 0; k < n; ++k) m = std::fmax(m, std::fabs(val(k)));
        int e = 0;
        if (m > 0.0) std::frexp(m, &e);
        sc[l] = std::ldexp(1.0, e - NB + 4 * (S - 1));
        const double f = std::ldexp(1.0, NB - e);
        for (int k = 0; k < n; ++k) {
            long long X = std::llrint(val(k) * f);
            for (int p = S - 1; p >= 0; --p) {
                int d;
                if (p > 0) {
                    d = (int)((X + 128) & 255) - 128;
                    X = (X - d) >> 8;
                } else {
                    d = (int)X;
                }
                tiles[dq::spl_offset(nkc, l, k, p)] = (signed char)d;
            }
        }
    }
}

int dqmc_engine_prepare(dqmc_engine *e, int nbin)
{
    if (!e || e->prepared) return set_err("dqmc_engine_prepare: engine missing or prepared");
    if (e->chains.empty()) return set_err("dqmc_engine_prepare: no chains");
    CU(cudaSetDevice(e->desc.device));
    e->nbin = nbin > 0 ? nbin : 1;
    /* models */
    const bool mixed = e->desc.precision == DQMC_PREC_MIXED;
    const bool alt = e->desc.sweep_order == DQMC_SWEEP_ALTERNATING;
    for (const HChain &c : e->chains) {
        if (e->models[c.model].ph) continue;
        /* dqmc_init_modes rejects the alternating order off the PH path
         * (src/dqmc.c:440-446) */
        if (alt)
            return set_err("dqmc_engine_prepare: sweep_order=alternating needs the "
                           "particle-hole path (half filling, bipartite lattice)");
        if (mixed)
            return set_err("dqmc_engine_prepare: precision=mixed needs the particle-hole path");
    }
    if (mixed) {
        for (const HModel &m : e->models)
            if (!dq::qr_cb(m.n))
                return set_err("dqmc_engine_prepare: mixed precision needs n <= %d here (n = %d)",
                               3 * DQMC_NT, m.n);
    }
    /* split operands of a model: expK, expK^-1 by rows (A) and columns (B) */
    auto spl_bytes = [](int n) {
        return rup(dq::spl_tile_bytes(n, n)) + rup((size_t)dq::spl_nlb(n) * dq::SPL_LB * 8);
    };
    size_t moff = 0;
    std::vector<size_t> mo(e->models.size() * 10);
    for (size_t k = 0; k < e->models.size(); ++k) {
        const HModel &m = e->models[k];
        const size_t nn = (size_t)m.n * m.n;
        mo[10 * k + 0] = moff; moff += rup(nn * 8);
        mo[10 * k + 1] = moff; moff += rup(nn * 8);
        mo[10 * k + 2] = moff; moff += rup(nn * 8);
        mo[10 * k + 3] = moff; moff += rup((size_t)m.n * 4);
        mo[10 * k + 4] = moff; moff += rup(m.cos_zz.size() * 8 + 8);
        mo[10 * k + 5] = moff; moff += rup(m.cos_perp.size() * 8 + 8);
        const size_t sa = mixed ? spl_bytes(m.n) : 0;
        const size_t sb = sa;
        mo[10 * k + 6] = moff; moff += sa;   /* expK by rows      */
        mo[10 * k + 7] = moff; moff += sb;   /* expK by columns   */
        mo[10 * k + 8] = moff; moff += sa;   /* expK^-1 by rows   */
        mo[10 * k + 9] = moff; moff += sb;   /* expK^-1 by columns */
    }
    const size_t mstruct = moff;
    moff += rup(sizeof(DqmcModelDev) * e->models.size());
    CU(cudaMalloc(&e->dmod, moff));
    std::vector<DqmcModelDev> hm(e->models.size());
    for (size_t k = 0; k < e->models.size(); ++k) {
        const HModel &m = e->models[k];
        const size_t nn = (size_t)m.n * m.n;
        DqmcModelDev &d = hm[k];
        std::memset(&d, 0, sizeof d);
        d.n = m.n;
        d.Lx = m.Lx;
        d.Ly = m.Ly;
        d.U = m.U;
        d.dtau = m.dtau;
        d.mu = m.mu;
        d.ph = m.ph;
        /* field.c:10-17, green.c:63-67 (sigma = +1 for the evolved spin,
         * -1 for G_down of the two-spin path) */
        const double lambda = std::acosh(std::exp(m.dtau * m.U / 2.0));
        const double c = -m.dtau * m.U / 2.0;
        d.expv[0] = std::exp(lambda * -1.0 + c);
        d.expv[1] = std::exp(lambda * 1.0 + c);
        d.expvinv[0] = 1.0 / d.expv[0];
        d.expvinv[1] = 1.0 / d.expv[1];
        d.expvd[0] = std::exp(lambda * 1.0 + c);
        d.expvd[1] = std::exp(lambda * -1.0 + c);
        d.expvinvd[0] = 1.0 / d.expvd[0];
        d.expvinvd[1] = 1.0 / d.expvd[1];
        for (int is = 0; is < 2; ++is) {
            const double sv = is ? 1.0 : -1.0;
            d.Nup[is] = std::exp(-2.0 * lambda * 1.0 * sv) - 1.0;
            d.Ndn[is] = std::exp(-2.0 * lambda * -1.0 * sv) - 1.0;
        }
        d.expK = (const double *)(e->dmod + mo[10 * k + 0]);
        d.expKinv = (const double *)(e->dmod + mo[10 * k + 1]);
        d.thop = (const double *)(e->dmod + mo[10 * k + 2]);
        d.bipart = (const int *)(e->dmod + mo[10 * k + 3]);
        d.cos_zz = (const double *)(e->dmod + mo[10 * k + 4]);
        d.cos_perp = (const double *)(e->dmod + mo[10 * k + 5]);
        d.nq_zz = m.nq_zz;
        d.nq_perp = m.nq_perp;
        CU(cudaMemcpy(e->dmod + mo[10 * k + 0], m.expK.data(), nn * 8, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(e->dmod + mo[10 * k + 1], m.expKinv.data(), nn * 8, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(e->dmod + mo[10 * k + 2], m.thop.data(), nn * 8, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(e->dmod + mo[10 * k + 3], m.bipart.data(), (size_t)m.n * 4,
                      cudaMemcpyHostToDevice));
        if (m.nq_zz)
            CU(cudaMemcpy(e->dmod + mo[10 * k + 4], m.cos_zz.data(), m.cos_zz.size() * 8,
                          cudaMemcpyHostToDevice));
        if (m.nq_perp)
            CU(cudaMemcpy(e->dmod + mo[10 * k + 5], m.cos_perp.data(), m.cos_perp.size() * 8,
                          cudaMemcpyHostToDevice));
        if (mixed) {
            std::vector<signed char> tl;
            std::vector<double> sc;
            auto put = [&](DqmcSplitDev &op, size_t off, const double *M, bool rows) -> int {
                split_host(m.n, M, rows, tl, sc);
                op.t = (signed char *)(e->dmod + off);
                op.sc = (double *)(e->dmod + off + rup(tl.size()));
                op.nlb = dq::spl_nlb(m.n);
                op.nkc = dq::spl_nkc(m.n);
                CU(cudaMemcpy(op.t, tl.data(), tl.size(), cudaMemcpyHostToDevice));
                CU(cudaMemcpy(op.sc, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice));
                return 0;
            };
            if (put(d.spK_r, mo[10 * k + 6], m.expK.data(), true) ||
                put(d.spK_c, mo[10 * k + 7], m.expK.data(), false) ||
                put(d.spKi_r, mo[10 * k + 8], m.expKinv.data(), true) ||
                put(d.spKi_c, mo[10 * k + 9], m.expKinv.data(), false))
                return 1;
        }
    }
    e->dmodels = (DqmcModelDev *)(e->dmod + mstruct);
    CU(cudaMemcpy(e->dmodels, hm.data(), sizeof(DqmcModelDev) * hm.size(),
                  cudaMemcpyHostToDevice));

    /* chain arena layout */
    const size_t nc = e->chains.size();
    std::vector<size_t> base(nc);
    size_t off = 0;
    size_t maxsmem = 0;
    int maxn = 0;
    for (size_t k = 0; k < nc; ++k) {
        const HChain &c = e->chains[k];
        const HModel &m = e->models[c.model];
        const int n = m.n;
        const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
        base[k] = off;
        off += rup((size_t)c.L * n);                          /* field */
        off += rup(nn * 8);                                   /* G */
        off += rup((size_t)(c.M + 1) * usz * 8);              /* S */
        if (alt) off += rup((size_t)(c.M + 1) * usz * 8);     /* P (alternating) */
        off += 3 * rup(usz * 8);                              /* left, comb, scr */
        off += rup((size_t)c.M * nn * 8);                     /* bcache */
        off += 6 * rup(nn * 8);                               /* w */
        off += 2 * rup((size_t)n * 2 * c.kb * 8);             /* Zs, Ys */
        if (e->desc.udv_diag)                                  /* UDV scale records */
            off += rup((size_t)(m.ph ? 1 : 2) * udv_cap(c.M) * DQMC_UDV_RECORD_DOUBLES * 8);
        if (!m.ph) {   /* G_down's state on the two-spin path */
            off += rup(nn * 8) + rup((size_t)(c.M + 1) * usz * 8) + 2 * rup(usz * 8) +
                   rup((size_t)c.M * nn * 8) + 2 * rup((size_t)n * 2 * c.kb * 8);
        }
        off += rup((size_t)((n + DQMC_QNB - 1) / DQMC_QNB) * DQMC_QNB * DQMC_QNB * 8);
        off += rup((size_t)e->nbin * DQMC_BIN_FIELDS * 8);
        off += rup((size_t)e->nbin * m.nq_zz * 8 + 8);
        off += rup((size_t)e->nbin * m.nq_perp * 8 + 8);
        if (mixed) off += 2 * spl_bytes(n);
        if (e->desc.green_log > 0) off += rup((size_t)e->desc.green_log * nn * 8);
        off += rup((size_t)DQMC_CL_STAGE_DOUBLES * 8);       /* cluster staging */
        const size_t sm = dq::smem_bytes(n, c.kb);
        if (sm > maxsmem) maxsmem = sm;
        const size_t sm2 = dq2x::smem_bytes(n, c.kb);
        if (sm2 > e->smem2) e->smem2 = sm2;
        if (n > maxn) maxn = n;
    }
    const size_t cstruct = off;
    off += rup(sizeof(DqmcChainDev) * nc);
    const size_t corder = off;
    off += rup(sizeof(int) * nc);
    CU(cudaMalloc(&e->darena, off));
    CU(cudaMemset(e->darena, 0, off));
    e->hdev.assign(nc, DqmcChainDev());
    for (size_t k = 0; k < nc; ++k) {
        const HChain &c = e->chains[k];
        const HModel &m = e->models[c.model];
        const int n = m.n;
        const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
        DqmcChainDev &d = e->hdev[k];
        std::memset(&d, 0, sizeof d);
        d.model = c.model;
        d.n = n;
        d.L = c.L;
        d.stab = c.stab;
        d.M = c.M;
        d.kb = c.kb;
        d.nbin = e->nbin;
        for (int i = 0; i < 4; ++i) d.rng[i] = c.rng[i];
        char *p = e->darena + base[k];
        auto take = [&](size_t bytes) { char *q = p; p += rup(bytes); return q; };
        d.field = (signed char *)take((size_t)c.L * n);
        d.G = (double *)take(nn * 8);
        d.S = (double *)take((size_t)(c.M + 1) * usz * 8);
        if (alt) d.P = (double *)take((size_t)(c.M + 1) * usz * 8);
        d.alt = alt ? 1 : 0;
        d.rebuild = e->desc.green_rebuild != DQMC_REBUILD_COMBINE ? 1 : 0;
        d.pair = c.pair_forced || c.pair_mode == DQMC_PAIRS_ON ||
                 (c.pair_mode == DQMC_PAIRS_AUTO && n >= 128);
        d.left = (double *)take(usz * 8);
        d.comb = (double *)take(usz * 8);
        d.scr = (double *)take(usz * 8);
        d.bcache = (double *)take((size_t)c.M * nn * 8);
        for (int i = 0; i < 6; ++i) d.w[i] = (double *)take(nn * 8);
        d.Zs = (double *)take((size_t)n * 2 * c.kb * 8);
        d.Ys = (double *)take((size_t)n * 2 * c.kb * 8);
        if (e->desc.udv_diag) {
            d.udv_cap = (m.ph ? 1 : 2) * udv_cap(c.M);
            d.udvrec = (double *)take((size_t)d.udv_cap * DQMC_UDV_RECORD_DOUBLES * 8);
        }
        d.ns = m.ph ? 1 : 2;
        if (!m.ph) {
            d.pair = 0;
            d.Gd = (double *)take(nn * 8);
            d.Sd = (double *)take((size_t)(c.M + 1) * usz * 8);
            d.leftd = (double *)take(usz * 8);
            d.combd = (double *)take(usz * 8);
            d.bcached = (double *)take((size_t)c.M * nn * 8);
            d.Zsd = (double *)take((size_t)n * 2 * c.kb * 8);
            d.Ysd = (double *)take((size_t)n * 2 * c.kb * 8);
        }
        d.twall = (double *)take((size_t)((n + DQMC_QNB - 1) / DQMC_QNB) * DQMC_QNB *
                                 DQMC_QNB * 8);
        d.bins = (double *)take((size_t)e->nbin * DQMC_BIN_FIELDS * 8);
        d.bins_zz = (double *)take((size_t)e->nbin * m.nq_zz * 8 + 8);
        d.bins_perp = (double *)take((size_t)e->nbin * m.nq_perp * 8 + 8);
        if (mixed) {
            for (int ab = 0; ab < 2; ++ab) {
                DqmcSplitDev &op = ab ? d.spB : d.spA;
                op.nlb = dq::spl_nlb(n);
                op.nkc = dq::spl_nkc(n);
                op.t = (signed char *)take(dq::spl_tile_bytes(n, n));
                op.sc = (double *)take((size_t)op.nlb * dq::SPL_LB * 8);
            }
        }
        if (e->desc.green_log > 0) {
            d.glog_cap = e->desc.green_log;
            d.glog = (double *)take((size_t)d.glog_cap * nn * 8);
        }
        d.clstage = (double *)take((size_t)DQMC_CL_STAGE_DOUBLES * 8);
        CU(cudaMemcpy(d.field, c.field.data(), c.field.size(), cudaMemcpyHostToDevice));
    }
    e->dchains = (DqmcChainDev *)(e->darena + cstruct);
    CU(cudaMemcpy(e->dchains, e->hdev.data(), sizeof(DqmcChainDev) * nc,
                  cudaMemcpyHostToDevice));
    /* sweep launch order: most expensive chain first (a sweep costs about
     * n^3 L, twice that on the two-spin path), ties in insertion order */
    {
        std::vector<int> order(nc);
        for (size_t k = 0; k < nc; ++k) order[k] = (int)k;
        auto cost = [&](int k) {
            const HChain &c = e->chains[k];
            const HModel &m = e->models[c.model];
            return (double)m.n * m.n * m.n * c.L * (m.ph ? 1.0 : 2.0);
        };
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return cost(a) > cost(b); });
        e->dorder = (int *)(e->darena + corder);
        CU(cudaMemcpy(e->dorder, order.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
    }
    e->smem = maxsmem;
    e->msmem = (size_t)2 * maxn * 8;
    if (e->smem > 227 * 1024) return set_err("shared memory need %zu B exceeds 227 KB", e->smem);
    CU(dq::set_attrs(e->smem, e->msmem));
    /* Two chains per SM when the batch has more chains than SMs and two
     * CTAs fit in shared memory: the second chain fills the first one's
     * barrier and reduction latency. */
    int nsm = 148;
    {
        int dev = 0;
        CU(cudaGetDevice(&dev));
        CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const bool fits2 = 2 * (e->smem2 + 1024) <= 228 * 1024;
        const int want = e->desc.ctas_per_sm;
        /* the two-spin proposals hold both spins' block columns in
         * registers: one CTA per SM */
        bool two = false;
        for (const HChain &c : e->chains) two = two || !e->models[c.model].ph;
        e->per_sm = (want == 2 || (want == 0 && (int)nc > nsm)) && fits2 && !mixed && !two &&
                            e->desc.chain_ctas <= 1
                        ? 2
                        : 1;
        if (e->per_sm == 2) CU(dq2x::set_attrs(e->smem2, e->msmem));
    }
    /* Thread-block clusters.  A cluster of cc CTAs either advances one chain
     * (the ncoop most expensive chains in launch order) or runs cc of the
     * other chains, one per CTA.  Explicit: chain_ctas > 1, cluster_chains
     * of them (0 = all).  Automatic (chain_ctas = 0) for batches of fewer
     * chains than SMs whose largest lattice has n >= 128: the (cc in 2..16,
     * ncoop)
     * whose slowest chain is predicted fastest, every cluster resident at
     * once (a second wave of clusters costs more than narrower ones), by
     * chain cost n^3 L (doubled on the two-spin path) over the speedup
     * 1 + a(n) log2(cc) of a chain on cc CTAs, a(n) interpolated through
     * measured points: (64, 0), (144, 0.245), (256, 0.30), (576, 0.67). */
    e->cl = 1;
    e->ncoop = (int)nc;
    e->nclus = (int)nc;
    {
        std::vector<double> w(nc), an(nc);
        std::vector<int> ord(nc);
        CU(cudaMemcpy(ord.data(), e->dorder, sizeof(int) * nc, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < nc; ++k) {
            const HChain &c = e->chains[ord[k]];
            const HModel &m = e->models[c.model];
            w[k] = (double)m.n * m.n * m.n * c.L * (m.ph ? 1.0 : 2.0);
            static const double px[] = {64, 144, 256, 576}, py[] = {0, 0.245, 0.30, 0.67};
            double a = py[3];
            if (m.n <= px[0]) a = 0.0;
            for (int q = 0; q < 3; ++q)
                if (m.n > px[q] && m.n <= px[q + 1])
                    a = py[q] + (py[q + 1] - py[q]) * (m.n - px[q]) / (px[q + 1] - px[q]);
            an[k] = a;
        }
        auto span = [&](int cc, int k) {   /* predicted time of the slowest chain */
            double t = 0.0;
            for (int i = 0; i < k; ++i)
                t = std::max(t, w[i] / (1.0 + an[i] * std::log2((double)cc)));
            if (k < (int)nc) t = std::max(t, w[k]);
            return t;
        };
        const int want = e->desc.chain_ctas;
        if (want > 1) {
            int fit = 0;
            CU(dq::cluster_fit(want, e->smem, &fit));
            const int k = e->desc.cluster_chains > 0 ? std::min(e->desc.cluster_chains, (int)nc)
                                                     : (int)nc;
            const int tot = k + ((int)nc - k + want - 1) / want;
            if (fit < 1)
                return set_err("dqmc_engine_prepare: a cluster of %d CTAs with %zu B of shared "
                               "memory each cannot be resident on this device",
                               want, e->smem);
            e->cl = want;
            e->ncoop = k;
            e->nclus = tot;
        } else if (want == 0 && e->per_sm == 1 && maxn >= 128) {
            double best = w.empty() ? 0.0 : w[0];
            for (int cc = DQMC_MAX_CHAIN_CTAS; cc >= 2; --cc) {
                int fit = 0;
                if (dq::cluster_fit(cc, e->smem, &fit) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                for (int k = 1; k <= (int)nc; ++k) {
                    const int tot = k + ((int)nc - k + cc - 1) / cc;
                    if ((long)tot * cc > nsm || tot > fit) continue;
                    const double t = span(cc, k);
                    if (t < 0.97 * best) {
                        best = t;
                        e->cl = cc;
                        e->ncoop = k;
                        e->nclus = tot;
                    }
                }
            }
        }
    }
    dq::k_init<<<(unsigned)nc, DQMC_NT, e->smem, e->stream>>>(e->dchains, e->dmodels);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(e->stream));
    e->prepared = true;
    return 0;
}

static int check_prepared(dqmc_engine *e, const char *who)
{
    if (!e || !e->prepared) return set_err("%s: engine not prepared", who);
    if (cudaSetDevice(e->desc.device) != cudaSuccess) return set_err("%s: cudaSetDevice", who);
    return 0;
}

static int kflags(const dqmc_engine *e)
{
    return ((e->desc.drift & DQMC_DRIFT_SCRATCH) ? dq::KF_SDRIFT : 0) |
           (e->desc.precision == DQMC_PREC_MIXED ? dq::KF_MIXED : 0);
}

static int chain_ok(dqmc_engine *e, int chain, const char *who);

/* Moves every chain's device UDV scale records to its host list (after
 * each sweep launch when the records are on: a launch of one sweep fills
 * at most udv_cap records per chain). */
static int udv_drain(dqmc_engine *e)
{
    if (!e->desc.udv_diag) return 0;
    CU(cudaStreamSynchronize(e->stream));
    for (size_t c = 0; c < e->chains.size(); ++c) {
        int cnt[3];   /* udv_cap, udv_n, udv_lost */
        CU(cudaMemcpy(cnt, (char *)(e->dchains + c) + offsetof(DqmcChainDev, udv_cap),
                      sizeof cnt, cudaMemcpyDeviceToHost));
        if (cnt[2]) return set_err("UDV scale records lost (chain %zu)", c);
        if (cnt[1] <= 0) continue;
        std::vector<double> &h = e->chains[c].udv;
        const size_t old = h.size(), add = (size_t)cnt[1] * DQMC_UDV_RECORD_DOUBLES;
        h.resize(old + add);
        CU(cudaMemcpy(h.data() + old, e->hdev[c].udvrec, add * 8, cudaMemcpyDeviceToHost));
        const int zero = 0;
        CU(cudaMemcpy((char *)(e->dchains + c) + offsetof(DqmcChainDev, udv_n), &zero,
                      sizeof zero, cudaMemcpyHostToDevice));
    }
    return 0;
}

int dqmc_sweep(dqmc_engine *e, int nsweeps)
{
    if (check_prepared(e, "dqmc_sweep")) return 1;
    if (nsweeps <= 0) return 0;
    const unsigned nc = (unsigned)e->chains.size();
    /* with UDV scale records, one launch per sweep, drained in between */
    const int per = e->desc.udv_diag ? 1 : nsweeps;
    for (int done = 0; done < nsweeps; done += per) {
        ev_begin(e, 0);
        if (e->cl > 1)
            CU(dq::launch_sweep_cluster((unsigned)e->nclus, e->cl, e->smem, e->stream,
                                        e->dchains, e->dmodels, kflags(e), per, e->dorder,
                                        e->ncoop, (int)nc));
        else if (e->per_sm == 2)
            dq2x::launch_sweep(nc, e->smem2, e->stream, e->dchains, e->dmodels, kflags(e), per,
                                 e->dorder);
        else
            dq::launch_sweep(nc, e->smem, e->stream, e->dchains, e->dmodels, kflags(e), per,
                               e->dorder);
        ev_end(e);
        CU(cudaGetLastError());
        if (udv_drain(e)) return 1;
    }
    return 0;
}

int dqmc_read_udv_records(dqmc_engine *e, int chain, double *out, int max_records)
{
    if (chain_ok(e, chain, "dqmc_read_udv_records")) return -1;
    if (!e->desc.udv_diag) {
        set_err("dqmc_read_udv_records: engine created without udv_diag");
        return -1;
    }
    if (max_records < 0 || (max_records > 0 && !out)) {
        set_err("dqmc_read_udv_records: bad output buffer");
        return -1;
    }
    std::vector<double> &h = e->chains[chain].udv;
    const int have = (int)(h.size() / DQMC_UDV_RECORD_DOUBLES);
    const int k = have < max_records ? have : max_records;
    const size_t nd = (size_t)k * DQMC_UDV_RECORD_DOUBLES;
    std::copy(h.begin(), h.begin() + nd, out);
    h.erase(h.begin(), h.begin() + nd);
    return k;
}

int dqmc_read_green_log(dqmc_engine *e, int chain, double *out, int max_snapshots)
{
    if (chain_ok(e, chain, "dqmc_read_green_log")) return -1;
    if (e->desc.green_log <= 0) {
        set_err("dqmc_read_green_log: engine created without green_log");
        return -1;
    }
    if (max_snapshots < 0 || (max_snapshots > 0 && !out)) {
        set_err("dqmc_read_green_log: bad output buffer");
        return -1;
    }
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) {
        set_err("dqmc_read_green_log: cudaStreamSynchronize");
        return -1;
    }
    const DqmcChainDev &h = e->hdev[chain];
    char *dc = (char *)(e->dchains + chain);
    int cnt[2];   /* glog_cap, glog_n */
    if (cudaMemcpy(cnt, dc + offsetof(DqmcChainDev, glog_cap), sizeof cnt,
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err("dqmc_read_green_log: cudaMemcpy");
        return -1;
    }
    const int k = cnt[1] < max_snapshots ? cnt[1] : max_snapshots;
    const size_t nn = (size_t)h.n * h.n;
    if (k > 0 && cudaMemcpy(out, h.glog, (size_t)k * nn * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err("dqmc_read_green_log: cudaMemcpy");
        return -1;
    }
    const int zero[2] = {0, 0};   /* glog_n, glog_lost */
    if (cudaMemcpy(dc + offsetof(DqmcChainDev, glog_n), zero, sizeof zero,
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        set_err("dqmc_read_green_log: cudaMemcpy");
        return -1;
    }
    return k;
}

int dqmc_sweep_measure(dqmc_engine *e, int nsweeps, int bin)
{
    if (check_prepared(e, "dqmc_sweep_measure")) return 1;
    if (bin < 0 || bin >= e->nbin) return set_err("dqmc_sweep_measure: bin %d out of range", bin);
    const unsigned nc = (unsigned)e->chains.size();
    for (int s = 0; s < nsweeps; ++s) {
        const int f = kflags(e) | dq::KF_MEASURE;
        ev_begin(e, 0);
        if (e->cl > 1)
            CU(dq::launch_sweep_cluster((unsigned)e->nclus, e->cl, e->smem, e->stream,
                                        e->dchains, e->dmodels, f, 1, e->dorder, e->ncoop,
                                        (int)nc));
        else if (e->per_sm == 2)
            dq2x::launch_sweep(nc, e->smem2, e->stream, e->dchains, e->dmodels, f, 1, e->dorder);
        else
            dq::launch_sweep(nc, e->smem, e->stream, e->dchains, e->dmodels, f, 1, e->dorder);
        ev_end(e);
        if (udv_drain(e)) return 1;
        ev_begin(e, 1);
        dq::launch_measure(nc, e->msmem, e->stream, e->dchains, e->dmodels, bin);
        ev_end(e);
    }
    CU(cudaGetLastError());
    return 0;
}

int dqmc_kernel_timing(dqmc_engine *e, int enable)
{
    if (!e) return set_err("dqmc_kernel_timing: null engine");
    CU(cudaSetDevice(e->desc.device));
    CU(cudaStreamSynchronize(e->stream));
    for (cudaEvent_t v : e->ev) cudaEventDestroy(v);
    e->ev.clear();
    e->ev_kind.clear();
    e->timing = enable != 0;
    return 0;
}

int dqmc_kernel_times(dqmc_engine *e, double *sweep_ms, int *sweep_launches,
                      double *measure_ms, int *measure_launches)
{
    if (!e) return set_err("dqmc_kernel_times: null engine");
    CU(cudaSetDevice(e->desc.device));
    CU(cudaStreamSynchronize(e->stream));
    double t[2] = {0.0, 0.0};
    int c[2] = {0, 0};
    for (size_t i = 0; i + 1 < e->ev.size(); i += 2) {
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, e->ev[i], e->ev[i + 1]));
        const int k = e->ev_kind[i];
        t[k] += ms;
        c[k] += 1;
    }
    if (sweep_ms) *sweep_ms = t[0];
    if (sweep_launches) *sweep_launches = c[0];
    if (measure_ms) *measure_ms = t[1];
    if (measure_launches) *measure_launches = c[1];
    return 0;
}

int dqmc_timer_mark(dqmc_engine *e, int which)
{
    if (!e || which < 0 || which > 1) return set_err("dqmc_timer_mark: bad arguments");
    CU(cudaSetDevice(e->desc.device));
    if (!e->mark[which]) CU(cudaEventCreate(&e->mark[which]));
    CU(cudaEventRecord(e->mark[which], e->stream));
    return 0;
}

int dqmc_timer_elapsed(dqmc_engine *e, double *ms)
{
    if (!e || !e->mark[0] || !e->mark[1]) return set_err("dqmc_timer_elapsed: marks missing");
    CU(cudaEventSynchronize(e->mark[1]));
    float f = 0.f;
    CU(cudaEventElapsedTime(&f, e->mark[0], e->mark[1]));
    *ms = f;
    return 0;
}

int dqmc_synchronize(dqmc_engine *e)
{
    if (!e) return set_err("dqmc_synchronize: null engine");
    CU(cudaSetDevice(e->desc.device));
    CU(cudaStreamSynchronize(e->stream));
    return 0;
}

int dqmc_chain_count(const dqmc_engine *e) { return e ? (int)e->chains.size() : 0; }

int dqmc_engine_residency(const dqmc_engine *e, int *ctas_per_sm, int *chain_ctas,
                          int *cluster_chains)
{
    if (!e || !e->prepared) return set_err("dqmc_engine_residency: engine not prepared");
    if (ctas_per_sm) *ctas_per_sm = e->per_sm;
    if (chain_ctas) *chain_ctas = e->cl;
    if (cluster_chains) *cluster_chains = e->cl > 1 ? e->ncoop : 0;
    return 0;
}

int dqmc_chain_dims(const dqmc_engine *e, int chain, int *n, int *L)
{
    if (!e || chain < 0 || chain >= (int)e->chains.size()) return set_err("bad chain");
    if (n) *n = e->models[e->chains[chain].model].n;
    if (L) *L = e->chains[chain].L;
    return 0;
}

static int chain_ok(dqmc_engine *e, int chain, const char *who)
{
    if (check_prepared(e, who)) return 1;
    if (chain < 0 || chain >= (int)e->chains.size()) return set_err("%s: bad chain %d", who, chain);
    /* engines on different devices may be driven from one host thread */
    if (cudaSetDevice(e->desc.device) != cudaSuccess) return set_err("%s: cudaSetDevice", who);
    return 0;
}

int dqmc_read_green(dqmc_engine *e, int chain, double *G)
{
    if (chain_ok(e, chain, "dqmc_read_green")) return 1;
    const int n = e->hdev[chain].n;
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(G, e->hdev[chain].G, (size_t)n * n * 8, cudaMemcpyDeviceToHost));
    return 0;
}

int dqmc_read_green_down(dqmc_engine *e, int chain, double *G)
{
    if (chain_ok(e, chain, "dqmc_read_green_down")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    const int n = d.n;
    CU(cudaStreamSynchronize(e->stream));
    if (d.ns == 2) {
        CU(cudaMemcpy(G, d.Gd, (size_t)n * n * 8, cudaMemcpyDeviceToHost));
        return 0;
    }
    /* PH path: G_down = I - P G_up^T P (dqmc_map_ph_down, src/dqmc.c:9-17) */
    std::vector<double> gu((size_t)n * n);
    CU(cudaMemcpy(gu.data(), d.G, gu.size() * 8, cudaMemcpyDeviceToHost));
    const std::vector<int> &p = e->models[e->chains[chain].model].bipart;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            G[i + (size_t)j * n] = (i == j ? 1.0 : 0.0) - (double)(p[i] * p[j]) * gu[j + (size_t)i * n];
    return 0;
}

int dqmc_read_field(dqmc_engine *e, int chain, signed char *field)
{
    if (chain_ok(e, chain, "dqmc_read_field")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(field, d.field, (size_t)d.L * d.n, cudaMemcpyDeviceToHost));
    return 0;
}

int dqmc_write_field(dqmc_engine *e, int chain, const signed char *field)
{
    if (chain_ok(e, chain, "dqmc_write_field")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    for (size_t k = 0; k < (size_t)d.L * d.n; ++k)
        if (field[k] != 1 && field[k] != -1) return set_err("field entries must be +/-1");
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(d.field, field, (size_t)d.L * d.n, cudaMemcpyHostToDevice));
    dq::k_init<<<1, DQMC_NT, e->smem, e->stream>>>(e->dchains + chain, e->dmodels);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(e->stream));
    return 0;
}

int dqmc_write_green(dqmc_engine *e, int chain, const double *G)
{
    if (chain_ok(e, chain, "dqmc_write_green")) return 1;
    if (!G) return set_err("dqmc_write_green: null G");
    const DqmcChainDev &d = e->hdev[chain];
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(d.G, G, (size_t)d.n * d.n * 8, cudaMemcpyHostToDevice));
    return 0;
}

int dqmc_write_rng(dqmc_engine *e, int chain, const uint64_t rng[4])
{
    if (chain_ok(e, chain, "dqmc_write_rng")) return 1;
    if (!rng || (rng[0] | rng[1] | rng[2] | rng[3]) == 0)
        return set_err("dqmc_write_rng: the all-zero xoshiro state is not valid");
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy((char *)(e->dchains + chain) + offsetof(DqmcChainDev, rng), rng,
                  4 * sizeof(uint64_t), cudaMemcpyHostToDevice));
    return 0;
}

int dqmc_read_counters(dqmc_engine *e, int chain, dqmc_chain_counters *out)
{
    if (chain_ok(e, chain, "dqmc_read_counters")) return 1;
    DqmcChainDev d;
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(&d, e->dchains + chain, sizeof d, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->attempts = d.attempts;
    out->accepted = d.accepted;
    out->sweeps = d.sweeps;
    out->status = d.status;
    out->sign = d.sign;
    out->drift_max = d.drift_max;
    out->drift_mean = d.drift_count ? d.drift_sum / (double)d.drift_count : 0.0;
    out->drift_samples = d.drift_count;
    out->scratch_drift_max = d.sdrift_max;
    out->scratch_drift_mean = d.sdrift_count ? d.sdrift_sum / (double)d.sdrift_count : 0.0;
    out->scratch_drift_samples = d.sdrift_count;
    out->scratch_drift_max_tau = d.sdrift_max_tau;
    out->scratch_drift_max_sweep = d.sdrift_max_sweep;
    for (int i = 0; i < 4; ++i) out->rng[i] = d.rng[i];
    return 0;
}

int dqmc_read_bins(dqmc_engine *e, int chain, double *scalars, double *szz, double *sperp)
{
    if (chain_ok(e, chain, "dqmc_read_bins")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    const HModel &m = e->models[e->chains[chain].model];
    CU(cudaStreamSynchronize(e->stream));
    if (scalars)
        CU(cudaMemcpy(scalars, d.bins, (size_t)e->nbin * DQMC_BIN_FIELDS * 8,
                      cudaMemcpyDeviceToHost));
    if (szz && m.nq_zz)
        CU(cudaMemcpy(szz, d.bins_zz, (size_t)e->nbin * m.nq_zz * 8, cudaMemcpyDeviceToHost));
    if (sperp && m.nq_perp)
        CU(cudaMemcpy(sperp, d.bins_perp, (size_t)e->nbin * m.nq_perp * 8,
                      cudaMemcpyDeviceToHost));
    return 0;
}

int dqmc_read_profile(dqmc_engine *e, int chain, unsigned long long *cycles, int count)
{
    if (chain_ok(e, chain, "dqmc_read_profile")) return 1;
    DqmcChainDev d;
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(&d, e->dchains + chain, sizeof d, cudaMemcpyDeviceToHost));
    for (int i = 0; i < count && i < DQMC_PH_COUNT; ++i) cycles[i] = d.prof[i];
    return 0;
}

int dqmc_read_profile_calls(dqmc_engine *e, int chain, unsigned long long *calls, int count)
{
    if (chain_ok(e, chain, "dqmc_read_profile_calls")) return 1;
    DqmcChainDev d;
    CU(cudaStreamSynchronize(e->stream));
    CU(cudaMemcpy(&d, e->dchains + chain, sizeof d, cudaMemcpyDeviceToHost));
    for (int i = 0; i < count && i < DQMC_PH_COUNT; ++i) calls[i] = d.pcalls[i];
    return 0;
}

double dqmc_clock_hz(dqmc_engine *e)
{
    int khz = 0;
    if (!e || cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, e->desc.device) != cudaSuccess)
        return 0.0;
    return 1e3 * khz;
}

int dqmc_clear_bins(dqmc_engine *e)
{
    if (check_prepared(e, "dqmc_clear_bins")) return 1;
    for (size_t k = 0; k < e->chains.size(); ++k) {
        const DqmcChainDev &d = e->hdev[k];
        const HModel &m = e->models[e->chains[k].model];
        CU(cudaMemsetAsync(d.bins, 0, (size_t)e->nbin * DQMC_BIN_FIELDS * 8, e->stream));
        if (m.nq_zz) CU(cudaMemsetAsync(d.bins_zz, 0, (size_t)e->nbin * m.nq_zz * 8, e->stream));
        if (m.nq_perp)
            CU(cudaMemsetAsync(d.bins_perp, 0, (size_t)e->nbin * m.nq_perp * 8, e->stream));
    }
    CU(cudaStreamSynchronize(e->stream));
    return 0;
}

int dqmc_green_from_scratch(dqmc_engine *e, int chain, int l0, double *G, int *det_sign)
{
    if (chain_ok(e, chain, "dqmc_green_from_scratch")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    if (l0 < 0 || l0 >= d.L) return set_err("l0 out of range");
    double *dG = nullptr;
    int *ddet = nullptr;
    CU(cudaMalloc(&dG, (size_t)d.n * d.n * 8 + 16));
    ddet = (int *)(dG + (size_t)d.n * d.n);
    dq::k_scratch<<<1, DQMC_NT, e->smem, e->stream>>>(e->dchains, e->dmodels, chain, l0, dG, ddet);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err == cudaSuccess) err = cudaMemcpy(G, dG, (size_t)d.n * d.n * 8, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(det_sign, ddet, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dG);
    if (err != cudaSuccess) return set_err("dqmc_green_from_scratch: %s", cudaGetErrorString(err));
    return 0;
}

int dqmc_wrap_green(dqmc_engine *e, int chain, int l, double *G)
{
    if (chain_ok(e, chain, "dqmc_wrap_green")) return 1;
    const DqmcChainDev &d = e->hdev[chain];
    if (l < 0 || l >= d.L) return set_err("l out of range");
    double *dG = nullptr;
    const size_t bytes = (size_t)d.n * d.n * 8;
    CU(cudaMalloc(&dG, bytes));
    cudaError_t err = cudaMemcpy(dG, G, bytes, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        dq::k_wrap<<<1, DQMC_NT, e->smem, e->stream>>>(e->dchains, e->dmodels, chain, l, dG,
                                                       kflags(e));
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err == cudaSuccess) err = cudaMemcpy(G, dG, bytes, cudaMemcpyDeviceToHost);
    cudaFree(dG);
    if (err != cudaSuccess) return set_err("dqmc_wrap_green: %s", cudaGetErrorString(err));
    return 0;
}

/* Host sign of det(U) for a small orthogonal U (partial-pivot LU). */
static int host_det_sign(int n, const double *U)
{
    std::vector<double> a(U, U + (size_t)n * n);
    int s = 1;
    for (int j = 0; j < n; ++j) {
        int p = j;
        for (int i = j + 1; i < n; ++i)
            if (std::fabs(a[i + (size_t)j * n]) > std::fabs(a[p + (size_t)j * n])) p = i;
        if (a[p + (size_t)j * n] == 0.0) return 0;
        if (p != j) {
            s = -s;
            for (int c = 0; c < n; ++c) std::swap(a[j + (size_t)c * n], a[p + (size_t)c * n]);
        }
        if (a[j + (size_t)j * n] < 0) s = -s;
        for (int i = j + 1; i < n; ++i) {
            const double f = a[i + (size_t)j * n] / a[j + (size_t)j * n];
            for (int c = j + 1; c < n; ++c) a[i + (size_t)c * n] -= f * a[j + (size_t)c * n];
        }
    }
    return s;
}

int dqmc_udv_green(int device, int n, const double *U, const double *D, const double *T,
                   double *G, int *det_sign)
{
    if (n <= 0 || n > DQMC_MAX_N || !U || !D || !T || !G || !det_sign)
        return set_err("dqmc_udv_green: bad arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err("dqmc_udv_green: no CUDA device");
    CU(cudaSetDevice(device));
    const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
    /* signed D -> positive D with the signs moved into U's columns */
    std::vector<double> slot(usz, 0.0);
    int dsign = host_det_sign(n, U);
    for (int j = 0; j < n; ++j) {
        const double sgn = D[j] < 0 ? -1.0 : 1.0;
        if (D[j] < 0) dsign = -dsign;
        for (int i = 0; i < n; ++i) slot[i + (size_t)j * n] = U[i + (size_t)j * n] * sgn;
        slot[2 * nn + j] = std::log(std::fabs(D[j]));
    }
    std::memcpy(slot.data() + nn, T, nn * 8);
    slot[2 * nn + n] = dsign;
    const size_t twsz = (size_t)((n + DQMC_QNB - 1) / DQMC_QNB) * DQMC_QNB * DQMC_QNB;
    char *buf = nullptr;
    const size_t bytes = usz * 8 + (3 * nn + twsz) * 8 + nn * 8 + 64;
    CU(cudaMalloc(&buf, bytes));
    double *dslot = (double *)buf;
    double *ws = dslot + usz;
    double *dG = ws + 3 * nn + twsz;
    int *ddet = (int *)(dG + nn);
    cudaError_t err = cudaMemcpy(dslot, slot.data(), usz * 8, cudaMemcpyHostToDevice);
    const size_t sm = dq::smem_bytes(n, 1);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(dq::k_udv_green, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sm);
    if (err == cudaSuccess) {
        dq::k_udv_green<<<1, DQMC_NT, sm>>>(n, dslot, ws, dG, ddet);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err == cudaSuccess) err = cudaMemcpy(G, dG, nn * 8, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(det_sign, ddet, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (err != cudaSuccess) return set_err("dqmc_udv_green: %s", cudaGetErrorString(err));
    return 0;
}

/* caller factor -> engine slot: signs of D into U's columns, log|D| + off */
static void host_udv_slot(int n, const double *U, const double *D, const double *T, double off,
                          std::vector<double> &slot)
{
    const size_t nn = (size_t)n * n;
    slot.assign(DQMC_UDV_SIZE(n), 0.0);
    int dsign = host_det_sign(n, U);
    for (int j = 0; j < n; ++j) {
        const double sgn = D[j] < 0 ? -1.0 : 1.0;
        if (D[j] < 0) dsign = -dsign;
        for (int i = 0; i < n; ++i) slot[i + (size_t)j * n] = U[i + (size_t)j * n] * sgn;
        slot[2 * nn + j] = std::log(std::fabs(D[j])) + off;
        slot[2 * nn + n + 2 + j] = j;   /* identity column permutation */
    }
    std::memcpy(slot.data() + nn, T, nn * 8);
    slot[2 * nn + n] = dsign;
}

int dqmc_udv_green2(int device, int n, const double *UL, const double *DL, const double *TL,
                    double off_L, const double *UR, const double *DR, const double *TR,
                    double off_R, double *G, int *det_sign)
{
    if (n <= 0 || n > DQMC_MAX_N || !UL || !DL || !TL || !UR || !DR || !TR || !G || !det_sign ||
        !std::isfinite(off_L) || !std::isfinite(off_R))
        return set_err("dqmc_udv_green2: bad arguments");
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i)
            if (TR[i + (size_t)j * n] != (i == j ? 1.0 : 0.0))
                return set_err("dqmc_udv_green2: T_R must be unit upper triangular");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err("dqmc_udv_green2: no CUDA device");
    CU(cudaSetDevice(device));
    const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
    std::vector<double> ls, rs;
    host_udv_slot(n, UL, DL, TL, off_L, ls);
    host_udv_slot(n, UR, DR, TR, off_R, rs);
    const size_t twsz = (size_t)((n + DQMC_QNB - 1) / DQMC_QNB) * DQMC_QNB * DQMC_QNB;
    char *buf = nullptr;
    const size_t bytes = 2 * usz * 8 + (4 * nn + twsz) * 8 + nn * 8 + 64;
    CU(cudaMalloc(&buf, bytes));
    double *dl = (double *)buf, *dr = dl + usz, *ws = dr + usz;
    double *dG = ws + 4 * nn + twsz;
    int *ddet = (int *)(dG + nn);
    cudaError_t err = cudaMemcpy(dl, ls.data(), usz * 8, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dr, rs.data(), usz * 8, cudaMemcpyHostToDevice);
    const size_t sm = dq::smem_bytes(n, 1);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(dq::k_udv_green2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sm);
    if (err == cudaSuccess) {
        dq::k_udv_green2<<<1, DQMC_NT, sm>>>(n, dl, dr, ws, dG, ddet);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err == cudaSuccess) err = cudaMemcpy(G, dG, nn * 8, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(det_sign, ddet, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (err != cudaSuccess) return set_err("dqmc_udv_green2: %s", cudaGetErrorString(err));
    return 0;
}

}  /* extern "C" */
