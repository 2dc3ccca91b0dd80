/* CTA-level FP64 building blocks for the BSS sweep.
 *
 * One CTA of DQMC_NT threads owns one Markov chain and calls these routines
 * with every thread; operands live in global memory (L2-resident for the
 * sizes this engine targets) and are staged through shared memory.  Nothing
 * here waits on another CTA, so a launch can never hang on a peer.
 */
#pragma once
#include <math.h>
#include <stdint.h>

#include "dqmc_common.h"

/* The device code is compiled twice (dqmc_k1.cu, dqmc_k2.cu) into distinct
 * namespaces: one CTA per SM with the full register file, and two CTAs per
 * SM (128 registers, narrower reflector chunks) for large batches. */
#ifndef DQMC_NS
#define DQMC_NS dq
#endif
#ifndef DQMC_MINB
#define DQMC_MINB 1
#endif
#ifndef DQMC_WCOLS
#define DQMC_WCOLS 256
#endif

namespace DQMC_NS {

constexpr int NT = DQMC_NT;
constexpr int NW = NT / 32;
constexpr int QNB = DQMC_QNB;
constexpr int WCOLS = DQMC_WCOLS;  /* column chunk of a block-reflector update */
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

/* Block-wide reduction; red needs 33 doubles of shared memory. */
template <bool MAX>
__device__ double block_reduce(double v, double *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = MAX ? warp_max(v) : warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = (lane < NW) ? red[lane] : (MAX ? 0.0 : 0.0);
        r = MAX ? warp_max(r) : warp_sum(r);
        if (lane == 0) red[32] = r;
    }
    __syncthreads();
    return red[32];
}

/* ------------------------------------------------------------------ GEMM */
/* Tile configuration: BM x BN output tile, BK-deep k slices, each thread
 * owns a TM x TN register tile at rows ty + TY*r, cols tx + TX*c (strided so
 * that shared-memory reads are broadcast or conflict-free). */
template <int BM_, int BN_, int BK_, int TM_, int TN_, bool MMA_ = false, int WM_ = 2>
struct Tile {
    static constexpr int BM = BM_, BN = BN_, BK = BK_, TM = TM_, TN = TN_;
    static constexpr bool MMA = MMA_;
    /* DMMA layout: WM x WN warps, each FM x FN m16n8 fragments */
    static constexpr int WM = WM_, WN = NW / WM_;
    static constexpr int FM = BM / (WM * 16), FN = BN / (WN * 8);
    static_assert(!MMA || (FM * WM * 16 == BM && FN * WN * 8 == BN && TM == FM * FN && TN == 4),
                  "DMMA tile shape");
    static constexpr int TX = BN / TN, TY = BM / TM;
    static_assert(MMA || TX * TY == NT, "thread grid must cover the CTA");
    /* SIMT tiles pad by one (broadcast/conflict-free reads); DMMA tiles pad
     * rows to 8 mod 32 banks so a fragment load is two wavefronts. */
    static constexpr int AP = MMA ? BM + 4 : BM + 1, BP = MMA ? BN + 4 : BN + 1;
    static constexpr int AL = BM * BK / NT, BL = BK * BN / NT;
    static_assert(AL * NT == BM * BK && BL * NT == BK * BN, "load split");
    static constexpr int SMEM = 2 * BK * AP + 2 * BK * BP;
};

using TSq = Tile<64, 64, 16, 4, 4>;     /* square-ish products            */
using TSm = Tile<32, 32, 16, 2, 2>;     /* small lattices                 */
using TWide = Tile<16, 128, 16, 1, 8>;  /* 16-row results (V^T X, trsm)    */
/* FP64 tensor-core tiles: 64 x 64 with 8 warps as 2 (M) x 4 (N), warp tile
 * 32 x 16 = 2 x 2 mma.m16n8k4 fragments; 16 x 128 with 1 x 8 warps. */
using TMma = Tile<64, 64, 16, 4, 4, true, 2>;
using TMmaWide = Tile<16, 128, 16, 2, 4, true, 1>;
/* 128 x 64 with 2 x 4 warps: 4 x 2 fragments per warp, twice the
 * independent accumulators per warp (needs the full register file) */
using TMmaBig = Tile<128, 64, 16, 8, 4, true, 2>;
#if DQMC_MINB == 1
using TSquare = TMmaBig;
#else
using TSquare = TMma;
#endif
constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int GEMM_SMEM = cmax(cmax(TWide::SMEM, TSq::SMEM),
                               cmax(cmax(TMma::SMEM, TMmaWide::SMEM), TSquare::SMEM));

/* D = A(16x4) B(4x8) + C, FP64 on the tensor cores (sm_90+ shape). */
__device__ __forceinline__ void dmma_16x8x4(double *c, double a0, double a1, double b0)
{
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

/* C(M x N) <- epilogue of sum_k la(i,k) * lb(k,j).
 * la/lb are element loaders (any transpose, scaling or gather lives there);
 * AMF: consecutive i are contiguous for la; BKF: consecutive k contiguous
 * for lb -- only affects which thread fetches which element (coalescing).
 * Epilogue: st(i, j, acc), or for RMW = true st(i, j, acc, c) with
 * c = lc(i, j) fetched one output tile ahead (read-modify-write products
 * such as G -= Z Y overlap the C reads with the previous tile's math).
 * The (tile, k-slice) sequence is one flat software pipeline: the next
 * slice -- possibly of the next output tile -- is fetched into registers
 * while the current one is multiplied, so short-K products stay busy.
 * Every thread of the CTA must call this. */
template <class T, bool AMF, bool BKF, bool RMW, class LA, class LB, class LC, class ST>
__device__ void gemm_core(int M, int N, int K, LA la, LB lb, LC lc, ST st, double *sm)
{
    constexpr int BM = T::BM, BN = T::BN, BK = T::BK, TM = T::TM, TN = T::TN;
    constexpr int TX = T::TX, TY = T::TY, AP = T::AP, BP = T::BP;
    constexpr int AL = T::AL, BL = T::BL;
    double *As = sm;
    double *Bs = sm + 2 * BK * AP;
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int lane = tid & 31, warp = tid >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp % T::WM, wn = warp / T::WM;
    const int tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
    const int nk = (K + BK - 1) / BK;
    const int total = tm * tn * nk;
    (void)tn;
    /* output coordinates of accumulator (r, c) of this thread in a tile */
    auto out_ij = [&](int r, int c, int &i, int &j) {
        if constexpr (T::MMA) {
            const int mi = r / T::FN, ni = r % T::FN;
            i = wm * (T::FM * 16) + mi * 16 + gid + (c >> 1) * 8;
            j = wn * (T::FN * 8) + ni * 8 + 2 * tig + (c & 1);
        } else {
            i = ty + TY * r;
            j = tx + TX * c;
        }
    };
    __syncthreads();
    if (total == 0) return;
    double ra[AL], rb[BL];
    /* fetch position (tile origin and k offset), advanced incrementally */
    int fm0 = 0, fn0 = 0, fk0 = 0;
    auto advance = [&](int &m0, int &n0, int &k0) {
        k0 += BK;
        if (k0 >= nk * BK) {
            k0 = 0;
            m0 += BM;
            if (m0 >= tm * BM) {
                m0 = 0;
                n0 += BN;
            }
        }
    };
    auto fetch = [&]() {
        const int m0 = fm0, n0 = fn0, k0 = fk0;
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = tid + q * NT;
            const int i = AMF ? e % BM : e / BK, k = AMF ? e / BM : e % BK;
            const int gi = m0 + i, gk = k0 + k;
            ra[q] = (gi < M && gk < K) ? la(gi, gk) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = tid + q * NT;
            const int k = BKF ? e % BK : e / BN, j = BKF ? e / BK : e % BN;
            const int gk = k0 + k, gj = n0 + j;
            rb[q] = (gk < K && gj < N) ? lb(gk, gj) : 0.0;
        }
    };
    auto put = [&](int buf) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = tid + q * NT;
            const int i = AMF ? e % BM : e / BK, k = AMF ? e / BM : e % BK;
            As[buf * BK * AP + k * AP + i] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = tid + q * NT;
            const int k = BKF ? e % BK : e / BN, j = BKF ? e / BK : e % BN;
            Bs[buf * BK * BP + k * BP + j] = rb[q];
        }
    };
    double cpre[TM][TN];
    auto fetch_c = [&](int m0, int n0) {
#pragma unroll
        for (int r = 0; r < TM; ++r)
#pragma unroll
            for (int c = 0; c < TN; ++c) {
                int i, j;
                out_ij(r, c, i, j);
                i += m0;
                j += n0;
                cpre[r][c] = (i < M && j < N) ? lc(i, j) : 0.0;
            }
    };
    double acc[TM][TN];
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[r][c] = 0.0;
    if constexpr (RMW) fetch_c(0, 0);
    fetch();
    put(0);
    __syncthreads();
    int cm0 = 0, cn0 = 0, ck0 = 0;   /* position being multiplied */
    advance(fm0, fn0, fk0);
    for (int it = 0; it < total; ++it) {
        const int cur = it & 1;
        if (it + 1 < total) fetch();
        const double *a = As + cur * BK * AP;
        const double *b = Bs + cur * BK * BP;
        if constexpr (T::MMA) {
            constexpr int FM = T::FM, FN = T::FN;
#pragma unroll
            for (int kk = 0; kk < BK; kk += 4) {
                double a0[FM], a1[FM], b0[FN];
#pragma unroll
                for (int mi = 0; mi < FM; ++mi) {
                    const int i = wm * (FM * 16) + mi * 16 + gid;
                    a0[mi] = a[(kk + tig) * AP + i];
                    a1[mi] = a[(kk + tig) * AP + i + 8];
                }
#pragma unroll
                for (int ni = 0; ni < FN; ++ni)
                    b0[ni] = b[(kk + tig) * BP + wn * (FN * 8) + ni * 8 + gid];
#pragma unroll
                for (int mi = 0; mi < FM; ++mi)
#pragma unroll
                    for (int ni = 0; ni < FN; ++ni)
                        dmma_16x8x4(acc[mi * FN + ni], a0[mi], a1[mi], b0[ni]);
            }
        } else {
#pragma unroll
            for (int k = 0; k < BK; ++k) {
                double av[TM], bv[TN];
#pragma unroll
                for (int r = 0; r < TM; ++r) av[r] = a[k * AP + ty + TY * r];
#pragma unroll
                for (int c = 0; c < TN; ++c) bv[c] = b[k * BP + tx + TX * c];
#pragma unroll
                for (int r = 0; r < TM; ++r)
#pragma unroll
                    for (int c = 0; c < TN; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
            }
        }
        if (ck0 == (nk - 1) * BK) {
            const int m0 = cm0, n0 = cn0;
            double cv[TM][TN];
            if constexpr (RMW) {
#pragma unroll
                for (int r = 0; r < TM; ++r)
#pragma unroll
                    for (int c = 0; c < TN; ++c) cv[r][c] = cpre[r][c];
                if (it + 1 < total) fetch_c(fm0, fn0);
            }
#pragma unroll
            for (int r = 0; r < TM; ++r)
#pragma unroll
                for (int c = 0; c < TN; ++c) {
                    int i, j;
                    out_ij(r, c, i, j);
                    i += m0;
                    j += n0;
                    if (i < M && j < N) {
                        if constexpr (RMW)
                            st(i, j, acc[r][c], cv[r][c]);
                        else
                            st(i, j, acc[r][c]);
                    }
                    acc[r][c] = 0.0;
                }
        }
        if (it + 1 < total) put(cur ^ 1);
        advance(cm0, cn0, ck0);
        advance(fm0, fn0, fk0);
        __syncthreads();
    }
}

template <class T, bool AMF, bool BKF, class LA, class LB, class ST>
__device__ __forceinline__ void gemm(int M, int N, int K, LA la, LB lb, ST st, double *sm)
{
    gemm_core<T, AMF, BKF, false>(
        M, N, K, la, lb, [](int, int) { return 0.0; }, st, sm);
}

/* C(i,j) <- st(i, j, sum_k a b, C(i,j)) with C read through lc */
template <class T, bool AMF, bool BKF, class LA, class LB, class LC, class ST>
__device__ __forceinline__ void gemm_rmw(int M, int N, int K, LA la, LB lb, LC lc, ST st,
                                         double *sm)
{
    gemm_core<T, AMF, BKF, true>(M, N, K, la, lb, lc, st, sm);
}

/* Square-product dispatch by size: small lattices use 32x32 tiles. */
template <bool AMF, bool BKF, class LA, class LB, class ST>
__device__ __forceinline__ void gemm_sq(int M, int N, int K, LA la, LB lb, ST st,
                                        double *sm)
{
    if (M <= 32 && N <= 32)
        gemm<TSm, AMF, BKF>(M, N, K, la, lb, st, sm);
    else if (M <= 64)
        gemm<TMma, AMF, BKF>(M, N, K, la, lb, st, sm);
    else
        gemm<TSquare, AMF, BKF>(M, N, K, la, lb, st, sm);
}

/* ------------------------------------------------------------ workspace */
/* Shared-memory carve-up of one CTA (sizes in doubles, all disjoint
 * except the phase union, which the QR and the site-block update share). */
struct Smem {
    double *gsm;     /* GEMM staging                                 */
    double *red;     /* 40: reductions                               */
    double *vA, *vB, *vC, *vD;  /* n each: scalings, new log D, signs, norms */
    int *perm;       /* n                                            */
    int *iscr;       /* 2*DQMC_MAX_KB + 8 ints                       */
    double *phase;   /* union area                                   */
    /* QR view of the union area */
    double *P, *W, *Tw, *gram, *taus;
    /* site-block view of the union area */
    double *g0, *gt, *gam, *xs, *colA;
};

__host__ __device__ inline size_t smem_doubles(int n, int kb)
{
    const size_t qr = (size_t)n * QNB + (size_t)QNB * WCOLS + 2 * QNB * QNB + QNB;
    (void)kb;
    const size_t pr = 4 * (size_t)DQMC_MAX_KB * (DQMC_MAX_KB + 1) + DQMC_MAX_KB;
    const size_t un = qr > pr ? qr : pr;
    const size_t ints = (size_t)n + 2 * DQMC_MAX_KB + 8;
    return (size_t)GEMM_SMEM + 40 + 4 * (size_t)n + (ints + 1) / 2 + un + 8;
}

__device__ inline Smem carve(double *base, int n, int kb)
{
    Smem s;
    double *p = base;
    s.gsm = p; p += GEMM_SMEM;
    s.red = p; p += 40;
    s.vA = p; p += n;
    s.vB = p; p += n;
    s.vC = p; p += n;
    s.vD = p; p += n;
    const size_t ints = (size_t)n + 2 * DQMC_MAX_KB + 8;
    s.perm = (int *)p;
    s.iscr = s.perm + n;
    p += (ints + 1) / 2;
    s.phase = p;
    s.P = p;
    s.W = s.P + (size_t)n * QNB;
    s.Tw = s.W + (size_t)QNB * WCOLS;
    s.gram = s.Tw + QNB * QNB;
    s.taus = s.gram + QNB * QNB;
    const int ld = kb + 1;
    s.g0 = p;
    s.gt = s.g0 + (size_t)kb * ld;
    s.gam = s.gt + (size_t)kb * ld;
    s.xs = s.gam + (size_t)kb * ld;
    s.colA = s.xs + kb;
    return s;
}

/* Per-chain error flag kept in shared memory (bit-or of DQMC_ST_*). */
__device__ __forceinline__ void raise_flag(int *flag, int bit)
{
    atomicOr(flag, bit);
}

/* ----------------------------------------------------------------- QR */
/* V(r, q) of a panel stored in P (ld m): unit diagonal, tail below. */
__device__ __forceinline__ double vpan(const double *P, int m, int r, int q)
{
    return r > q ? P[r + (size_t)q * m] : (r == q ? 1.0 : 0.0);
}

/* Compact-WY factor (LAPACK dlarft, forward, columnwise): H_1...H_nb =
 * I - V Tw V^T with Tw upper triangular (ld QNB). */
__device__ __noinline__ void build_tw(int m, int nb, const double *P, const double *tau,
                         double *Tw, double *gram)
{
    for (int e = threadIdx.x; e < QNB * QNB; e += NT) Tw[e] = 0.0;
    for (int e = threadIdx.x; e < nb * nb; e += NT) {
        const int q = e % nb, i = e / nb;
        if (q < i) {
            double s = P[i + (size_t)q * m];
            for (int r = i + 1; r < m; ++r) s += P[r + (size_t)q * m] * P[r + (size_t)i * m];
            gram[q + i * QNB] = s;
        }
    }
    __syncthreads();
    for (int i = 0; i < nb; ++i) {
        const int r = threadIdx.x;
        if (r < i) {
            double s = 0.0;
            for (int q = r; q < i; ++q) s += Tw[r + q * QNB] * gram[q + i * QNB];
            Tw[r + i * QNB] = -tau[i] * s;
        } else if (r == i) {
            Tw[i + i * QNB] = tau[i];
        }
        __syncthreads();
    }
}

/* X(m x nc, ld ldx) <- op(H) X with H = I - V Tw V^T of the panel in P.
 * transT: apply H^T = I - V Tw^T V^T (what a QR applies to A). */
__device__ __noinline__ void apply_block(int m, int nb, const double *P, const double *Tw,
                            bool transT, double *X, int ldx, int nc, Smem &s)
{
    for (int cc = 0; cc < nc; cc += WCOLS) {
        const int ncc = min(WCOLS, nc - cc);
        double *Xc = X + (size_t)cc * ldx;
        double *W = s.W;
        gemm<TMmaWide, false, true>(
            nb, ncc, m, [=](int i, int k) { return vpan(P, m, k, i); },
            [=](int k, int j) { return Xc[k + (size_t)j * ldx]; },
            [=](int i, int j, double v) { W[i + j * QNB] = v; }, s.gsm);
        for (int j = threadIdx.x; j < ncc; j += NT) {
            double w[QNB], o[QNB];
#pragma unroll
            for (int i = 0; i < QNB; ++i) w[i] = (i < nb) ? W[i + j * QNB] : 0.0;
#pragma unroll
            for (int i = 0; i < QNB; ++i) {
                double acc = 0.0;
                if (transT) {
#pragma unroll
                    for (int q = 0; q <= i; ++q) acc += Tw[q + i * QNB] * w[q];
                } else {
#pragma unroll
                    for (int q = i; q < QNB; ++q) acc += Tw[i + q * QNB] * w[q];
                }
                o[i] = acc;
            }
#pragma unroll
            for (int i = 0; i < QNB; ++i)
                if (i < nb) W[i + j * QNB] = o[i];
        }
        __syncthreads();
        gemm_rmw<TSquare, true, true>(
            m, ncc, nb, [=](int i, int k) { return vpan(P, m, i, k); },
            [=](int k, int j) { return W[k + j * QNB]; },
            [=](int i, int j) { return Xc[i + (size_t)j * ldx]; },
            [=](int i, int j, double v, double c) { Xc[i + (size_t)j * ldx] = c - v; }, s.gsm);
    }
}

/* Householder QR of the n x n matrix A (ld n) in place, LAPACK dgeqrf
 * layout and dlarfg sign convention.  tw receives each panel's Tw
 * (QNB*QNB per panel).  Returns the number of non-trivial reflectors (the
 * parity gives det Q). */
__device__ __noinline__ int qr_factor(int n, double *A, double *tw, Smem &s, int *flag)
{
    int nontrivial = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j0 = 0; j0 < n; j0 += QNB) {
        const int nb = min(QNB, n - j0), m = n - j0;
        double *P = s.P;
        for (int e = threadIdx.x; e < m * nb; e += NT) {
            const int r = e % m, c = e / m;
            P[e] = A[(j0 + r) + (size_t)(j0 + c) * n];
        }
        __syncthreads();
        for (int jj = 0; jj < nb; ++jj) {
            double sq = 0.0;
            for (int r = jj + 1 + threadIdx.x; r < m; r += NT) {
                const double x = P[r + (size_t)jj * m];
                sq += x * x;
            }
            const double xn2 = block_reduce<false>(sq, s.red);
            const double alpha = P[jj + (size_t)jj * m];
            double tau = 0.0, beta = alpha;
            if (xn2 > 0.0) {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                tau = (beta - alpha) / beta;
                const double scal = 1.0 / (alpha - beta);
                for (int r = jj + 1 + threadIdx.x; r < m; r += NT) P[r + (size_t)jj * m] *= scal;
                ++nontrivial;
            }
            if (!isfinite(beta) || !isfinite(tau)) raise_flag(flag, DQMC_ST_NONFINITE);
            __syncthreads();
            if (threadIdx.x == 0) {
                P[jj + (size_t)jj * m] = beta;
                s.taus[jj] = tau;
            }
            if (tau != 0.0) {
                for (int c = jj + 1 + warp; c < nb; c += NW) {
                    const double pj = P[jj + (size_t)c * m];
                    double w = 0.0;
                    for (int r = jj + 1 + lane; r < m; r += 32)
                        w += P[r + (size_t)jj * m] * P[r + (size_t)c * m];
                    w = tau * (warp_sum(w) + pj);
                    for (int r = jj + 1 + lane; r < m; r += 32)
                        P[r + (size_t)c * m] -= w * P[r + (size_t)jj * m];
                    if (lane == 0) P[jj + (size_t)c * m] = pj - w;
                }
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < m * nb; e += NT) {
            const int r = e % m, c = e / m;
            A[(j0 + r) + (size_t)(j0 + c) * n] = P[e];
        }
        build_tw(m, nb, P, s.taus, s.Tw, s.gram);
        double *twp = tw + (size_t)(j0 / QNB) * QNB * QNB;
        for (int e = threadIdx.x; e < QNB * QNB; e += NT) twp[e] = s.Tw[e];
        if (j0 + nb < n)
            apply_block(m, nb, P, s.Tw, true, A + j0 + (size_t)(j0 + nb) * n, n,
                        n - j0 - nb, s);
        __syncthreads();
    }
    return nontrivial;
}

/* Load panel j0 of a factored A (reflector tails) and its Tw into smem. */
__device__ __noinline__ void load_panel(int n, const double *A, const double *tw, int j0, Smem &s)
{
    const int nb = min(QNB, n - j0), m = n - j0;
    for (int e = threadIdx.x; e < m * nb; e += NT) {
        const int r = e % m, c = e / m;
        s.P[e] = A[(j0 + r) + (size_t)(j0 + c) * n];
    }
    const double *twp = tw + (size_t)(j0 / QNB) * QNB * QNB;
    for (int e = threadIdx.x; e < QNB * QNB; e += NT) s.Tw[e] = twp[e];
    __syncthreads();
}

/* Q = H_1 ... H_n of a factored A written to Q (ld n). */
__device__ __noinline__ void qr_form_q(int n, const double *A, const double *tw, double *Q, Smem &s)
{
    for (int e = threadIdx.x; e < n * n; e += NT) Q[e] = (e % n == e / n) ? 1.0 : 0.0;
    __syncthreads();
    for (int j0 = ((n - 1) / QNB) * QNB; j0 >= 0; j0 -= QNB) {
        load_panel(n, A, tw, j0, s);
        const int nb = min(QNB, n - j0), m = n - j0;
        apply_block(m, nb, s.P, s.Tw, false, Q + j0 + (size_t)j0 * n, n, n - j0, s);
    }
}

/* Y (n x nc, ld n) <- Q^T Y for a factored A. */
__device__ __noinline__ void qr_apply_qt(int n, const double *A, const double *tw, double *Y, int nc,
                            Smem &s)
{
    for (int j0 = 0; j0 < n; j0 += QNB) {
        load_panel(n, A, tw, j0, s);
        const int nb = min(QNB, n - j0), m = n - j0;
        apply_block(m, nb, s.P, s.Tw, true, Y + j0, n, nc, s);
    }
}

/* Solve R X = Y for the upper triangle R of A (ld n); X, Y n x n, X may not
 * alias Y.  Blocked by QNB rows from the bottom. */
__device__ __noinline__ void trsm_upper(int n, const double *A, const double *Y, double *X, Smem &s)
{
    for (int i1 = n; i1 > 0; i1 -= QNB) {
        const int i0 = max(0, i1 - QNB), bs = i1 - i0;
        if (i1 < n) {
            gemm_rmw<TMmaWide, true, true>(
                bs, n, n - i1,
                [=](int i, int k) { return A[(i0 + i) + (size_t)(i1 + k) * n]; },
                [=](int k, int j) { return X[(i1 + k) + (size_t)j * n]; },
                [=](int i, int j) { return Y[(i0 + i) + (size_t)j * n]; },
                [=](int i, int j, double v, double c) { X[(i0 + i) + (size_t)j * n] = c - v; },
                s.gsm);
        } else {
            for (int e = threadIdx.x; e < bs * n; e += NT) {
                const int i = e % bs, j = e / bs;
                X[(i0 + i) + (size_t)j * n] = Y[(i0 + i) + (size_t)j * n];
            }
        }
        double *Rb = s.Tw;
        for (int e = threadIdx.x; e < QNB * QNB; e += NT) {
            const int i = e % QNB, k = e / QNB;
            Rb[e] = (i < bs && k < bs) ? A[(i0 + i) + (size_t)(i0 + k) * n] : 0.0;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += NT) {
            double x[QNB];
#pragma unroll
            for (int i = 0; i < QNB; ++i) x[i] = (i < bs) ? X[(i0 + i) + (size_t)j * n] : 0.0;
#pragma unroll
            for (int i = QNB - 1; i >= 0; --i) {
                if (i < bs) {
                    double acc = x[i];
#pragma unroll
                    for (int k = i + 1; k < QNB; ++k) acc -= Rb[i + k * QNB] * x[k];
                    x[i] = acc / Rb[i + i * QNB];
                }
            }
#pragma unroll
            for (int i = 0; i < QNB; ++i)
                if (i < bs) X[(i0 + i) + (size_t)j * n] = x[i];
        }
        __syncthreads();
    }
}

/* ------------------------------------------------- pre-pivoted factor */
/* Column pivoting by a one-time norm sort (pre-pivoting): perm[r] is the
 * column of M with the r-th largest 2-norm; Aout[:, r] = M[:, perm[r]]. */
__device__ __noinline__ void prepivot(int n, const double *M, double *Aout, Smem &s, int *flag)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *nrm = s.vD;
    for (int c = warp; c < n; c += NW) {
        double mx = 0.0;
        for (int r = lane; r < n; r += 32) mx = fmax(mx, fabs(M[r + (size_t)c * n]));
        mx = warp_max(mx);
        double sq = 0.0;
        if (mx > 0.0 && isfinite(mx)) {
            const double inv = 1.0 / mx;
            for (int r = lane; r < n; r += 32) {
                const double x = M[r + (size_t)c * n] * inv;
                sq += x * x;
            }
        }
        sq = warp_sum(sq);
        if (lane == 0) {
            double v = (mx > 0.0) ? log(mx) + 0.5 * log(sq) : -INFINITY;
            if (!isfinite(mx) || isnan(v)) {
                raise_flag(flag, DQMC_ST_NONFINITE);
                v = -INFINITY;
            }
            nrm[c] = v;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < n; c += NT) {
        const double v = nrm[c];
        int rank = 0;
        for (int d = 0; d < n; ++d) {
            const double w = nrm[d];
            rank += (w > v) || (w == v && d < c);
        }
        s.perm[rank] = c;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e % n, r = e / n;
        Aout[e] = M[i + (size_t)s.perm[r] * n];
    }
    __syncthreads();
}

/* After qr_factor: vB = log|R_ii| (new log D), vC = sign(R_ii).  Returns
 * the sign of prod sign(R_ii). */
__device__ int qr_diag(int n, const double *A, Smem &s, int *flag)
{
    for (int i = threadIdx.x; i < n; i += NT) {
        const double r = A[i + (size_t)i * n];
        if (r == 0.0) raise_flag(flag, DQMC_ST_SINGULAR);
        if (!isfinite(r)) raise_flag(flag, DQMC_ST_NONFINITE);
        s.vB[i] = log(fabs(r));
        s.vC[i] = r < 0.0 ? -1.0 : 1.0;
    }
    __syncthreads();
    double neg = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) neg += (s.vC[i] < 0.0) ? 1.0 : 0.0;
    neg = block_reduce<false>(neg, s.red);
    return (((long long)neg) & 1) ? -1 : 1;
}

/* ------------------------------------------------------------------ UDV */
struct Udv {
    double *U, *T, *ell, *det;
};

__device__ __forceinline__ Udv udv_at(double *base, int n)
{
    const size_t nn = (size_t)n * n;
    return Udv{base, base + nn, base + 2 * nn, base + 2 * nn + n};
}

__device__ void udv_identity(Udv u, int n)
{
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const double v = (e % n == e / n) ? 1.0 : 0.0;
        u.U[e] = v;
        u.T[e] = v;
    }
    for (int i = threadIdx.x; i < n; i += NT) u.ell[i] = 0.0;
    if (threadIdx.x == 0) *u.det = 1.0;
    __syncthreads();
}

__device__ void udv_copy(Udv d, Udv s, int n)
{
    for (int e = threadIdx.x; e < n * n; e += NT) {
        d.U[e] = s.U[e];
        d.T[e] = s.T[e];
    }
    for (int i = threadIdx.x; i < n; i += NT) d.ell[i] = s.ell[i];
    if (threadIdx.x == 0) *d.det = *s.det;
    __syncthreads();
}

__device__ __forceinline__ double checked_exp(double x, int *flag)
{
    if (!(x < 700.0)) raise_flag(flag, DQMC_ST_LOGRANGE);
    return exp(x);
}

/* Scratch buffers (n x n each) a UDV update may use. */
struct Scr {
    double *m0, *m1, *m2, *tw;
};

/* u <- Bop * u where Bop = B (if B != nullptr) or expK * diag(v_l) for the
 * field row fl (single slice).  udv_lmul_impl, linalg.c:515-642, with
 * pre-pivoting and positive D (signs folded into U). */
__device__ __noinline__ void udv_lmul(int n, Udv u, const double *B, const double *expK,
                         const signed char *fl, double v0, double v1, Scr w, Smem &s,
                         int *flag)
{
    for (int j = threadIdx.x; j < n; j += NT) {
        s.vA[j] = checked_exp(u.ell[j], flag);
        if (B == nullptr) s.vD[j] = fl[j] > 0 ? v1 : v0;
    }
    __syncthreads();
    const double *U = u.U;
    double *eD = s.vA, *vl = s.vD;
    double *M = w.m0;
    if (B != nullptr) {
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return B[i + (size_t)k * n]; },
            [=](int k, int j) { return U[k + (size_t)j * n] * eD[j]; },
            [=](int i, int j, double v) { M[i + (size_t)j * n] = v; }, s.gsm);
    } else {
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return expK[i + (size_t)k * n]; },
            [=](int k, int j) { return vl[k] * U[k + (size_t)j * n] * eD[j]; },
            [=](int i, int j, double v) { M[i + (size_t)j * n] = v; }, s.gsm);
    }
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    const double *R = w.m1;
    const double *T = u.T;
    const int *perm = s.perm;
    double *Tn = w.m2;
    gemm_sq<true, true>(
        n, n, n,
        [=](int i, int k) { return k >= i ? R[i + (size_t)k * n] / R[i + (size_t)i * n] : 0.0; },
        [=](int k, int j) { return T[perm[k] + (size_t)j * n]; },
        [=](int i, int j, double v) { Tn[i + (size_t)j * n] = v; }, s.gsm);
    for (int e = threadIdx.x; e < n * n; e += NT) u.T[e] = Tn[e];
    qr_form_q(n, w.m1, w.tw, u.U, s);
    for (int e = threadIdx.x; e < n * n; e += NT) u.U[e] *= s.vC[e / n];
    for (int i = threadIdx.x; i < n; i += NT) u.ell[i] = s.vB[i];
    if (threadIdx.x == 0) *u.det = ((nt & 1) ? -1.0 : 1.0) * sg;
    __syncthreads();
}

/* u <- u * B (udv_rmul_impl, linalg.c:662-784), pre-pivoted. */
__device__ __noinline__ void udv_rmul(int n, Udv u, const double *B, Scr w, Smem &s, int *flag)
{
    for (int j = threadIdx.x; j < n; j += NT) s.vA[j] = checked_exp(u.ell[j], flag);
    __syncthreads();
    const double *T = u.T;
    const double *eD = s.vA;
    double *M = w.m0;
    gemm_sq<true, true>(
        n, n, n, [=](int i, int k) { return eD[i] * T[i + (size_t)k * n]; },
        [=](int k, int j) { return B[k + (size_t)j * n]; },
        [=](int i, int j, double v) { M[i + (size_t)j * n] = v; }, s.gsm);
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    qr_form_q(n, w.m1, w.tw, w.m0, s);
    const double *U = u.U;
    const double *Q = w.m0;
    const double *sgn = s.vC;
    double *Un = w.m2;
    gemm_sq<true, true>(
        n, n, n, [=](int i, int k) { return U[i + (size_t)k * n]; },
        [=](int k, int j) { return Q[k + (size_t)j * n]; },
        [=](int i, int j, double v) { Un[i + (size_t)j * n] = v * sgn[j]; }, s.gsm);
    for (int e = threadIdx.x; e < n * n; e += NT) u.U[e] = Un[e];
    const double *R = w.m1;
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e % n, r = e / n;
        u.T[i + (size_t)s.perm[r] * n] =
            r >= i ? R[i + (size_t)r * n] / R[i + (size_t)i * n] : 0.0;
    }
    for (int i = threadIdx.x; i < n; i += NT) u.ell[i] = s.vB[i];
    __syncthreads();
    if (threadIdx.x == 0) *u.det = *u.det * ((nt & 1) ? -1.0 : 1.0) * sg;
    __syncthreads();
}

/* o <- l * r (udv_combine, linalg.c:796-909), pre-pivoted. */
__device__ __noinline__ void udv_combine(int n, Udv l, Udv r, Udv o, Scr w, Smem &s, int *flag)
{
    for (int j = threadIdx.x; j < n; j += NT) {
        s.vA[j] = checked_exp(l.ell[j], flag);
        s.vD[j] = checked_exp(r.ell[j], flag);
    }
    __syncthreads();
    const double *TL = l.T, *UR = r.U;
    const double *eL = s.vA;
    double *M = w.m0;
    {
        const double *eR = s.vD;
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return TL[i + (size_t)k * n]; },
            [=](int k, int j) { return UR[k + (size_t)j * n]; },
            [=](int i, int j, double v) { M[i + (size_t)j * n] = eL[i] * v * eR[j]; },
            s.gsm);
    }
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    qr_form_q(n, w.m1, w.tw, w.m0, s);
    const double *UL = l.U, *Q = w.m0, *sgn = s.vC;
    double *Uo = o.U;
    gemm_sq<true, true>(
        n, n, n, [=](int i, int k) { return UL[i + (size_t)k * n]; },
        [=](int k, int j) { return Q[k + (size_t)j * n]; },
        [=](int i, int j, double v) { Uo[i + (size_t)j * n] = v * sgn[j]; }, s.gsm);
    const double *R = w.m1, *TR = r.T;
    const int *perm = s.perm;
    double *To = o.T;
    gemm_sq<true, true>(
        n, n, n,
        [=](int i, int k) { return k >= i ? R[i + (size_t)k * n] / R[i + (size_t)i * n] : 0.0; },
        [=](int k, int j) { return TR[perm[k] + (size_t)j * n]; },
        [=](int i, int j, double v) { To[i + (size_t)j * n] = v; }, s.gsm);
    for (int i = threadIdx.x; i < n; i += NT) o.ell[i] = s.vB[i];
    if (threadIdx.x == 0) *o.det = *l.det * ((nt & 1) ? -1.0 : 1.0) * sg;
    __syncthreads();
}

/* G = (1 + U D T)^{-1} with D = exp(ell) > 0, via the split D = Db Ds,
 * Db = max(D,1), Ds = min(D,1):  1 + U D T = U Db X with
 * X = Db^{-1} U^T + Ds T, so G = X^{-1} Db^{-1} U^T (QR solve).
 * Replaces udv_inv_one_plus_work (linalg.c:911-1115).  Returns the sign of
 * det(1 + U D T) = det U * det X (det Db > 0). */
__device__ __noinline__ int udv_green(int n, Udv u, double *G, Scr w, Smem &s, int *flag)
{
    const double *U = u.U, *T = u.T, *ell = u.ell;
    double *X = w.m1, *Y = w.m0;
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e % n, j = e / n;
        const double l = ell[i];
        const double dbi = exp(-fmax(l, 0.0)), ds = exp(fmin(l, 0.0));
        const double ut = U[j + (size_t)i * n];
        Y[e] = dbi * ut;
        X[e] = dbi * ut + ds * T[e];
    }
    __syncthreads();
    const int nt = qr_factor(n, X, w.tw, s, flag);
    const int sg = qr_diag(n, X, s, flag);
    qr_apply_qt(n, X, w.tw, Y, n, s);
    trsm_upper(n, X, Y, G, s);
    double bad = 0.0;
    for (int e = threadIdx.x; e < n * n; e += NT) bad += isfinite(G[e]) ? 0.0 : 1.0;
    bad = block_reduce<false>(bad, s.red);
    if (bad != 0.0) raise_flag(flag, DQMC_ST_NONFINITE);
    const double dU = *u.det;
    return (int)(dU * ((nt & 1) ? -1.0 : 1.0) * sg);
}

/* ----------------------------------------------------- slice operations */
/* G <- B_l G B_l^{-1} = expK diag(v) G diag(1/v) expKinv (green.c:509-527). */
__device__ __noinline__ void wrap_green(int n, double *G, double *tmp, const double *expK,
                           const double *expKinv, const signed char *fl, double v0,
                           double v1, double vi0, double vi1, Smem &s)
{
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    gemm_sq<true, true>(
        n, n, n, [=](int i, int k) { return expK[i + (size_t)k * n]; },
        [=](int k, int j) { return vv[k] * G[k + (size_t)j * n] * vi[j]; },
        [=](int i, int j, double v) { tmp[i + (size_t)j * n] = v; }, s.gsm);
    gemm_sq<true, true>(
        n, n, n, [=](int i, int k) { return tmp[i + (size_t)k * n]; },
        [=](int k, int j) { return expKinv[k + (size_t)j * n]; },
        [=](int i, int j, double v) { G[i + (size_t)j * n] = v; }, s.gsm);
}

/* out = B_{l0+len-1} ... B_{l0} (green.c:151-166); X, Y ping-pong scratch. */
__device__ __noinline__ void bblock(int n, int l0, int len, const signed char *field, const double *expK,
                       double v0, double v1, double *out, double *X, double *Y, Smem &s)
{
    const signed char *f0 = field + (size_t)l0 * n;
    double *first = (len == 1) ? out : X;
    for (int e = threadIdx.x; e < n * n; e += NT)
        first[e] = expK[e] * (f0[e / n] > 0 ? v1 : v0);
    __syncthreads();
    const double *src = first;
    double *vv = s.vA;
    for (int p = 1; p < len; ++p) {
        double *dst = (p == len - 1) ? out : ((src == X) ? Y : X);
        const signed char *fp = field + (size_t)(l0 + p) * n;
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += NT) vv[k] = fp[k] > 0 ? v1 : v0;
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return expK[i + (size_t)k * n]; },
            [=](int k, int j) { return vv[k] * src[k + (size_t)j * n]; },
            [=](int i, int j, double v) { dst[i + (size_t)j * n] = v; }, s.gsm);
        src = dst;
    }
}

/* ------------------------------------------------ RNG (rng.c:23-37) */
__device__ __forceinline__ uint64_t rotl64(uint64_t x, int k)
{
    return (x << k) | (x >> (64 - k));
}

__device__ __forceinline__ double rng_next(uint64_t *s)
{
    const uint64_t res = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return (double)(res >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace DQMC_NS
