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

#include <type_traits>

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
template <int BM_, int BN_, int BK_, int TM_, int TN_, bool MMA_ = false, int WM_ = 2, int KS_ = 4>
struct Tile {
    static constexpr int BM = BM_, BN = BN_, BK = BK_, TM = TM_, TN = TN_;
    static constexpr bool MMA = MMA_;
    /* k extent of one mma instruction: m16n8k4, m16n8k8 or m16n8k16 */
    static constexpr int KS = KS_;
    static_assert(BK % KS_ == 0, "k slice must hold whole mma steps");
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
/* 128 x 128 with 2 x 4 warps: 4 x 4 fragments (16 accumulators) per warp,
 * for products without a read-modify-write epilogue */
using TMmaWideSq = Tile<128, 128, 16, 16, 4, true, 2>;
#if DQMC_MINB == 1
using TSquare = TMmaBig;
using TSquareNR = TMmaWideSq;
#else
using TSquare = TMma;
using TSquareNR = TMma;
#endif
constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int GEMM_SMEM =
    cmax(cmax(TWide::SMEM, TSq::SMEM),
         cmax(cmax(TMma::SMEM, TMmaWide::SMEM), cmax(TSquare::SMEM, TSquareNR::SMEM)));


/* D = A(16xKS) B(KSx8) + C, FP64 on the tensor cores.  Fragments: lane
 * (gid = lane/4, tig = lane%4) holds a[2q] = A(gid, tig+4q), a[2q+1] =
 * A(gid+8, tig+4q), b[q] = B(tig+4q, gid), c = D(gid|gid+8, 2tig|2tig+1). */
template <int KS>
__device__ __forceinline__ void dmma(double *c, const double *a, const double *b)
{
    if constexpr (KS == 4) {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
    } else if constexpr (KS == 8) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    } else {
        static_assert(KS == 16, "mma k extent");
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
            "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
              "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
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
/* Operand transform applied when a fetched slice is staged (identity). */
struct Ident {
    __device__ __forceinline__ double operator()(int, int, double x) const { return x; }
};

/* Share of a product's output tiles taken by one CTA: tiles r, r + c,
 * r + 2c, ... of the column-major tile grid.  {0, 1} is the whole product;
 * the CTAs of a cluster that advance one chain together take {rank, size}.
 * Every output element is formed by the same instruction sequence whatever
 * the share, so a split product equals the unsplit one bit for bit. */
struct Part {
    int r = 0, c = 1;
};

template <class T, bool AMF, bool BKF, bool RMW, bool PART = false, class LA, class LB, class LC,
          class ST, class SA = Ident, class SB = Ident>
__device__ void gemm_core(int M, int N, int K, LA la, LB lb, LC lc, ST st, double *sm,
                          SA sa = SA(), SB sb = SB(), Part pt = Part())
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
    const int ntile = tm * tn;
    const int mine = !PART ? ntile : ntile > pt.r ? (ntile - pt.r + pt.c - 1) / pt.c : 0;
    const int total = mine * nk;
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
    /* fetch position (tile index, tile origin and k offset), advanced
     * incrementally over this CTA's share of the tiles */
    int fti = PART ? pt.r : 0, fk0 = 0;
    int fm0 = PART ? (pt.r % tm) * BM : 0, fn0 = PART ? (pt.r / tm) * BN : 0;
    auto advance = [&](int &ti, int &m0, int &n0, int &k0) {
        k0 += BK;
        if (k0 >= nk * BK) {
            k0 = 0;
            if constexpr (PART) {
                ti += pt.c;
                m0 = (ti % tm) * BM;
                n0 = (ti / tm) * BN;
            } else {
                m0 += BM;
                if (m0 >= tm * BM) {
                    m0 = 0;
                    n0 += BN;
                }
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
    /* Loaders only load: any arithmetic on a loaded value (sa, sb) runs
     * here, after the slice's math, so the loads stay in flight across it. */
    auto put = [&](int buf) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = tid + q * NT;
            const int i = AMF ? e % BM : e / BK, k = AMF ? e / BM : e % BK;
            double v = ra[q];
            if constexpr (!std::is_same<SA, Ident>::value) {
                const int gi = fm0 + i, gk = fk0 + k;
                v = (gi < M && gk < K) ? sa(gi, gk, v) : 0.0;
            }
            As[buf * BK * AP + k * AP + i] = v;
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = tid + q * NT;
            const int k = BKF ? e % BK : e / BN, j = BKF ? e / BK : e % BN;
            double v = rb[q];
            if constexpr (!std::is_same<SB, Ident>::value) {
                const int gk = fk0 + k, gj = fn0 + j;
                v = (gk < K && gj < N) ? sb(gk, gj, v) : 0.0;
            }
            Bs[buf * BK * BP + k * BP + j] = v;
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
    if constexpr (RMW) fetch_c(fm0, fn0);
    fetch();
    put(0);
    __syncthreads();
    int cti = fti, cm0 = fm0, cn0 = fn0, ck0 = 0;   /* position being multiplied */
    advance(fti, fm0, fn0, fk0);
    for (int it = 0; it < total; ++it) {
        const int cur = it & 1;
        if (it + 1 < total) fetch();
        const double *a = As + cur * BK * AP;
        const double *b = Bs + cur * BK * BP;
        if constexpr (T::MMA) {
            constexpr int FM = T::FM, FN = T::FN, KS = T::KS, KQ = KS / 4;
#pragma unroll
            for (int kk = 0; kk < BK; kk += KS) {
                double af[FM][2 * KQ], bf[FN][KQ];
#pragma unroll
                for (int mi = 0; mi < FM; ++mi) {
                    const int i = wm * (FM * 16) + mi * 16 + gid;
#pragma unroll
                    for (int q = 0; q < KQ; ++q) {
                        af[mi][2 * q] = a[(kk + tig + 4 * q) * AP + i];
                        af[mi][2 * q + 1] = a[(kk + tig + 4 * q) * AP + i + 8];
                    }
                }
#pragma unroll
                for (int ni = 0; ni < FN; ++ni)
#pragma unroll
                    for (int q = 0; q < KQ; ++q)
                        bf[ni][q] = b[(kk + tig + 4 * q) * BP + wn * (FN * 8) + ni * 8 + gid];
#pragma unroll
                for (int mi = 0; mi < FM; ++mi)
#pragma unroll
                    for (int ni = 0; ni < FN; ++ni) dmma<KS>(acc[mi * FN + ni], af[mi], bf[ni]);
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
        advance(cti, cm0, cn0, ck0);
        advance(fti, fm0, fn0, fk0);
        __syncthreads();
    }
}

template <class T, bool AMF, bool BKF, class LA, class LB, class ST, class SA = Ident,
          class SB = Ident>
__device__ __forceinline__ void gemm(int M, int N, int K, LA la, LB lb, ST st, double *sm,
                                     SA sa = SA(), SB sb = SB())
{
    gemm_core<T, AMF, BKF, false>(
        M, N, K, la, lb, [](int, int) { return 0.0; }, st, sm, sa, sb);
}

/* One CTA's share pt of gemm's output tiles. */
template <class T, bool AMF, bool BKF, class LA, class LB, class ST>
__device__ __forceinline__ void gemm_part(int M, int N, int K, LA la, LB lb, ST st, double *sm,
                                          Part pt)
{
    gemm_core<T, AMF, BKF, false, true>(
        M, N, K, la, lb, [](int, int) { return 0.0; }, st, sm, Ident(), Ident(), pt);
}

/* C(i,j) <- st(i, j, sum_k a b, C(i,j)) with C read through lc */
template <class T, bool AMF, bool BKF, class LA, class LB, class LC, class ST>
__device__ __forceinline__ void gemm_rmw(int M, int N, int K, LA la, LB lb, LC lc, ST st,
                                         double *sm)
{
    gemm_core<T, AMF, BKF, true>(M, N, K, la, lb, lc, st, sm);
}

/* One CTA's share pt of gemm_rmw's output tiles. */
template <class T, bool AMF, bool BKF, class LA, class LB, class LC, class ST>
__device__ __forceinline__ void gemm_rmw_part(int M, int N, int K, LA la, LB lb, LC lc, ST st,
                                              double *sm, Part pt)
{
    gemm_core<T, AMF, BKF, true, true>(M, N, K, la, lb, lc, st, sm, Ident(), Ident(), pt);
}

/* Square-product dispatch by size: small lattices use 32x32 tiles. */
template <bool AMF, bool BKF, class LA, class LB, class ST, class SA = Ident, class SB = Ident>
__device__ __forceinline__ void gemm_sq(int M, int N, int K, LA la, LB lb, ST st,
                                        double *sm, SA sa = SA(), SB sb = SB())
{
    if (M <= 32 && N <= 32)
        gemm<TSm, AMF, BKF>(M, N, K, la, lb, st, sm, sa, sb);
    else if (M <= 64)
        gemm<TMma, AMF, BKF>(M, N, K, la, lb, st, sm, sa, sb);
    else if (N > 64)
        gemm<TSquareNR, AMF, BKF>(M, N, K, la, lb, st, sm, sa, sb);
    else
        gemm<TSquare, AMF, BKF>(M, N, K, la, lb, st, sm, sa, sb);
}

/* C = A B for column-major A (lda) and B (ldb), epilogue st(i, j, acc). */
template <class ST>
__device__ __forceinline__ void gemm_nn(int M, int N, int K, const double *A, int lda,
                                        const double *B, int ldb, ST st, double *sm)
{
    gemm_sq<true, true>(
        M, N, K, [=](int i, int k) { return A[i + (size_t)k * lda]; },
        [=](int k, int j) { return B[k + (size_t)j * ldb]; }, st, sm);
}

/* C(i, j) <- st(i, j, (A B)(i, j), C(i, j)), C read through lc. */
template <class LC, class ST>
__device__ __forceinline__ void gemm_nn_rmw(int M, int N, int K, const double *A, int lda,
                                            const double *B, int ldb, LC lc, ST st, double *sm)
{
    gemm_rmw<TSquare, true, true>(
        M, N, K, [=](int i, int k) { return A[i + (size_t)k * lda]; },
        [=](int k, int j) { return B[k + (size_t)j * ldb]; }, lc, st, sm);
}

/* A CTA's share of C = sum_k la lb (epilogue st) among pt.c > 1 CTAs, the
 * tiles of the kind gemm_sq uses (SIMT for <= 32 x 32, else DMMA): among
 * the DMMA shapes the one whose slowest share is cheapest (128 x 128 tiles
 * issue about 1.5x the rate of 64 x 64 ones).  Every DMMA shape runs the
 * same k sequence, so the result does not depend on the choice. */
template <bool AMF, bool BKF, class LA, class LB, class ST>
__device__ __forceinline__ void gemm_sq_part(int M, int N, int K, LA la, LB lb, ST st,
                                             double *sm, Part pt)
{
    if (M <= 32 && N <= 32) {
        gemm_part<TSm, AMF, BKF>(M, N, K, la, lb, st, sm, pt);
        return;
    }
    const int w1 = ((M + 127) / 128 * ((N + 127) / 128) + pt.c - 1) / pt.c;
    const int w2 = ((M + 63) / 64 * ((N + 63) / 64) + pt.c - 1) / pt.c;
    if (M > 64 && N > 64 && 8 * w1 <= 3 * w2)
        gemm_part<TSquareNR, AMF, BKF>(M, N, K, la, lb, st, sm, pt);
    else
        gemm_part<TMma, AMF, BKF>(M, N, K, la, lb, st, sm, pt);
}

/* A CTA's share of C = A B (column-major A, B), as gemm_nn. */
template <class ST>
__device__ __forceinline__ void gemm_nn_part(int M, int N, int K, const double *A, int lda,
                                             const double *B, int ldb, ST st, double *sm,
                                             Part pt)
{
    gemm_sq_part<true, true>(
        M, N, K, [=](int i, int k) { return A[i + (size_t)k * lda]; },
        [=](int k, int j) { return B[k + (size_t)j * ldb]; }, st, sm, pt);
}

/* A CTA's share of the read-modify-write product (as gemm_nn_rmw). */
template <class LC, class ST>
__device__ __forceinline__ void gemm_nn_rmw_part(int M, int N, int K, const double *A, int lda,
                                                 const double *B, int ldb, LC lc, ST st,
                                                 double *sm, Part pt)
{
    auto la = [=](int i, int k) { return A[i + (size_t)k * lda]; };
    auto lb = [=](int k, int j) { return B[k + (size_t)j * ldb]; };
    const int w1 = ((M + 127) / 128 * ((N + 63) / 64) + pt.c - 1) / pt.c;
    const int w2 = ((M + 63) / 64 * ((N + 63) / 64) + pt.c - 1) / pt.c;
    if (20 * w1 <= 13 * w2)
        gemm_rmw_part<TSquare, true, true>(M, N, K, la, lb, lc, st, sm, pt);
    else
        gemm_rmw_part<TMma, true, true>(M, N, K, la, lb, lc, st, sm, pt);
}

/* ------------------------------------------------------------ workspace */
/* Shared-memory resident QR (qr_*_sm): the active block of cb columns (or,
 * transposed, rows) lives in shared memory with leading dimension
 * qr_ld(n) = round16(n) + 4 (so DMMA fragment reads hit distinct banks),
 * next to one reflector panel V (qr_ld x 16), the panel product W and
 * small scratch.  cb is the widest of 64/48/32/16 that fits the CTA's
 * shared-memory budget; 0 selects the global-memory QR. */
constexpr int QW = 20;              /* leading dimension of W (16 rows) */
/* staging of the split-product GEMM (dqmc_split.cuh), one-CTA build only:
 * DQMC_SPL_STAGES stages of DQMC_MIX_DIGITS x (128 + 128) lines x 32 bytes */
constexpr size_t MIX_SMEM_DOUBLES =
    (DQMC_MINB == 1) ? (size_t)DQMC_SPL_STAGES * DQMC_MIX_DIGITS * (128 + 128) * 32 / 8 : 0;
constexpr size_t QR_MISC = 1920;    /* T, gram, taus, reductions        */
constexpr size_t SMEM_BUDGET = (DQMC_MINB == 1 ? 227 * 1024 : 113 * 1024) / 8;

__host__ __device__ inline int qr_ld(int n) { return ((n + 15) / 16) * 16 + 4; }
__host__ __device__ inline size_t qr_wp(int cb)
{
    const size_t a = (size_t)NW * 128, b = (size_t)QW * cb;
    return a > b ? a : b;
}
__host__ __device__ inline size_t qr_sm_doubles(int n, int cb)
{
    return (size_t)qr_ld(n) * (cb + 16) + (size_t)QW * cb + qr_wp(cb) + QR_MISC;
}
__host__ __device__ inline size_t smem_fixed(int n)
{
    const size_t ints = (size_t)n + 2 * DQMC_MAX_KB + 8;
    return ((40 + 4 * (size_t)n + (ints + 1) / 2) + 1) & ~(size_t)1;
}
/* GEMM staging + the phase area behind it: with the shared-memory QR
 * (cb > 0) the phase area holds the site block or a 16 x 16 triangle
 * block; otherwise also the global-memory QR's panel. */
__host__ __device__ inline size_t smem_gemm_union(int n, int cb)
{
    const size_t qr = cb ? 256 : (size_t)n * QNB + (size_t)QNB * WCOLS + 2 * QNB * QNB + QNB;
    const size_t pr = 4 * (size_t)DQMC_MAX_KB * (DQMC_MAX_KB + 1) + DQMC_MAX_KB;
    return (size_t)GEMM_SMEM + (qr > pr ? qr : pr);
}
__host__ __device__ inline int qr_cb(int n)
{
    if (n > 3 * NT) return 0;
    const size_t base = smem_fixed(n) + 8;
    const size_t gu = smem_gemm_union(n, 16);
    for (int cb = 64; cb >= 16; cb -= 16) {
        const size_t q = qr_sm_doubles(n, cb);
        if (base + (q > gu ? q : gu) <= SMEM_BUDGET) return cb;
    }
    return 0;
}

/* Shared-memory carve-up of one CTA (sizes in doubles).  The fixed part
 * (reductions, per-row vectors, permutation) is followed by a union of
 * two views: GEMM staging + QR panel / site-block area, or the
 * shared-memory QR area. */
struct QrSm {
    double *X;       /* ld x cb active block                          */
    double *V;       /* ld x 16 reflector panel, unit diagonal        */
    double *W;       /* 16 x cb (ld QW) panel product                 */
    double *Wp;      /* NW x 128 partial products                     */
    double *T;       /* 16 x 16 compact-WY factor                     */
    double *gram;    /* 16 x 16 V^T V of the panel                    */
    double *taus;    /* 16                                            */
    double *rp;      /* 16 x NW + NW + 8 reduction partials           */
    double *rf;      /* 16 reduction results                          */
    int ld, cb;
};

struct Smem {
    double *gsm;     /* GEMM staging                                 */
    double *red;     /* 40: reductions                               */
    double *vA, *vB, *vC, *vD;  /* n each: scalings, new log D, signs, norms */
    int *perm;       /* n                                            */
    int *iscr;       /* 2*DQMC_MAX_KB + 8 ints                       */
    double *phase;   /* area after the GEMM staging                  */
    /* global-memory QR view of the phase area */
    double *P, *W, *Tw, *gram, *taus;
    /* site-block view of the phase area */
    double *g0, *gt, *gam, *xs, *colA;
    QrSm q;          /* shared-memory QR view (overlaps gsm + phase) */
    void *spl;       /* split-GEMM context (mixed precision), else null   */
    /* cluster cooperation: this CTA's rank among the CTAs that advance the
     * chain together ({0, 1}: one CTA per chain) and the chain's command
     * block through which rank 0 hands the others a product */
    Part cl;
    DqmcClCmd *cmd;
    double *stage;   /* the chain's DQMC_CL_STAGE_DOUBLES global staging */
};

__host__ __device__ inline size_t smem_doubles(int n, int kb)
{
    (void)kb;
    const int cb = qr_cb(n);
    const size_t gu = smem_gemm_union(n, cb);
    size_t q = cb ? qr_sm_doubles(n, cb) : 0;
    if (cb) q = q > MIX_SMEM_DOUBLES ? q : MIX_SMEM_DOUBLES;
    return smem_fixed(n) + (q > gu ? q : gu) + 8;
}

__device__ inline Smem carve(double *base, int n, int kb)
{
    Smem s;
    double *p = base;
    s.red = p; p += 40;
    s.vA = p; p += n;
    s.vB = p; p += n;
    s.vC = p; p += n;
    s.vD = p; p += n;
    s.perm = (int *)p;
    s.iscr = s.perm + n;
    p = base + smem_fixed(n);
    s.gsm = p;
    s.phase = p + GEMM_SMEM;
    s.P = s.phase;
    s.W = s.P + (size_t)n * QNB;
    s.Tw = s.W + (size_t)QNB * WCOLS;
    s.gram = s.Tw + QNB * QNB;
    s.taus = s.gram + QNB * QNB;
    const int ld = kb + 1;
    s.g0 = s.phase;
    s.gt = s.g0 + (size_t)kb * ld;
    s.gam = s.gt + (size_t)kb * ld;
    s.xs = s.gam + (size_t)kb * ld;
    s.colA = s.xs + kb;
    QrSm &q = s.q;
    q.ld = qr_ld(n);
    q.cb = qr_cb(n);
    q.X = p;
    q.V = q.X + (size_t)q.ld * q.cb;
    q.W = q.V + (size_t)q.ld * 16;
    q.Wp = q.W + (size_t)QW * q.cb;
    q.T = q.Wp + qr_wp(q.cb);
    q.gram = q.T + 256;
    q.taus = q.gram + 256;
    q.rp = q.taus + 16;
    q.rf = q.rp + 16 * NW + NW + 8;
    s.spl = nullptr;
    s.cl = Part();
    s.cmd = nullptr;
    s.stage = nullptr;
    return s;
}

/* ------------------------------------------------- cluster cooperation */
/* One chain advanced by the s.cl.c CTAs of a thread-block cluster: rank 0
 * runs the sweep; at a product that splits by output tiles (the wrap, the
 * B-block chain, the delayed-update G update) it writes a command into the
 * chain's command block and every rank, rank 0 included, forms its share
 * of the tiles.  The other ranks only ever wait at the cluster barrier for
 * the next command (cl_serve); rank 0 ends every launch with CL_EXIT.
 * Operands and results stay in global memory; the barrier's release /
 * acquire at cluster scope orders them.  Every command runs the same
 * barriers on every rank whatever its share, so the ranks cannot fall out
 * of step. */
enum {
    CL_EXIT = 0,
    CL_WRAP,        /* wrap_green                                      */
    CL_WRAP_BACK,   /* wrap_green_back                                 */
    CL_BBLOCK,      /* bblock                                          */
    CL_GUPD,        /* delayed-update G update                         */
    CL_QFORM,       /* qr_form_q_sm: column blocks                     */
    CL_QT,          /* qr_apply_qt_sm: column blocks                   */
    CL_QRIGHT,      /* qr_apply_right_sm: row blocks                   */
    CL_TRSM,        /* trsm_upper: column ranges                       */
    CL_UGEMM,       /* the UDV updates' products (udv_gemm kinds)      */
    CL_ZY,          /* flush_zy: row and column ranges                 */
    CL_PREPIV,      /* prepivot: column norms and the gather by columns */
    CL_WSPLIT,      /* wrap_green_split: lines of each split, tiles     */
    CL_FSPLIT,      /* flush_split: lines of each split, tiles          */
    CL_QRF          /* qr_factor_cl: a column block per rank            */
};

__device__ __forceinline__ void cl_sync()
{
    asm volatile("barrier.cluster.arrive.release;\n\t"
                 "barrier.cluster.wait.acquire;\n" ::: "memory");
}

__device__ __forceinline__ unsigned cl_rank_hw()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ unsigned cl_size_hw()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

/* Between two dependent steps of a split command: all ranks' shares. */
__device__ __forceinline__ void part_sync(const Smem &s)
{
    if (s.cl.c > 1)
        cl_sync();
    else
        __syncthreads();
}

/* Rank 0 hands a command to the cluster (no-op for one CTA per chain). */
__device__ __forceinline__ void cl_post(const Smem &s, int op, const void *p0, const void *p1,
                                        const void *p2, const void *p3, const void *p4,
                                        const void *p5, int i0, int i1, int i2, double d0 = 0.0,
                                        double d1 = 0.0, double d2 = 0.0, double d3 = 0.0)
{
    if (s.cl.c <= 1 || s.cl.r != 0) return;
    if (threadIdx.x == 0) {
        DqmcClCmd *c = s.cmd;
        c->op = op;
        c->i[0] = i0;
        c->i[1] = i1;
        c->i[2] = i2;
        c->p[0] = p0;
        c->p[1] = p1;
        c->p[2] = p2;
        c->p[3] = p3;
        c->p[4] = p4;
        c->p[5] = p5;
        c->d[0] = d0;
        c->d[1] = d1;
        c->d[2] = d2;
        c->d[3] = d3;
    }
    cl_sync();
}

/* End of a split command: every rank's share is in memory. */
__device__ __forceinline__ void cl_done(const Smem &s)
{
    if (s.cl.c > 1) cl_sync();
}

/* Rank 0's copy of a shared-memory location of this CTA (every rank carves
 * the same layout), read through distributed shared memory: the other
 * ranks take the small per-call vectors (scalings, signs, the pivot order)
 * that rank 0 holds in shared memory when a command starts. */
__device__ __forceinline__ unsigned cl_rank0_addr(const void *p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(r) : "r"(a));
    return r;
}

/* Copies count doubles / ints at p from rank 0's shared memory into this
 * CTA's (ranks > 0 only; rank 0 leaves them unchanged until the command's
 * last barrier). */
__device__ __forceinline__ void cl_pull(double *p, int count)
{
    for (int e = threadIdx.x; e < count; e += NT) {
        double v;
        asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(cl_rank0_addr(p + e))
                     : "memory");
        p[e] = v;
    }
}
__device__ __forceinline__ void cl_pull(int *p, int count)
{
    for (int e = threadIdx.x; e < count; e += NT) {
        int v;
        asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(cl_rank0_addr(p + e))
                     : "memory");
        p[e] = v;
    }
}

/* This rank's contiguous share [lo, hi) of count elementwise items. */
__device__ __forceinline__ void part_range(const Smem &s, int count, int &lo, int &hi)
{
    const int per = (count + s.cl.c - 1) / s.cl.c;
    lo = min(count, s.cl.r * per);
    hi = min(count, lo + per);
}

/* Elementwise pass over e < count with U loads in flight per thread:
 * ld(e) for a batch of U elements first, then st(e, value) for each, so
 * no load waits behind a store the compiler cannot prove independent. */
template <int U = 8, class LD, class ST>
__device__ __forceinline__ void ew_batched(int count, LD ld, ST st)
{
    for (int e0 = threadIdx.x; e0 < count; e0 += NT * U) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * NT;
            v[u] = e < count ? ld(e) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * NT;
            if (e < count) st(e, v[u]);
        }
    }
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
__device__ __noinline__ int qr_factor_gm(int n, double *A, double *tw, Smem &s, int *flag)
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
__device__ __noinline__ void qr_form_q_gm(int n, const double *A, const double *tw, double *Q,
                                          Smem &s)
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
__device__ __noinline__ void qr_apply_qt_gm(int n, const double *A, const double *tw, double *Y,
                                            int nc, Smem &s)
{
    for (int j0 = 0; j0 < n; j0 += QNB) {
        load_panel(n, A, tw, j0, s);
        const int nb = min(QNB, n - j0), m = n - j0;
        apply_block(m, nb, s.P, s.Tw, true, Y + j0, n, nc, s);
    }
}

/* Solve R X = Y for the upper triangle R of A (ld n); X, Y n x n, X may not
 * alias Y.  Blocked by QNB rows from the bottom.  Columns are independent:
 * a split command (each rank of a cluster solves a range of columns). */
__device__ __noinline__ void trsm_upper(int n, const double *A, const double *Y, double *X, Smem &s)
{
    cl_post(s, CL_TRSM, A, Y, X, nullptr, nullptr, nullptr, n, 0, 0);
    int j0, j1;
    part_range(s, n, j0, j1);
    const int nj = j1 - j0;
    const double *Yc = Y + (size_t)j0 * n;
    double *Xc = X + (size_t)j0 * n;
    for (int i1 = n; i1 > 0; i1 -= QNB) {
        const int i0 = max(0, i1 - QNB), bs = i1 - i0;
        if (i1 < n) {
            gemm_rmw<TMmaWide, true, true>(
                bs, nj, n - i1,
                [=](int i, int k) { return A[(i0 + i) + (size_t)(i1 + k) * n]; },
                [=](int k, int j) { return Xc[(i1 + k) + (size_t)j * n]; },
                [=](int i, int j) { return Yc[(i0 + i) + (size_t)j * n]; },
                [=](int i, int j, double v, double c) { Xc[(i0 + i) + (size_t)j * n] = c - v; },
                s.gsm);
        } else {
            for (int e = threadIdx.x; e < bs * nj; e += NT) {
                const int i = e % bs, j = e / bs;
                Xc[(i0 + i) + (size_t)j * n] = Yc[(i0 + i) + (size_t)j * n];
            }
        }
        double *Rb = s.phase;
        for (int e = threadIdx.x; e < QNB * QNB; e += NT) {
            const int i = e % QNB, k = e / QNB;
            Rb[e] = (i < bs && k < bs) ? A[(i0 + i) + (size_t)(i0 + k) * n] : 0.0;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nj; j += NT) {
            double x[QNB];
#pragma unroll
            for (int i = 0; i < QNB; ++i) x[i] = (i < bs) ? Xc[(i0 + i) + (size_t)j * n] : 0.0;
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
                if (i < bs) Xc[(i0 + i) + (size_t)j * n] = x[i];
        }
        __syncthreads();
    }
    cl_done(s);
}

/* ------------------------------------------------- pre-pivoted factor */
/* Column pivoting by a one-time norm sort (pre-pivoting): perm[r] is the
 * column of M with the r-th largest 2-norm; Aout[:, r] = M[:, perm[r]]. */
/* prepivot as a split command of a cluster per chain: the ranks share the
 * columns' norms (same per-column arithmetic, through the chain's global
 * staging; a norm that would raise the non-finite flag travels as NaN and
 * rank 0 raises it), every rank forms the same order, and the ranks gather
 * a range of columns each.  flag: rank 0's (unused elsewhere). */
__device__ __noinline__ void prepivot_cl(int n, const double *M, double *Aout, Smem &s,
                                         int *flag)
{
    cl_post(s, CL_PREPIV, M, Aout, nullptr, nullptr, nullptr, nullptr, n, 0, 0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *nst = s.stage + DQMC_CL_FLUSH_DOUBLES;
    double *nrm = s.vD;
    for (int c = s.cl.r * NW + warp; c < n; c += s.cl.c * NW) {
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
            if (!isfinite(mx) || isnan(v)) v = NAN;
            nst[c] = v;
        }
    }
    cl_sync();
    bool bad = false;
    for (int c = threadIdx.x; c < n; c += NT) {
        double v = nst[c];
        if (isnan(v)) {
            bad = true;
            v = -INFINITY;
        }
        nrm[c] = v;
    }
    if (bad && s.cl.r == 0) raise_flag(flag, DQMC_ST_NONFINITE);
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
    int lo, hi;
    part_range(s, n, lo, hi);
    for (int e = lo * n + threadIdx.x; e < hi * n; e += NT) {
        const int i = e % n, r = e / n;
        Aout[e] = M[i + (size_t)s.perm[r] * n];
    }
    cl_done(s);
}

__device__ __noinline__ void prepivot(int n, const double *M, double *Aout, Smem &s, int *flag)
{
    if (s.cl.c > 1) {
        prepivot_cl(n, M, Aout, s, flag);
        return;
    }
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

/* ------------------------------------------- shared-memory resident QR */
/* The factorization of qr_factor_gm (dgeqrf layout in A, dlarfg signs,
 * forward columnwise compact-WY factors in tw, so either routine's output
 * feeds the other's form/apply routines), organised so that one CTA works
 * out of shared memory:
 *  - left-looking over blocks of cb columns: a block is loaded once, the
 *    earlier panels' block reflectors are applied to it from a staged
 *    panel V, its own panels are factored in place and it is stored once;
 *  - a panel is factored with its rows in registers (panel row r on thread
 *    r mod NT): per column one CTA reduction for the norm and one 16-wide
 *    reduction for the dot products with the trailing panel columns; the
 *    compact-WY factor (dlarft) comes from V^T V on the tensor cores;
 *  - W = V^T X, op(T) W and X -= V W run on the FP64 tensor cores with
 *    every operand in shared memory.
 * Padding rows (to round16(n)) of the block and of V are kept at zero so
 * the 16-deep mma steps may run past the matrix edge. */

/* v[c] <- CTA-wide sum of v[c], c < 16, in every thread. */
__device__ __forceinline__ void block_sum16(double (&v)[16], double *rp, double *rf)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
    double h8[8], h4[4], h2[2];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double send = b4 ? v[k] : v[k + 8], keep = b4 ? v[k + 8] : v[k];
        h8[k] = keep + __shfl_xor_sync(FULL, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double send = b3 ? h8[k] : h8[k + 4], keep = b3 ? h8[k + 4] : h8[k];
        h4[k] = keep + __shfl_xor_sync(FULL, send, 8);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double send = b2 ? h4[k] : h4[k + 2], keep = b2 ? h4[k + 2] : h4[k];
        h2[k] = keep + __shfl_xor_sync(FULL, send, 4);
    }
    double h1;
    {
        const double send = b1 ? h2[0] : h2[1], keep = b1 ? h2[1] : h2[0];
        h1 = keep + __shfl_xor_sync(FULL, send, 2);
    }
    h1 += __shfl_xor_sync(FULL, h1, 1);
    /* the warp sum of value (lane >> 1) & 15 */
    if ((lane & 1) == 0) rp[((lane >> 1) & 15) * NW + warp] = h1;
    __syncthreads();
    if (threadIdx.x < 16) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) t += rp[threadIdx.x * NW + w];
        rf[threadIdx.x] = t;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = rf[c];
}

/* Partial products of V^T Xr (16 x nc, K = m rows): warp (f, g) computes
 * column fragment f over the g-th share of the 16-deep k steps. */
__device__ void qr_vtx(QrSm &q, const double *Xr, int m, int nc)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int ld = q.ld;
    const int nfr = (nc + 7) >> 3, ngr = NW / nfr, nks = (m + 15) >> 4;
    if (warp < nfr * ngr) {
        const int f = warp % nfr, g = warp / nfr;
        const int ks0 = g * nks / ngr, ks1 = (g + 1) * nks / ngr;
        const double *vb = q.V + tig + (size_t)gid * ld;
        const double *xb = Xr + tig + (size_t)(f * 8 + gid) * ld;
        double c0[4] = {0.0, 0.0, 0.0, 0.0}, c1[4] = {0.0, 0.0, 0.0, 0.0};
        int ks = ks0;
        for (; ks + 1 < ks1; ks += 2) {
            double a0[8], b0[4], a1[8], b1[4];
            const int k0 = ks * 16, k1 = k0 + 16;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a0[2 * u] = vb[k0 + 4 * u];
                a0[2 * u + 1] = vb[k0 + 4 * u + 8 * ld];
                b0[u] = xb[k0 + 4 * u];
                a1[2 * u] = vb[k1 + 4 * u];
                a1[2 * u + 1] = vb[k1 + 4 * u + 8 * ld];
                b1[u] = xb[k1 + 4 * u];
            }
            dmma<16>(c0, a0, b0);
            dmma<16>(c1, a1, b1);
        }
        if (ks < ks1) {
            double a0[8], b0[4];
            const int k0 = ks * 16;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a0[2 * u] = vb[k0 + 4 * u];
                a0[2 * u + 1] = vb[k0 + 4 * u + 8 * ld];
                b0[u] = xb[k0 + 4 * u];
            }
            dmma<16>(c0, a0, b0);
        }
        double *o = q.Wp + (size_t)(g * nfr + f) * 128;
        o[gid * 8 + 2 * tig] = c0[0] + c1[0];
        o[gid * 8 + 2 * tig + 1] = c0[1] + c1[1];
        o[(gid + 8) * 8 + 2 * tig] = c0[2] + c1[2];
        o[(gid + 8) * 8 + 2 * tig + 1] = c0[3] + c1[3];
    }
    __syncthreads();
}

/* q.V <- reflectors (unit diagonal, zero above and in the padding) of the
 * panel whose tails are at src (ld lds, m rows, nb columns). */
__device__ __forceinline__ void qr_stage_v(QrSm &q, const double *src, size_t lds, int m, int nb)
{
    const int R = (m + 15) & ~15, ld = q.ld;
    for (int r = threadIdx.x; r < R; r += NT) {
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c)
            v[c] = (c < nb && r < m && r > c) ? src[r + c * lds] : 0.0;
#pragma unroll
        for (int c = 0; c < 16; ++c) q.V[r + c * ld] = (r == c && c < nb) ? 1.0 : v[c];
    }
}

/* Householder panel of nb <= 16 columns, m rows, at Xp (ld q.ld) in
 * place: R on and above the diagonal, reflector tails below; q.taus, the
 * staged panel q.V and its compact-WY factor q.T.  Returns the number of
 * non-trivial reflectors.  The panel's columns jj.. of row r live in
 * registers x[t][0..] of thread r mod NT (t = r / NT < RPT) and shift
 * down one slot per column, so the column loop stays rolled. */
template <int RPT>
__device__ __noinline__ int qr_panel(QrSm &q, double *Xp, int m, int nb, int *flag)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ld = q.ld;
    double x[RPT][16];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        const int r = tid + NT * t;
#pragma unroll
        for (int c = 0; c < 16; ++c)
            x[t][c] = (r < m && c < nb) ? Xp[r + (size_t)c * ld] : 0.0;
    }
    int nontrivial = 0;
#pragma unroll 1
    for (int jj = 0; jj < nb; ++jj) {
        double sq = 0.0;
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const int r = tid + NT * t;
            if (r > jj && r < m) sq = fma(x[t][0], x[t][0], sq);
        }
        sq = warp_sum(sq);
        if (lane == 0) q.rp[16 * NW + warp] = sq;
        if (tid == jj) q.rp[17 * NW] = x[0][0];
        __syncthreads();
        double xn2 = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) xn2 += q.rp[16 * NW + w];
        const double alpha = q.rp[17 * NW];
        double tau = 0.0, beta = alpha, scal = 0.0;
        if (xn2 > 0.0) {
            beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
            tau = (beta - alpha) / beta;
            scal = 1.0 / (alpha - beta);
            ++nontrivial;
        }
        if (tid == 0 && (!isfinite(beta) || !isfinite(tau))) raise_flag(flag, DQMC_ST_NONFINITE);
        double vr[RPT];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const int r = tid + NT * t;
            const bool below = r > jj && r < m;
            if (below && xn2 > 0.0) x[t][0] *= scal;
            vr[t] = (r == jj) ? 1.0 : (below ? x[t][0] : 0.0);
        }
        /* d[c] = v^T (panel column jj + c), c >= 1 */
        double d[16];
        d[0] = 0.0;
#pragma unroll
        for (int c = 1; c < 16; ++c) {
            double acc = 0.0;
#pragma unroll
            for (int t = 0; t < RPT; ++t) acc = fma(vr[t], x[t][c], acc);
            d[c] = acc;
        }
        block_sum16(d, q.rp, q.rf);
        if (tid == 0) q.taus[jj] = tau;
        if (tau != 0.0) {
#pragma unroll
            for (int c = 1; c < 16; ++c) {
                const double wc = tau * d[c];
#pragma unroll
                for (int t = 0; t < RPT; ++t) x[t][c] = fma(-wc, vr[t], x[t][c]);
            }
        }
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const int r = tid + NT * t;
            if (r < m) Xp[r + (size_t)jj * ld] = (r == jj) ? beta : x[t][0];
#pragma unroll
            for (int c = 0; c < 15; ++c) x[t][c] = x[t][c + 1];
            x[t][15] = 0.0;
        }
    }
    __syncthreads();
    /* gram = V^T V on the tensor cores, then dlarft (forward columnwise):
     * T[:i, i] = -tau_i T[:i, :i] V^T v_i, T[i, i] = tau_i */
    qr_stage_v(q, Xp, ld, m, nb);
    __syncthreads();
    qr_vtx(q, q.V, m, 16);
    if (warp == 0) {
        for (int e = lane; e < 256; e += 32) {
            const int k = e & 15, i = e >> 4;
            double g = 0.0;
            if (k < i) {
#pragma unroll
                for (int gg = 0; gg < NW / 2; ++gg)
                    g += q.Wp[(size_t)(gg * 2 + (i >> 3)) * 128 + k * 8 + (i & 7)];
            }
            q.gram[k + i * 16] = g;
            q.T[e] = 0.0;
        }
        __syncwarp();
        for (int i = 0; i < nb; ++i) {
            const double ti = q.taus[i];
            if (lane < i) {
                double acc = 0.0;
                for (int k = lane; k < i; ++k) acc += q.T[lane + k * 16] * q.gram[k + i * 16];
                q.T[lane + i * 16] = -ti * acc;
            } else if (lane == i) {
                q.T[i + i * 16] = ti;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    return nontrivial;
}

/* q.V <- reflectors of panel p0 of a factored A, q.T <- its factor. */
__device__ void qr_load_v(QrSm &q, int n, const double *A, const double *tw, int p0)
{
    qr_stage_v(q, A + p0 + (size_t)p0 * n, (size_t)n, n - p0, min(16, n - p0));
    const double *twp = tw + (size_t)(p0 / 16) * 256;
    for (int e = threadIdx.x; e < 256; e += NT) q.T[e] = twp[e];
    __syncthreads();
}

/* q.W (16 x nc, ld QW) <- op(T) * (sum of the partials): T^T for H^T
 * (trans), T for H; one m16n8k16 per column fragment. */
__device__ void qr_tw(QrSm &q, int nc, bool trans)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int nfr = (nc + 7) >> 3, ngr = NW / nfr;
    if (warp < nfr) {
        const int f = warp;
        double a[8], b[4], c[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = tig + 4 * u;
            a[2 * u] = trans ? q.T[k + gid * 16] : q.T[gid + k * 16];
            a[2 * u + 1] = trans ? q.T[k + (gid + 8) * 16] : q.T[gid + 8 + k * 16];
            double t = 0.0;
            for (int g = 0; g < ngr; ++g) t += q.Wp[(size_t)(g * nfr + f) * 128 + k * 8 + gid];
            b[u] = t;
        }
        dmma<16>(c, a, b);
        double *o = q.W + (f * 8 + 2 * tig) * QW + gid;
        o[0] = c[0];
        o[QW] = c[1];
        o[8] = c[2];
        o[QW + 8] = c[3];
    }
    __syncthreads();
}

/* Xr (m rows, nc columns) -= V q.W. */
__device__ void qr_vupd(QrSm &q, double *Xr, int m, int nc)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int ld = q.ld;
    const int nrb = (m + 15) >> 4, nfr = (nc + 7) >> 3;
    for (int rb = warp; rb < nrb; rb += NW) {
        const double *vb = q.V + rb * 16 + gid + (size_t)tig * ld;
        double a[8];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[2 * u] = -vb[(size_t)4 * u * ld];
            a[2 * u + 1] = -vb[(size_t)4 * u * ld + 8];
        }
        double *xb = Xr + rb * 16 + gid;
#pragma unroll
        for (int f = 0; f < 8; ++f) {
            if (f < nfr) {
                const double *wb = q.W + tig + (f * 8 + gid) * QW;
                double b[4], c[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) b[u] = wb[4 * u];
                double *x0 = xb + (size_t)(f * 8 + 2 * tig) * ld;
                c[0] = x0[0];
                c[1] = x0[ld];
                c[2] = x0[8];
                c[3] = x0[ld + 8];
                dmma<16>(c, a, b);
                x0[0] = c[0];
                x0[ld] = c[1];
                x0[8] = c[2];
                x0[ld + 8] = c[3];
            }
        }
    }
    __syncthreads();
}

/* Xr <- op(H) Xr for the block reflector staged in q.V / q.T. */
__device__ __forceinline__ void qr_apply_sm(QrSm &q, double *Xr, int m, int nc, bool trans)
{
    qr_vtx(q, Xr, m, nc);
    qr_tw(q, nc, trans);
    qr_vupd(q, Xr, m, nc);
}

/* q.X <- columns [c0, c0+nc) of M (n x *, ld n), zero padding up to
 * round16(n) rows and cb columns; eight loads in flight per thread. */
__device__ void qr_load_cols(QrSm &q, int n, const double *M, int c0, int nc)
{
    const int R = (n + 15) & ~15, ld = q.ld;
    for (int cc = 0; cc < q.cb; cc += 8) {
        for (int r = threadIdx.x; r < R; r += NT) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                v[u] = (r < n && cc + u < nc) ? M[r + (size_t)(c0 + cc + u) * n] : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u) q.X[r + (size_t)(cc + u) * ld] = v[u];
        }
    }
    __syncthreads();
}

__device__ void qr_store_cols(QrSm &q, int n, double *M, int c0, int nc)
{
    const int ld = q.ld;
    for (int cc = 0; cc < nc; cc += 8) {
        for (int r = threadIdx.x; r < n; r += NT) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = q.X[r + (size_t)(cc + u) * ld];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (cc + u < nc) M[r + (size_t)(c0 + cc + u) * n] = v[u];
        }
    }
    __syncthreads();
}

/* Transposed block: q.X[c + rr*ld] <-> M[(r0 + rr) + c*n] for rr < nr
 * rows of M and c < n.  A warp covers 8 rows x 4 columns of M per step
 * (64-byte row runs in global memory, at most two-way bank conflicts). */
struct QrTmap {
    int rr, c, cstep;
    bool active;
};
__device__ __forceinline__ QrTmap qr_tmap(int cb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rg = cb >> 3, ncw = NW / rg;
    return QrTmap{(lane & 7) + 8 * (warp % rg), (lane >> 3) + 4 * (warp / rg), 4 * ncw,
                  warp < rg * ncw};
}

__device__ void qr_load_rows_t(QrSm &q, int n, const double *M, int r0, int nr)
{
    const int R = (n + 15) & ~15, ld = q.ld;
    const QrTmap t = qr_tmap(q.cb);
    const bool rok = t.rr < nr;
    const double *src = M + r0 + t.rr;
    double *dst = q.X + (size_t)t.rr * ld;
    for (int c0 = t.active ? t.c : R; c0 < R; c0 += 8 * t.cstep) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int c = c0 + u * t.cstep;
            v[u] = (rok && c < n) ? src[(size_t)c * n] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int c = c0 + u * t.cstep;
            if (c < R) dst[c] = v[u];
        }
    }
    __syncthreads();
}

__device__ void qr_store_rows_t(QrSm &q, int n, double *M, int r0, int nr, const double *cs)
{
    const int ld = q.ld;
    const QrTmap t = qr_tmap(q.cb);
    if (t.active && t.rr < nr) {
        double *dst = M + r0 + t.rr;
        const double *src = q.X + (size_t)t.rr * ld;
        for (int c0 = t.c; c0 < n; c0 += 8 * t.cstep) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int c = c0 + u * t.cstep;
                v[u] = c < n ? src[c] * cs[c] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int c = c0 + u * t.cstep;
                if (c < n) dst[(size_t)c * n] = v[u];
            }
        }
    }
    __syncthreads();
}

/* Applies reflector panels p0 = first, first + step, ... (count panels) of
 * a factored A to the active block: apply(p0) runs qr_apply_sm on the
 * staged panel.  While panel p0 is applied, the next panel's reflector
 * rows and compact-WY factor are already loading into registers (one row
 * of 16 per thread), so the global-memory latency of the staging overlaps
 * the products; the staged values equal qr_load_v's.  Panels taller than
 * the CTA stage through qr_load_v. */
template <class F>
__device__ __forceinline__ void qr_panels(QrSm &q, int n, const double *A, const double *tw,
                                          int first, int step, int count, F apply)
{
    if (count <= 0) return;
    const int lo = step > 0 ? first : first + step * (count - 1);
    if (((n - lo + 15) & ~15) > NT) {
        for (int i = 0; i < count; ++i) {
            const int p0 = first + i * step;
            qr_load_v(q, n, A, tw, p0);
            apply(p0);
        }
        return;
    }
    const int r = threadIdx.x, ld = q.ld;
    double v[16], t = 0.0;
    auto fetch = [&](int p0) {
        const int m = n - p0, nb = min(16, m);
        const double *src = A + p0 + (size_t)p0 * n;
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = (c < nb && r < m && r > c) ? src[r + (size_t)c * n] : 0.0;
        if (r < 256) t = tw[(size_t)(p0 / 16) * 256 + r];
    };
    fetch(first);
    for (int i = 0; i < count; ++i) {
        const int p0 = first + i * step, m = n - p0, nb = min(16, m), R = (m + 15) & ~15;
        if (r < R) {
#pragma unroll
            for (int c = 0; c < 16; ++c) q.V[r + c * ld] = (r == c && c < nb) ? 1.0 : v[c];
        }
        if (r < 256) q.T[r] = t;
        __syncthreads();
        if (i + 1 < count) fetch(p0 + step);
        apply(p0);
    }
}

/* qr_factor_sm as a split command of a cluster per chain (no more column
 * blocks than ranks): column block b belongs to rank b, which keeps it in
 * its shared memory from its load to its store.  At step b the owner of
 * block b factors it (every earlier panel is already applied) and stores
 * it; after the barrier every owner of a later block applies block b's
 * panels to its own.  Each block thus sees the one-CTA code's sequence of
 * panel applications (only their grouping into qr_panels calls differs,
 * which moves no arithmetic), so A, tw and the reflector count are the same
 * to the bit; the critical path holds one block's applications per step
 * instead of all earlier panels.  Counts and flags of the other ranks come
 * back through the chain's staging area. */
__device__ __noinline__ int qr_factor_cl(int n, double *A, double *tw, Smem &s, int *flag)
{
    cl_post(s, CL_QRF, A, tw, nullptr, nullptr, nullptr, nullptr, n, 0, 0);
    QrSm &q = s.q;
    const int ld = q.ld, cb = q.cb, r = s.cl.r;
    const int nblk = (n + cb - 1) / cb;
    const bool own = r < nblk;
    const int jb = r * cb, nc = own ? min(cb, n - jb) : 0;
    int nontrivial = 0;
    if (own) qr_load_cols(q, n, A, jb, nc);
    for (int b = 0; b < nblk; ++b) {
        if (own && r == b) {
            for (int pc = 0; pc < nc; pc += 16) {
                const int j0 = jb + pc, m = n - j0, nb = min(16, m);
                double *Xp = q.X + j0 + (size_t)pc * ld;
                if (m <= NT)
                    nontrivial += qr_panel<1>(q, Xp, m, nb, flag);
                else if (m <= 2 * NT)
                    nontrivial += qr_panel<2>(q, Xp, m, nb, flag);
                else
                    nontrivial += qr_panel<3>(q, Xp, m, nb, flag);
                double *twp = tw + (size_t)(j0 / 16) * 256;
                for (int e = threadIdx.x; e < 256; e += NT) twp[e] = q.T[e];
                if (pc + 16 < nc) qr_apply_sm(q, Xp + (size_t)16 * ld, m, nc - pc - 16, true);
            }
            qr_store_cols(q, n, A, jb, nc);
            __syncthreads();
        }
        cl_sync();
        if (own && r > b)
            qr_panels(q, n, A, tw, b * cb, 16, cb / 16,
                      [&](int p0) { qr_apply_sm(q, q.X + p0, n - p0, nc, true); });
    }
    int *rep = reinterpret_cast<int *>(s.stage + DQMC_CL_FLUSH_DOUBLES + DQMC_MAX_N);
    if (own && threadIdx.x == 0) {
        rep[2 * r] = nontrivial;
        rep[2 * r + 1] = *flag;
    }
    cl_sync();
    if (r == 0) {
        int tot = 0, bits = 0;
        for (int k = 0; k < nblk; ++k) {
            tot += rep[2 * k];
            bits |= rep[2 * k + 1];
        }
        nontrivial = tot;
        if (bits && threadIdx.x == 0) raise_flag(flag, bits);
    }
    __syncthreads();
    return nontrivial;
}

__device__ __noinline__ int qr_factor_sm(int n, double *A, double *tw, Smem &s, int *flag)
{
    QrSm &q = s.q;
    const int ld = q.ld, cb = q.cb;
    if (s.cl.c > 1 && s.cl.r == 0 && n > cb && (n + cb - 1) / cb <= s.cl.c)
        return qr_factor_cl(n, A, tw, s, flag);
    int nontrivial = 0;
    for (int jb = 0; jb < n; jb += cb) {
        const int nc = min(cb, n - jb);
        qr_load_cols(q, n, A, jb, nc);
        qr_panels(q, n, A, tw, 0, 16, jb / 16,
                  [&](int p0) { qr_apply_sm(q, q.X + p0, n - p0, nc, true); });
        for (int pc = 0; pc < nc; pc += 16) {
            const int j0 = jb + pc, m = n - j0, nb = min(16, m);
            double *Xp = q.X + j0 + (size_t)pc * ld;
            if (m <= NT)
                nontrivial += qr_panel<1>(q, Xp, m, nb, flag);
            else if (m <= 2 * NT)
                nontrivial += qr_panel<2>(q, Xp, m, nb, flag);
            else
                nontrivial += qr_panel<3>(q, Xp, m, nb, flag);
            double *twp = tw + (size_t)(j0 / 16) * 256;
            for (int e = threadIdx.x; e < 256; e += NT) twp[e] = q.T[e];
            if (pc + 16 < nc) qr_apply_sm(q, Xp + (size_t)16 * ld, m, nc - pc - 16, true);
        }
        qr_store_cols(q, n, A, jb, nc);
    }
    return nontrivial;
}

/* Q = H_1 ... H_n (n x n, ld n), column block by column block; panels
 * that start below a block's last column leave it unchanged.  A split
 * command (the ranks of a cluster take every c-th block). */
__device__ __noinline__ void qr_form_q_sm(int n, const double *A, const double *tw, double *Q,
                                          Smem &s)
{
    cl_post(s, CL_QFORM, A, tw, Q, nullptr, nullptr, nullptr, n, 0, 0);
    QrSm &q = s.q;
    const int ld = q.ld, cb = q.cb, R = (n + 15) & ~15;
    for (int jb = s.cl.r * cb; jb < n; jb += s.cl.c * cb) {
        const int nc = min(cb, n - jb);
        for (int c = 0; c < cb; ++c)
            for (int r = threadIdx.x; r < R; r += NT)
                q.X[r + (size_t)c * ld] = (c < nc && r == jb + c) ? 1.0 : 0.0;
        __syncthreads();
        const int top = ((jb + nc - 1) / 16) * 16;
        qr_panels(q, n, A, tw, top, -16, top / 16 + 1,
                  [&](int p0) { qr_apply_sm(q, q.X + p0, n - p0, nc, false); });
        qr_store_cols(q, n, Q, jb, nc);
    }
    cl_done(s);
}

/* Y (n x ncols, ld n) <- Q^T Y.  A split command (column blocks). */
__device__ __noinline__ void qr_apply_qt_sm(int n, const double *A, const double *tw, double *Y,
                                            int ncols, Smem &s)
{
    cl_post(s, CL_QT, A, tw, Y, nullptr, nullptr, nullptr, n, ncols, 0);
    QrSm &q = s.q;
    for (int jb = s.cl.r * q.cb; jb < ncols; jb += s.cl.c * q.cb) {
        const int nc = min(q.cb, ncols - jb);
        qr_load_cols(q, n, Y, jb, nc);
        qr_panels(q, n, A, tw, 0, 16, (n + 15) / 16,
                  [&](int p0) { qr_apply_sm(q, q.X + p0, n - p0, nc, true); });
        qr_store_cols(q, n, Y, jb, nc);
    }
    cl_done(s);
}

/* Xout = Xin Q diag(cs) (n x n, ld n; Xout may be Xin), a block of rows
 * at a time as (Xin Q)^T = Q^T Xin^T.  A split command (row blocks) when cs
 * is the signs vector s.vC, which the other ranks take from rank 0. */
__device__ __noinline__ void qr_apply_right_sm(int n, const double *A, const double *tw,
                                               const double *Xin, double *Xout,
                                               const double *cs, Smem &s)
{
    QrSm &q = s.q;
    const Part pt = cs == s.vC ? s.cl : Part();
    if (pt.c > 1) {
        cl_post(s, CL_QRIGHT, A, tw, Xin, Xout, nullptr, nullptr, n, 0, 0);
        if (pt.r > 0) {
            cl_pull(s.vC, n);
            __syncthreads();
        }
    }
    for (int r0 = pt.r * q.cb; r0 < n; r0 += pt.c * q.cb) {
        const int nr = min(q.cb, n - r0);
        qr_load_rows_t(q, n, Xin, r0, nr);
        qr_panels(q, n, A, tw, 0, 16, (n + 15) / 16,
                  [&](int p0) { qr_apply_sm(q, q.X + p0, n - p0, nr, true); });
        qr_store_rows_t(q, n, Xout, r0, nr, cs);
    }
    if (pt.c > 1) cl_done(s);
}

/* Dispatch: shared-memory QR when the block fits, else the global one. */
__device__ __forceinline__ int qr_factor(int n, double *A, double *tw, Smem &s, int *flag)
{
    return s.q.cb ? qr_factor_sm(n, A, tw, s, flag) : qr_factor_gm(n, A, tw, s, flag);
}
__device__ __forceinline__ void qr_form_q(int n, const double *A, const double *tw, double *Q,
                                          Smem &s)
{
    if (s.q.cb)
        qr_form_q_sm(n, A, tw, Q, s);
    else
        qr_form_q_gm(n, A, tw, Q, s);
}
__device__ __forceinline__ void qr_apply_qt(int n, const double *A, const double *tw, double *Y,
                                            int nc, Smem &s)
{
    if (s.q.cb)
        qr_apply_qt_sm(n, A, tw, Y, nc, s);
    else
        qr_apply_qt_gm(n, A, tw, Y, nc, s);
}

/* ------------------------------------------------------------------ UDV */
struct Udv {
    double *U, *T, *ell, *det, *perm;
};

__device__ __forceinline__ Udv udv_at(double *base, int n)
{
    const size_t nn = (size_t)n * n;
    return Udv{base, base + nn, base + 2 * nn, base + 2 * nn + n, base + 2 * nn + n + 2};
}

__device__ void udv_identity(Udv u, int n)
{
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const double v = (e % n == e / n) ? 1.0 : 0.0;
        u.U[e] = v;
        u.T[e] = v;
    }
    for (int i = threadIdx.x; i < n; i += NT) {
        u.ell[i] = 0.0;
        u.perm[i] = (double)i;
    }
    if (threadIdx.x == 0) *u.det = 1.0;
    __syncthreads();
}

__device__ void udv_copy(Udv d, Udv s, int n)
{
    const double *sU = s.U, *sT = s.T;
    double *dU = d.U, *dT = d.T;
    ew_batched(n * n, [=](int e) { return sU[e]; }, [=](int e, double x) { dU[e] = x; });
    ew_batched(n * n, [=](int e) { return sT[e]; }, [=](int e, double x) { dT[e] = x; });
    for (int i = threadIdx.x; i < n; i += NT) {
        d.ell[i] = s.ell[i];
        d.perm[i] = s.perm[i];
    }
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

/* The UDV updates' n x n products as split commands of a cluster per
 * chain (each rank forms a share of the output tiles; the small vectors the
 * epilogues read come from rank 0's shared memory):
 *   UG_LMUL1  C = (A B) diag(vA)            udv_lmul's B U D
 *   UG_RMUL1  C = diag(vA) (A B)            udv_rmul's D T B
 *   UG_COMB1  C = diag(vA) (A B) diag(vD)   udv_combine's D_L T_L U_R D_R
 *   UG_RT     C = diag(1/vD) triu(A) B[perm, :]   R T_old of lmul / combine
 * with the epilogue expressions of the one-CTA code, so the results are the
 * same to the bit. */
enum { UG_LMUL1 = 0, UG_RMUL1, UG_COMB1, UG_RT };

__device__ __noinline__ void udv_gemm(int kind, int n, const double *A, const double *B,
                                      double *C, Smem &s)
{
    cl_post(s, CL_UGEMM, A, B, C, nullptr, nullptr, nullptr, n, kind, 0);
    if (s.cl.r > 0) {
        if (kind == UG_RT) {
            cl_pull(s.vD, n);
            cl_pull(s.perm, n);
        } else {
            cl_pull(s.vA, n);
            if (kind == UG_COMB1) cl_pull(s.vD, n);
        }
    }
    const double *va = s.vA, *vd = s.vD;
    const int *perm = s.perm;
    switch (kind) {
    case UG_LMUL1:
        gemm_nn_part(n, n, n, A, n, B, n,
                     [=](int i, int j, double v) { C[i + (size_t)j * n] = v * va[j]; }, s.gsm,
                     s.cl);
        break;
    case UG_RMUL1:
        gemm_nn_part(n, n, n, A, n, B, n,
                     [=](int i, int j, double v) { C[i + (size_t)j * n] = va[i] * v; }, s.gsm,
                     s.cl);
        break;
    case UG_COMB1:
        gemm_nn_part(n, n, n, A, n, B, n,
                     [=](int i, int j, double v) { C[i + (size_t)j * n] = va[i] * v * vd[j]; },
                     s.gsm, s.cl);
        break;
    default:
        gemm_sq_part<true, true>(
            n, n, n, [=](int i, int k) { return k >= i ? A[i + (size_t)k * n] : 0.0; },
            [=](int k, int j) { return B[perm[k] + (size_t)j * n]; },
            [=](int i, int j, double v) { C[i + (size_t)j * n] = v / vd[i]; }, s.gsm, s.cl);
        break;
    }
    cl_done(s);
}

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
    if (B != nullptr && s.cl.c > 1) {
        udv_gemm(UG_LMUL1, n, B, U, M, s);
    } else if (B != nullptr) {
        gemm_nn(n, n, n, B, n, U, n,
                [=](int i, int j, double v) { M[i + (size_t)j * n] = v * eD[j]; }, s.gsm);
    } else {
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return expK[i + (size_t)k * n]; },
            [=](int k, int j) { return U[k + (size_t)j * n]; },
            [=](int i, int j, double v) { M[i + (size_t)j * n] = v * eD[j]; }, s.gsm, Ident(),
            [=](int k, int, double x) { return vl[k] * x; });
    }
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    const double *R = w.m1;
    const double *T = u.T;
    const int *perm = s.perm;
    double *Tn = w.m2;
    double *rd = s.vD;
    for (int i = threadIdx.x; i < n; i += NT) rd[i] = R[i + (size_t)i * n];
    __syncthreads();
    if (s.cl.c > 1)
        udv_gemm(UG_RT, n, R, T, Tn, s);
    else
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return k >= i ? R[i + (size_t)k * n] : 0.0; },
            [=](int k, int j) { return T[perm[k] + (size_t)j * n]; },
            [=](int i, int j, double v) { Tn[i + (size_t)j * n] = v / rd[i]; }, s.gsm);
    {
        double *uT = u.T;
        const double *tn = Tn;
        ew_batched(n * n, [=](int e) { return tn[e]; }, [=](int e, double x) { uT[e] = x; });
    }
    qr_form_q(n, w.m1, w.tw, u.U, s);
    {
        double *uU = u.U;
        const double *sg = s.vC;
        ew_batched(n * n, [=](int e) { return uU[e]; },
                   [=](int e, double x) { uU[e] = x * sg[e / n]; });
    }
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
    if (s.cl.c > 1)
        udv_gemm(UG_RMUL1, n, T, B, M, s);
    else
        gemm_nn(n, n, n, T, n, B, n,
                [=](int i, int j, double v) { M[i + (size_t)j * n] = eD[i] * v; }, s.gsm);
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    if (s.q.cb) {
        /* U <- U Q diag(sign R_ii), Q applied from the right in blocks */
        qr_apply_right_sm(n, w.m1, w.tw, u.U, u.U, s.vC, s);
    } else {
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
    }
    const double *R = w.m1;
    {
        double *rd = s.vD, *uT = u.T;
        const int *perm = s.perm;
        for (int i = threadIdx.x; i < n; i += NT) rd[i] = R[i + (size_t)i * n];
        __syncthreads();
        ew_batched(
            n * n, [=](int e) { return (e % n) <= (e / n) ? R[e] : 0.0; },
            [=](int e, double x) {
                const int i = e % n, r = e / n;
                uT[i + (size_t)perm[r] * n] = r >= i ? x / rd[i] : 0.0;
            });
    }
    for (int i = threadIdx.x; i < n; i += NT) {
        u.ell[i] = s.vB[i];
        u.perm[i] = (double)s.perm[i];
    }
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
        if (s.cl.c > 1)
            udv_gemm(UG_COMB1, n, TL, UR, M, s);
        else
            gemm_nn(n, n, n, TL, n, UR, n,
                    [=](int i, int j, double v) { M[i + (size_t)j * n] = eL[i] * v * eR[j]; },
                    s.gsm);
    }
    prepivot(n, M, w.m1, s, flag);
    const int nt = qr_factor(n, w.m1, w.tw, s, flag);
    const int sg = qr_diag(n, w.m1, s, flag);
    if (s.q.cb) {
        qr_apply_right_sm(n, w.m1, w.tw, l.U, o.U, s.vC, s);
    } else {
        qr_form_q(n, w.m1, w.tw, w.m0, s);
        const double *UL = l.U, *Q = w.m0, *sgn = s.vC;
        double *Uo = o.U;
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return UL[i + (size_t)k * n]; },
            [=](int k, int j) { return Q[k + (size_t)j * n]; },
            [=](int i, int j, double v) { Uo[i + (size_t)j * n] = v * sgn[j]; }, s.gsm);
    }
    const double *R = w.m1, *TR = r.T;
    const int *perm = s.perm;
    double *To = o.T;
    double *rd = s.vD;
    for (int i = threadIdx.x; i < n; i += NT) rd[i] = R[i + (size_t)i * n];
    __syncthreads();
    if (s.cl.c > 1)
        udv_gemm(UG_RT, n, R, TR, To, s);
    else
        gemm_sq<true, true>(
            n, n, n, [=](int i, int k) { return k >= i ? R[i + (size_t)k * n] : 0.0; },
            [=](int k, int j) { return TR[perm[k] + (size_t)j * n]; },
            [=](int i, int j, double v) { To[i + (size_t)j * n] = v / rd[i]; }, s.gsm);
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
    double *dbi = s.vA, *dsm = s.vB;
    double bad_ell = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        const double l = ell[i];
        bad_ell += isfinite(l) ? 0.0 : 1.0;   /* fmax/fmin below would drop a NaN */
        dbi[i] = exp(-fmax(l, 0.0));
        dsm[i] = exp(fmin(l, 0.0));
    }
    if (block_reduce<false>(bad_ell, s.red) != 0.0) raise_flag(flag, DQMC_ST_NONFINITE);
    if (s.q.cb >= 32) {
        /* U^T through shared memory, 32 columns of U at a time: columns of U
         * are read and rows of Y / X written in contiguous runs */
        const int lds = n + 1;
        double *S = s.q.X;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int nc = min(32, n - c0);
            ew_batched(n * 32, [=](int e) {
                const int j = e % n, c = e / n;
                return c < nc ? U[j + (size_t)(c0 + c) * n] : 0.0;
            }, [=](int e, double x) { S[(e % n) + (e / n) * lds] = x; });
            __syncthreads();
            ew_batched(n * 32, [=](int e) {
                const int c = e & 31, j = e >> 5;
                return c < nc ? T[(c0 + c) + (size_t)j * n] : 0.0;
            }, [=](int e, double t) {
                const int c = e & 31, j = e >> 5;
                if (c < nc) {
                    const int i = c0 + c;
                    const double y = dbi[i] * S[j + c * lds];
                    Y[i + (size_t)j * n] = y;
                    X[i + (size_t)j * n] = y + dsm[i] * t;
                }
            });
            __syncthreads();
        }
    } else {
        for (int e = threadIdx.x; e < n * n; e += NT) {
            const int i = e % n, j = e / n;
            const double ut = U[j + (size_t)i * n];
            Y[e] = dbi[i] * ut;
            X[e] = dbi[i] * ut + dsm[i] * T[e];
        }
        __syncthreads();
    }
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

/* Y[i, j] = sc[i] * U[j, i] (n x n): U^T row-scaled, read through shared
 * memory 32 columns of U at a time when the shared-memory QR area exists. */
__device__ void scaled_transpose(int n, const double *U, const double *sc, double *Y, Smem &s)
{
    if (s.q.cb >= 32) {
        const int lds = n + 1;
        double *S = s.q.X;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int nc = min(32, n - c0);
            ew_batched(n * 32, [=](int e) {
                const int j = e % n, c = e / n;
                return c < nc ? U[j + (size_t)(c0 + c) * n] : 0.0;
            }, [=](int e, double x) { S[(e % n) + (e / n) * lds] = x; });
            __syncthreads();
            for (int e = threadIdx.x; e < n * 32; e += NT) {
                const int c = e & 31, j = e >> 5;
                if (c < nc) Y[(c0 + c) + (size_t)j * n] = sc[c0 + c] * S[j + c * lds];
            }
            __syncthreads();
        }
    } else {
        for (int e = threadIdx.x; e < n * n; e += NT) {
            const int i = e % n, j = e / n;
            Y[e] = sc[i] * U[j + (size_t)i * n];
        }
        __syncthreads();
    }
}

/* G = (1 + L R)^{-1} for two UDV factors without forming their product
 * (udv_inv_one_plus_two_sided_work, linalg.c:1117-1389; green_rebuild =
 * two_sided | centered): with D = Db Ds (Db = max(D,1), Ds = min(D,1), all
 * held as exp of the log scale, so every factor below is <= 1)
 *     1 + U_L D_L T_L U_R D_R T_R = U_L Db_L H Db_R T_R,
 *     H = Db_L^-1 U_L^T T_R^-1 Db_R^-1 + Ds_L (T_L U_R) Ds_R,
 *     G = T_R^-1 Db_R^-1 H^-1 Db_L^-1 U_L^T,
 * with T_R = R_unit P^T (the right factor is an rmul product), so T_R^-1 =
 * P R_unit^-1.  H^-1 by a Householder QR solve.  Sign of det(1 + L R) =
 * det U_L * det H.  X: one more n x n scratch. */
__device__ __noinline__ int udv_green2(int n, Udv l, Udv r, double *G, double *X, Scr w, Smem &s,
                                       int *flag)
{
    double *Ru = w.m2, *Tinv = w.m0, *A = w.m1;
    const double *TR = r.T, *rp = r.perm;
    /* R_unit = T_R P (column gather), R_unit^-1 by a unit-triangular solve */
    ew_batched(n * n, [=](int e) {
        const int i = e % n, c = e / n;
        return TR[i + (size_t)rp[c] * n];
    }, [=](int e, double x) { Ru[e] = x; });
    for (int e = threadIdx.x; e < n * n; e += NT) Tinv[e] = (e % n == e / n) ? 1.0 : 0.0;
    __syncthreads();
    trsm_upper(n, Ru, Tinv, A, s);
    /* T_R^-1 = P R_unit^-1: row r of R_unit^-1 is row perm[r] of T_R^-1 */
    ew_batched(n * n, [=](int e) { return A[e]; }, [=](int e, double x) {
        const int rr = e % n, c = e / n;
        Tinv[(int)rp[rr] + (size_t)c * n] = x;
    });
    __syncthreads();
    double *dbl = s.vA, *dsl = s.vB, *dsr = s.vC, *dbr = s.vD;
    double bad_ell = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        const double a = l.ell[i], b = r.ell[i];
        bad_ell += (isfinite(a) && isfinite(b)) ? 0.0 : 1.0;
        dbl[i] = exp(-fmax(a, 0.0));
        dsl[i] = exp(fmin(a, 0.0));
        dbr[i] = exp(-fmax(b, 0.0));
        dsr[i] = exp(fmin(b, 0.0));
    }
    if (block_reduce<false>(bad_ell, s.red) != 0.0) raise_flag(flag, DQMC_ST_NONFINITE);
    const double *UL = l.U, *TL = l.T, *UR = r.U, *Ti = Tinv;
    /* A = U_L^T T_R^-1, H (in Ru) = T_L U_R, then H <- scalings */
    gemm_sq<false, true>(
        n, n, n, [=](int i, int k) { return UL[k + (size_t)i * n]; },
        [=](int k, int j) { return Ti[k + (size_t)j * n]; },
        [=](int i, int j, double v) { A[i + (size_t)j * n] = v; }, s.gsm);
    gemm_nn(n, n, n, TL, n, UR, n, [=](int i, int j, double v) { Ru[i + (size_t)j * n] = v; },
            s.gsm);
    {
        const double *Ac = A;
        double *H = Ru;
        ew_batched(n * n, [=](int e) { return Ac[e]; }, [=](int e, double a) {
            const int i = e % n, j = e / n;
            H[e] = (dbl[i] * a) * dbr[j] + (dsl[i] * H[e]) * dsr[j];
        });
    }
    __syncthreads();
    /* right-hand side Db_L^-1 U_L^T, QR solve of H */
    scaled_transpose(n, UL, dbl, A, s);
    const int nt = qr_factor(n, Ru, w.tw, s, flag);
    const int sg = qr_diag(n, Ru, s, flag);
    qr_apply_qt(n, Ru, w.tw, A, n, s);
    trsm_upper(n, Ru, A, X, s);
    /* G = T_R^-1 (Db_R^-1 X) */
    ew_batched(n * n, [=](int e) { return X[e]; }, [=](int e, double x) { X[e] = dbr[e % n] * x; });
    __syncthreads();
    gemm_nn(n, n, n, Tinv, n, X, n, [=](int i, int j, double v) { G[i + (size_t)j * n] = v; },
            s.gsm);
    double bad = 0.0;
    for (int e = threadIdx.x; e < n * n; e += NT) bad += isfinite(G[e]) ? 0.0 : 1.0;
    bad = block_reduce<false>(bad, s.red);
    if (bad != 0.0) raise_flag(flag, DQMC_ST_NONFINITE);
    return (int)(*l.det * ((nt & 1) ? -1.0 : 1.0) * sg);
}

/* ----------------------------------------------------- slice operations */
/* G <- B_l G B_l^{-1} = expK diag(v) G diag(1/v) expKinv (green.c:509-527). */
/* The wrap and the B-block chain as split commands of a cluster per chain:
 * rank 0 posts them (cl_post) and every rank forms its share of the
 * elementwise pass and of each product's tiles, with a cluster barrier
 * between dependent steps.  Same arithmetic per element as wrap_green,
 * wrap_green_back and bblock below. */
__device__ __noinline__ void wrap_green_cl(int n, double *G, double *tmp, const double *expK,
                           const double *expKinv, const signed char *fl, double v0,
                           double v1, double vi0, double vi1, Smem &s)
{
    cl_post(s, CL_WRAP, G, tmp, expK, expKinv, fl, nullptr, n, 0, 0, v0, v1, vi0, vi1);
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    __syncthreads();
    /* G <- diag(v) G diag(1/v) in place (G is overwritten below), so both
     * products are plain */
    int lo, hi;
    part_range(s, n * n, lo, hi);
    ew_batched(hi - lo, [=](int e) { return G[lo + e]; }, [=](int e, double x) {
        const int f = lo + e;
        G[f] = x * (vv[f % n] * vi[f / n]);
    });
    part_sync(s);
    gemm_nn_part(n, n, n, expK, n, G, n,
                 [=](int i, int j, double v) { tmp[i + (size_t)j * n] = v; }, s.gsm, s.cl);
    part_sync(s);
    gemm_nn_part(n, n, n, tmp, n, expKinv, n,
                 [=](int i, int j, double v) { G[i + (size_t)j * n] = v; }, s.gsm, s.cl);
    cl_done(s);
}

__device__ __noinline__ void wrap_green_back_cl(int n, double *G, double *tmp, const double *expK,
                                             const double *expKinv, const signed char *fl,
                                             double v0, double v1, double vi0, double vi1,
                                             Smem &s)
{
    cl_post(s, CL_WRAP_BACK, G, tmp, expK, expKinv, fl, nullptr, n, 0, 0, v0, v1, vi0, vi1);
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    gemm_nn_part(n, n, n, expKinv, n, G, n,
                 [=](int i, int j, double v) { tmp[i + (size_t)j * n] = v; }, s.gsm, s.cl);
    part_sync(s);
    gemm_nn_part(n, n, n, tmp, n, expK, n,
                 [=](int i, int j, double v) { G[i + (size_t)j * n] = (vi[i] * v) * vv[j]; },
                 s.gsm, s.cl);
    cl_done(s);
}

__device__ __noinline__ void bblock_cl(int n, int l0, int len, const signed char *field, const double *expK,
                       double v0, double v1, double *out, double *X, double *Y, Smem &s)
{
    cl_post(s, CL_BBLOCK, field, expK, out, X, Y, nullptr, n, l0, len, v0, v1);
    /* Intermediate products are stored row-scaled by the next slice's
     * diag(v) (folded into the producing GEMM's epilogue), so every
     * product is a plain expK * X. */
    const signed char *f0 = field + (size_t)l0 * n;
    double *first = (len == 1) ? out : X;
    double *vv = s.vA;
    for (int i = threadIdx.x; i < n; i += NT)
        vv[i] = (len == 1) ? 1.0 : (field[(size_t)(l0 + 1) * n + i] > 0 ? v1 : v0);
    __syncthreads();
    int lo, hi;
    part_range(s, n * n, lo, hi);
    ew_batched(hi - lo, [=](int e) { return expK[lo + e]; }, [=](int e, double x) {
        const int f = lo + e;
        first[f] = vv[f % n] * (x * (f0[f / n] > 0 ? v1 : v0));
    });
    part_sync(s);
    const double *src = first;
    for (int p = 1; p < len; ++p) {
        const bool lastp = (p == len - 1);
        double *dst = lastp ? out : ((src == X) ? Y : X);
        if (!lastp) {
            const signed char *fn = field + (size_t)(l0 + p + 1) * n;
            for (int i = threadIdx.x; i < n; i += NT) vv[i] = fn[i] > 0 ? v1 : v0;
        }
        gemm_nn_part(n, n, n, expK, n, src, n,
                     [=](int i, int j, double v) { dst[i + (size_t)j * n] = lastp ? v : vv[i] * v; },
                     s.gsm, s.cl);
        if (!lastp) part_sync(s);
        src = dst;
    }
    cl_done(s);
}

__device__ __noinline__ void wrap_green(int n, double *G, double *tmp, const double *expK,
                           const double *expKinv, const signed char *fl, double v0,
                           double v1, double vi0, double vi1, Smem &s)
{
    if (s.cl.c > 1) {
        wrap_green_cl(n, G, tmp, expK, expKinv, fl, v0, v1, vi0, vi1, s);
        return;
    }
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    __syncthreads();
    /* G <- diag(v) G diag(1/v) in place (G is overwritten below), so both
     * products are plain */
    ew_batched(n * n, [=](int e) { return G[e]; },
               [=](int e, double x) { G[e] = x * (vv[e % n] * vi[e / n]); });
    gemm_nn(n, n, n, expK, n, G, n, [=](int i, int j, double v) { tmp[i + (size_t)j * n] = v; },
            s.gsm);
    gemm_nn(n, n, n, tmp, n, expKinv, n,
            [=](int i, int j, double v) { G[i + (size_t)j * n] = v; }, s.gsm);
}

/* G <- B_l^{-1} G B_l = diag(1/v) expKinv G expK diag(v)
 * (green_wrap_backward, green.c:529-548); the diagonals in the epilogue. */
__device__ __noinline__ void wrap_green_back(int n, double *G, double *tmp, const double *expK,
                                             const double *expKinv, const signed char *fl,
                                             double v0, double v1, double vi0, double vi1,
                                             Smem &s)
{
    if (s.cl.c > 1) {
        wrap_green_back_cl(n, G, tmp, expK, expKinv, fl, v0, v1, vi0, vi1, s);
        return;
    }
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    gemm_nn(n, n, n, expKinv, n, G, n, [=](int i, int j, double v) { tmp[i + (size_t)j * n] = v; },
            s.gsm);
    gemm_nn(n, n, n, tmp, n, expK, n,
            [=](int i, int j, double v) { G[i + (size_t)j * n] = (vi[i] * v) * vv[j]; }, s.gsm);
}

/* out = B_{l0+len-1} ... B_{l0} (green.c:151-166); X, Y ping-pong scratch. */
__device__ __noinline__ void bblock(int n, int l0, int len, const signed char *field, const double *expK,
                       double v0, double v1, double *out, double *X, double *Y, Smem &s)
{
    if (s.cl.c > 1) {
        bblock_cl(n, l0, len, field, expK, v0, v1, out, X, Y, s);
        return;
    }
    /* Intermediate products are stored row-scaled by the next slice's
     * diag(v) (folded into the producing GEMM's epilogue), so every
     * product is a plain expK * X. */
    const signed char *f0 = field + (size_t)l0 * n;
    double *first = (len == 1) ? out : X;
    double *vv = s.vA;
    for (int i = threadIdx.x; i < n; i += NT)
        vv[i] = (len == 1) ? 1.0 : (field[(size_t)(l0 + 1) * n + i] > 0 ? v1 : v0);
    __syncthreads();
    ew_batched(n * n, [=](int e) { return expK[e]; }, [=](int e, double x) {
        first[e] = vv[e % n] * (x * (f0[e / n] > 0 ? v1 : v0));
    });
    __syncthreads();
    const double *src = first;
    for (int p = 1; p < len; ++p) {
        const bool lastp = (p == len - 1);
        double *dst = lastp ? out : ((src == X) ? Y : X);
        if (!lastp) {
            const signed char *fn = field + (size_t)(l0 + p + 1) * n;
            for (int i = threadIdx.x; i < n; i += NT) vv[i] = fn[i] > 0 ? v1 : v0;
        }
        gemm_nn(n, n, n, expK, n, src, n,
                [=](int i, int j, double v) { dst[i + (size_t)j * n] = lastp ? v : vv[i] * v; },
                s.gsm);
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
