/* Sweep, measurement and test kernels.  One CTA = one chain. */
#pragma once
#include "dqmc_device.cuh"
#include "dqmc_gpu.h"
#include "dqmc_split.cuh"

namespace DQMC_NS {

enum { KF_MEASURE = 1, KF_SDRIFT = 2, KF_STAB_DRIFT = 4, KF_MIXED = 8 };

/* Phase timer: thread 0 charges the cycles since the last mark to a phase.
 * Phases end at a CTA barrier, so thread 0's clock covers all threads. */
struct PhaseClock {
    long long t;
    __device__ __forceinline__ void mark() { t = clock64(); }
    __device__ __forceinline__ void charge(DqmcChainDev *ch, int ph, unsigned calls = 0)
    {
        if (threadIdx.x == 0) {
            const long long now = clock64();
            ch->prof[ph] += (unsigned long long)(now - t);
            ch->pcalls[ph] += calls;
            t = now;
        }
    }
};

__device__ __forceinline__ Scr chain_scr(const DqmcChainDev *ch)
{
    return Scr{ch->w[0], ch->w[1], ch->w[2], ch->twall};
}

/* One site block of the delayed update (green.c:384-480, PH path).
 *
 * Proposals: warp 0, lane b holding column b of the block's current G~
 * (gt[c][b] = G~[i0+c, i0+b]) in registers; the site loop is unrolled so
 * every index is static.  The ratio uses gt[a][a] exactly as
 * green_delay_ratio_N / green_ph_down_ratio_N (green.c:402-416), one RNG
 * draw per site, always consumed (dqmc.c:666-668).  An accepted flip
 * applies green_delay_accept's rank-1 update G~ -= fac (e_a - G~[:,a])
 * G~[a,:] to the trailing block (rows and columns > a, the only entries
 * later sites read) and records row a and column a of G~ at that moment.
 *
 * Flush: the reference's delayed vectors C[:,p] = fac_p u_p, V[:,p] = v_p
 * satisfy u_p = e - G[:,i_p] + sum_{q<p} C[:,q] V[i_p,q] and v_p = G[i_p,:]
 * - sum_{q<p} V[:,q] C[i_p,q]; with the recorded entries this is
 * U (I - F Su) = E_A - G[:,A] and V (I + Sc) = G[A,:]^T (Su, Sc strictly
 * upper m x m), so U and V come from two unit-triangular inverses, and
 * G -= U F V^T is one rank-m GEMM (green_delay_flush, green.c:462-475).
 *
 * Pairing: with mA > 0 the previous block's Zs_A, Ys_A (mA columns / rows)
 * are staged but not yet subtracted from G, so this block works on
 * G~ = G - Zs_A Ys_A: its proposals read G~[B,B], and by Woodbury
 *   Zs_B = [(E_B - G[:,B]) Tu + Zs_A Qa] F,  Qa = Ys_A[:,B] Tu,
 *   Ys_B = Tv^T G[B,:] - Pa Ys_A,            Pa = Tv^T Zs_A[B,:];
 * one GEMM then subtracts both blocks (rank mA + m).  Returns the number
 * of staged columns left for the next block (0 after a flush).
 *
 * Zs and Ys are formed one row / one column per thread (FP64 FMAs on the
 * accepted columns / rows of G, coalesced across the CTA): no CTA-wide GEMM
 * pipeline for these thin products. */
/* Zs_B rows and Ys_B columns of a site block's flush (block_flush, after
 * the inverses): TuP, facs and the pair-staging operands TvP, Qa, PaT (in
 * the GEMM staging area) and the accepted list are in shared memory.  Rows
 * and columns are independent: a split command of a cluster per chain.
 * Rank 0 copies those small operands to the chain's global staging area
 * before posting (`stage`, DQMC_CL_STAGE_DOUBLES; the other ranks read it
 * from L2 into the same shared-memory places, rather than all reading rank
 * 0's shared memory at once), and every rank forms a contiguous range of
 * rows and columns. */
__device__ __noinline__ void flush_zy(int n, int i0, int m, int mA, const double *G, double *Zs,
                                      double *Ys, int ldy, const double *TuP,
                                      const double *facs, double *stage, Smem &s)
{
    constexpr int KB = DQMC_MAX_KB;
    constexpr int LT = KB + 2;
    const int tid = threadIdx.x;
    double *TvP = s.gsm + 2 * KB * LT, *YA = s.gsm + KB * LT, *ZA = s.gsm;
    const int *alist = s.iscr;
    if (s.cl.c > 1) {
        /* stage: TuP | TvP | YA | ZA (KB x LT each) | facs | accepted list */
        double *tuS = stage, *tvS = stage + KB * LT, *yaS = stage + 2 * KB * LT,
               *zaS = stage + 3 * KB * LT, *fS = stage + 4 * KB * LT;
        int *aS = reinterpret_cast<int *>(fS + KB);
        const int nblk = mA > 0 ? 4 : 2;
        double *tuL = const_cast<double *>(TuP), *fL = const_cast<double *>(facs);
        int *aL = s.iscr;
        auto src = [=](int e) -> const double * {
            const int b = e / (KB * LT), o = e % (KB * LT);
            return b == 0 ? tuL + o : b == 1 ? TvP + o : b == 2 ? YA + o : ZA + o;
        };
        auto dst = [=](int e) -> double * {
            const int b = e / (KB * LT), o = e % (KB * LT);
            return b == 0 ? tuS + o : b == 1 ? tvS + o : b == 2 ? yaS + o : zaS + o;
        };
        if (s.cl.r == 0) {
            ew_batched(nblk * KB * LT, [=](int e) { return *src(e); },
                       [=](int e, double x) { *dst(e) = x; });
            for (int e = tid; e < KB; e += NT) {
                fS[e] = fL[e];
                aS[e] = aL[e];
            }
        }
        cl_post(s, CL_ZY, G, Zs, Ys, TuP, facs, stage, n, i0, m | (mA << 8) | (ldy << 16));
        if (s.cl.r > 0) {
            ew_batched(nblk * KB * LT, [=](int e) { return *dst(e); },
                       [=](int e, double x) { *const_cast<double *>(src(e)) = x; });
            for (int e = tid; e < KB; e += NT) {
                fL[e] = fS[e];
                aL[e] = aS[e];
            }
            __syncthreads();
        }
    }
    int lo, hi;
    part_range(s, n, lo, hi);
    /* Zs_B rows and Ys_B columns, after the mA staged ones.  Pass 1: the
     * G part, (E_B - G[:,B]) Tu and Tv^T G[B,:]; pass 2 (staged block):
     * + Zs_A Qa and - Pa Ys_A, the staged operands of a row / column loaded
     * as one batch; F scales Zs_B once, at the end. */
    const double *Qa = YA, *PaT = ZA;
    double *ZsB = Zs + (size_t)mA * n;
    double *YsB = Ys + mA;
    const bool two = mA > 0;
    for (int i = lo + tid; i < hi; i += NT) {
        double x[KB];
#pragma unroll
        for (int q = 0; q < KB; ++q) {
            const int c = i0 + alist[q];
            x[q] = q < m ? (i == c ? 1.0 : 0.0) - G[i + (size_t)c * n] : 0.0;
        }
        for (int p0 = 0; p0 < m; p0 += 8) {
            double z[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) z[u] = 0.0;
#pragma unroll
            for (int q0 = 0; q0 < KB; q0 += 8) {
                if (q0 < m) {
#pragma unroll
                    for (int q = q0; q < q0 + 8; ++q) {
#pragma unroll
                        for (int u = 0; u < 8; u += 2) {
                            const double2 t =
                                *reinterpret_cast<const double2 *>(TuP + q * LT + p0 + u);
                            z[u] = fma(x[q], t.x, z[u]);
                            z[u + 1] = fma(x[q], t.y, z[u + 1]);
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (p0 + u < m) ZsB[i + (size_t)(p0 + u) * n] = two ? z[u] : z[u] * facs[p0 + u];
        }
    }
    /* Ys_B: a warp per column j, lane p its entry p, lane q loading row
     * i0 + alist[q] of column j (one coalesced segment of the column) and
     * handing it to the other lanes by shuffles; each entry sums over q in
     * the order of the row-per-thread Zs loop above.  YS_COLS columns per
     * warp at a time for independent FMA chains. */
    constexpr int YS_COLS = 8;
    const int lane = tid & 31, warp = tid >> 5;
    const int m8 = (m + 7) & ~7, mA8 = (mA + 7) & ~7;
    const int rq = i0 + alist[lane < m ? lane : 0];
    for (int j0 = lo + warp * YS_COLS; j0 < hi; j0 += NW * YS_COLS) {
        double yv[YS_COLS], z[YS_COLS];
#pragma unroll
        for (int c = 0; c < YS_COLS; ++c) {
            const int j = j0 + c;
            yv[c] = (j < hi && lane < m) ? G[rq + (size_t)j * n] : 0.0;
            z[c] = 0.0;
        }
        for (int q = 0; q < m8; ++q) {
            const double t = TvP[q * LT + lane];
#pragma unroll
            for (int c = 0; c < YS_COLS; ++c) z[c] = fma(t, __shfl_sync(FULL, yv[c], q), z[c]);
        }
#pragma unroll
        for (int c = 0; c < YS_COLS; ++c)
            if (j0 + c < hi && lane < m) YsB[lane + (size_t)(j0 + c) * ldy] = z[c];
    }
    if (two) {
        /* each thread re-reads only what it wrote in pass 1 */
        for (int i = lo + tid; i < hi; i += NT) {
            double za[KB];
#pragma unroll
            for (int k = 0; k < KB; ++k) za[k] = k < mA ? Zs[i + (size_t)k * n] : 0.0;
            for (int p0 = 0; p0 < m; p0 += 8) {
                double z[8];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    z[u] = p0 + u < m ? ZsB[i + (size_t)(p0 + u) * n] : 0.0;
#pragma unroll
                for (int k0 = 0; k0 < KB; k0 += 8) {
                    if (k0 < mA) {
#pragma unroll
                        for (int k = k0; k < k0 + 8; ++k) {
#pragma unroll
                            for (int u = 0; u < 8; u += 2) {
                                const double2 t =
                                    *reinterpret_cast<const double2 *>(Qa + k * LT + p0 + u);
                                z[u] = fma(za[k], t.x, z[u]);
                                z[u + 1] = fma(za[k], t.y, z[u + 1]);
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (p0 + u < m) ZsB[i + (size_t)(p0 + u) * n] = z[u] * facs[p0 + u];
            }
        }
        for (int j0 = lo + warp * YS_COLS; j0 < hi; j0 += NW * YS_COLS) {
            double ya[YS_COLS], z[YS_COLS];
#pragma unroll
            for (int c = 0; c < YS_COLS; ++c) {
                const int j = j0 + c;
                ya[c] = (j < hi && lane < mA) ? Ys[lane + (size_t)j * ldy] : 0.0;
                z[c] = (j < hi && lane < m) ? YsB[lane + (size_t)j * ldy] : 0.0;
            }
            for (int k = 0; k < mA8; ++k) {
                const double t = PaT[k * LT + lane];
#pragma unroll
                for (int c = 0; c < YS_COLS; ++c)
                    z[c] = fma(t, __shfl_sync(FULL, ya[c], k), z[c]);
            }
#pragma unroll
            for (int c = 0; c < YS_COLS; ++c)
                if (j0 + c < hi && lane < m) YsB[lane + (size_t)(j0 + c) * ldy] = z[c];
        }
    }
    if (s.cl.c > 1)
        cl_done(s);
    else
        __syncthreads();
}

/* The flush of one spin's site block after the proposals: the inverses Tu,
 * Tv from the recorded rows / columns, Zs and Ys (with the staged block's
 * corrections when mA > 0), and the G update when `flush`.  Rrow, Ccol,
 * facs: that spin's records; TuP: where Tu is laid out with even rows (the
 * spin's own Rrow area, free once the inverses exist).  Returns the staged
 * count left for the next block (0 after a G update). */
/* G -= Zs Ys as a split command of a cluster per chain (FP64). */
__device__ __noinline__ void g_update_cl(int n, int mt, double *G, const double *Zs,
                                         const double *Ys, int ldy, Smem &s)
{
    cl_post(s, CL_GUPD, G, Zs, Ys, nullptr, nullptr, nullptr, n, mt, ldy);
    gemm_nn_rmw_part(
        n, n, mt, Zs, n, Ys, ldy, [=](int i, int j) { return G[i + (size_t)j * n]; },
        [=](int i, int j, double v, double c) { G[i + (size_t)j * n] = c - v; }, s.gsm, s.cl);
    cl_done(s);
}

/* G -= Zs Ys (rank mt): FP64 tiles, or the split product in mixed mode. */
__device__ __forceinline__ void g_update(int n, int mt, double *G, const double *Zs,
                                         const double *Ys, int ldy, const DqmcChainDev *ch,
                                         Smem &s)
{
#if DQMC_MINB == 1
    if (s.spl) {
        flush_split(n, mt, G, Zs, Ys, ldy, ch, s);
        return;
    }
#endif
    (void)ch;
    if (s.cl.c > 1) {
        g_update_cl(n, mt, G, Zs, Ys, ldy, s);
        return;
    }
    gemm_nn_rmw(
        n, n, mt, Zs, n, Ys, ldy, [=](int i, int j) { return G[i + (size_t)j * n]; },
        [=](int i, int j, double v, double c) { G[i + (size_t)j * n] = c - v; }, s.gsm);
}

/* Ranks 1.. of a chain's cluster: form this rank's share of each command
 * rank 0 posts, until CL_EXIT.  The command block is read after the
 * barrier that publishes it and before the command's own barriers, so
 * rank 0 never rewrites it while it is being read. */
__device__ __noinline__ void cl_serve(Smem &s)
{
    __shared__ int sflag;   /* flags this rank raises in a command */
    for (;;) {
        cl_sync();
        const DqmcClCmd *c = s.cmd;
        const int op = c->op;
        if (op == CL_EXIT) break;
        const int i0 = c->i[0], i1 = c->i[1], i2 = c->i[2];
        const void *p0 = c->p[0], *p1 = c->p[1], *p2 = c->p[2], *p3 = c->p[3], *p4 = c->p[4],
                   *p5 = c->p[5];
        const double d0 = c->d[0], d1 = c->d[1], d2 = c->d[2], d3 = c->d[3];
        switch (op) {
        case CL_WRAP:
            wrap_green_cl(i0, (double *)p0, (double *)p1, (const double *)p2,
                          (const double *)p3, (const signed char *)p4, d0, d1, d2, d3, s);
            break;
        case CL_WRAP_BACK:
            wrap_green_back_cl(i0, (double *)p0, (double *)p1, (const double *)p2,
                               (const double *)p3, (const signed char *)p4, d0, d1, d2, d3, s);
            break;
        case CL_BBLOCK:
            bblock_cl(i0, i1, i2, (const signed char *)p0, (const double *)p1, d0, d1,
                      (double *)p2, (double *)p3, (double *)p4, s);
            break;
        case CL_GUPD:
            g_update_cl(i0, i1, (double *)p0, (const double *)p1, (const double *)p2, i2, s);
            break;
        case CL_QFORM:
            qr_form_q_sm(i0, (const double *)p0, (const double *)p1, (double *)p2, s);
            break;
        case CL_QT:
            qr_apply_qt_sm(i0, (const double *)p0, (const double *)p1, (double *)p2, i1, s);
            break;
        case CL_QRIGHT:
            qr_apply_right_sm(i0, (const double *)p0, (const double *)p1, (const double *)p2,
                              (double *)p3, s.vC, s);
            break;
        case CL_TRSM:
            trsm_upper(i0, (const double *)p0, (const double *)p1, (double *)p2, s);
            break;
        case CL_UGEMM:
            udv_gemm(i1, i0, (const double *)p0, (const double *)p1, (double *)p2, s);
            break;
        case CL_QRF:
            if (threadIdx.x == 0) sflag = 0;
            __syncthreads();
            qr_factor_cl(i0, (double *)p0, (double *)p1, s, &sflag);
            break;
        case CL_PREPIV:
            prepivot_cl(i0, (const double *)p0, (double *)p1, s, nullptr);
            break;
#if DQMC_MINB == 1
        case CL_WSPLIT:
            wrap_green_split(i0, (double *)p0, (double *)p1, *(const DqmcModelDev *)p2,
                             (const DqmcChainDev *)p3, (const signed char *)p4, d0, d1, d2, d3,
                             i1 != 0, s);
            break;
        case CL_FSPLIT:
            flush_split(i0, i1, (double *)p0, (const double *)p1, (const double *)p2, i2,
                        (const DqmcChainDev *)p3, s);
            break;
#endif
        case CL_ZY:
            flush_zy(i0, i1, i2 & 255, (i2 >> 8) & 255, (const double *)p0, (double *)p1,
                     (double *)p2, i2 >> 16, (const double *)p3, (const double *)p4,
                     (double *)p5, s);
            break;
        default:
            break;
        }
    }
}

__device__ __noinline__ int block_flush(int n, int kb, int i0, int m, double *G, double *Zs,
                                        double *Ys, int mA, bool flush, double *Rrow,
                                        double *Ccol, double *facs, double *TuP, Smem &s,
                                        DqmcChainDev *ch, PhaseClock &pc)
{
    constexpr int KB = DQMC_MAX_KB;
    constexpr int LD = KB + 1;
    constexpr int LT = KB + 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *Tu = s.g0 + 2 * KB * LD, *Tv = Tu + KB * LD;
    double *ZA = s.gsm, *YA = s.gsm + KB * LT, *TvP = s.gsm + 2 * KB * LT;
    const int *alist = s.iscr;
    const int ldy = 2 * kb;
    if (m == 0) {
        if (!flush || mA == 0) return mA;
        g_update(n, mA, G, Zs, Ys, ldy, ch, s);
        pc.charge(ch, DQMC_PH_FLUSH, 1);
        return 0;
    }
    /* Tu = (I - F Su)^-1 (warp 0), Tv = (I + Sc)^-1 (warp 1); lane q owns
     * row q.  Su[r][p] = V[i_p, r] = Rrow[r][a_p], Sc[r][p] = C[i_p, r] =
     * -fac_r Ccol[r][a_p], both for r < p.  Column p of row q is
     * delta_qp + sum_{r<p} (T[q][r] fac_r) S[r][a_p]; rolled loops over
     * shared memory keep the code small and the register count low. */
    if (warp < 2) {
        const double *Src = (warp == 0) ? Rrow : Ccol;
        double *T = (warp == 0) ? Tu : Tv;
        const int q = lane;
        for (int p = 0; p < m; ++p) {
            const double *sp = Src + alist[p];
            const double *tq = T + q * LD;
            /* four interleaved partial sums (r mod 4) to overlap the FP64
             * latency, combined in a fixed order */
            double x0 = (p == q) ? 1.0 : 0.0, x1 = 0.0, x2 = 0.0, x3 = 0.0;
            int r = 0;
            for (; r + 4 <= p; r += 4) {
                x0 = fma(tq[r] * facs[r], sp[r * LD], x0);
                x1 = fma(tq[r + 1] * facs[r + 1], sp[(r + 1) * LD], x1);
                x2 = fma(tq[r + 2] * facs[r + 2], sp[(r + 2) * LD], x2);
                x3 = fma(tq[r + 3] * facs[r + 3], sp[(r + 3) * LD], x3);
            }
            for (; r < p; ++r) x0 = fma(tq[r] * facs[r], sp[r * LD], x0);
            T[q * LD + p] = (x0 + x1) + (x2 + x3);
        }
    }
    __syncthreads();
    /* TuP, TvP: Tu, Tv with even rows, zero outside m x m.  With a staged
     * block: Qa[k][p] = sum_q YA[k][a_q] Tu[q][p] and -Pa^T[k][p] =
     * -sum_q ZA[a_q][k] Tv[q][p] (k < mA), kept in registers until every
     * thread has read ZA and YA. */
    constexpr int KR = KB * KB / NT;
    static_assert(KR * NT == KB * KB, "block split");
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const int e = tid + r * NT, q = e / KB, p = e % KB;
        const bool on = q < m && p < m;
        TuP[q * LT + p] = on ? Tu[q * LD + p] : 0.0;
        TvP[q * LT + p] = on ? Tv[q * LD + p] : 0.0;
    }
    if (mA > 0) {
        /* element r of this thread: staged index k = (tid + r NT) / KB
         * (uniform across a warp), column p = lane; the KR sums interleave */
        double qa[KR], pa[KR];
#pragma unroll
        for (int r = 0; r < KR; ++r) qa[r] = pa[r] = 0.0;
        if (lane < m) {
            for (int t = 0; t < m; ++t) {
                const int at = alist[t];
                const double tu = Tu[t * LD + lane], tv = Tv[t * LD + lane];
#pragma unroll
                for (int r = 0; r < KR; ++r) {
                    const int k = (tid + r * NT) / KB;
                    qa[r] = fma(YA[k * LD + at], tu, qa[r]);
                    pa[r] = fma(ZA[at * LD + k], tv, pa[r]);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int k = (tid + r * NT) / KB;
            const bool on = k < mA;
            YA[k * LT + lane] = on ? qa[r] : 0.0;
            ZA[k * LT + lane] = on ? -pa[r] : 0.0;
        }
    }
    __syncthreads();
    pc.charge(ch, DQMC_PH_FLUSH);
    flush_zy(n, i0, m, mA, G, Zs, Ys, ldy, TuP, facs, ch->clstage, s);
    const int mt = mA + m;
    if (!flush) {
        pc.charge(ch, DQMC_PH_FLUSH);
        return mt;
    }
    /* G -= Zs Ys, rank mA + m */
    g_update(n, mt, G, Zs, Ys, ldy, ch, s);
    pc.charge(ch, DQMC_PH_FLUSH, 1);
    return 0;
}

template <int NS>
__device__ __noinline__ int site_block(int n, int kb, int kbs, int i0, double *G,
                                       signed char *fl, const DqmcModelDev &md,
                                       uint64_t *rng, unsigned long long *att,
                                       unsigned long long *acc, double *Zs, double *Ys,
                                       int mA, bool flush, Smem &s, DqmcChainDev *ch,
                                       PhaseClock &pc, double *Gd = nullptr,
                                       double *Zsd = nullptr, double *Ysd = nullptr)
{
    constexpr int KB = DQMC_MAX_KB;   /* 32: one lane per block column */
    constexpr int LD = KB + 1;
    constexpr int LT = KB + 2;        /* even rows: 16-byte pair loads  */
    static_assert(GEMM_SMEM >= 3 * KB * LT && GEMM_SMEM % 2 == 0, "site-block staging");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *Rrow = s.g0;              /* [q*LD + b] = G~_q[a_q, b]      */
    double *Ccol = Rrow + KB * LD;    /* [q*LD + c] = G~_q[c, a_q]      */
    double *Tu = Ccol + KB * LD;      /* (I - F Su)^-1, row-major [q*LD+p] */
    double *Tv = Tu + KB * LD;        /* (I + Sc)^-1                     */
    double *facs = Tv + KB * LD;      /* fac_q                           */
    /* GEMM staging area, idle until the final flush: the staged block's
     * entries at this block ZA[a][k] = Zs_A[i0+a, k], YA[k][b] = Ys_A[k,
     * i0+b] (row length LD; block_flush reuses the area) */
    double *ZA = s.gsm, *YA = s.gsm + KB * LT;
    int *alist = s.iscr;              /* accepted block positions, in order */
    /* two-spin path: G_down's records in the GEMM staging area (pairing is
     * off there, and the down spin is flushed first) */
    double *RrowD = s.gsm, *CcolD = RrowD + KB * LD, *facsD = CcolD + KB * LD;
    const int ldy = 2 * kb;
    if (mA > 0) {
        for (int e = tid; e < KB * KB; e += NT) {
            const int a = e % KB, k = e / KB;
            if (k < mA) ZA[a * LD + k] = a < kbs ? Zs[(i0 + a) + (size_t)k * n] : 0.0;
            const int k2 = e % KB, b = e / KB;
            if (k2 < mA) YA[k2 * LD + b] = b < kbs ? Ys[k2 + (size_t)(i0 + b) * ldy] : 0.0;
        }
        __syncthreads();
        /* G~[B,B] = G[B,B] - ZA YA, row-major in the Tu area */
        for (int e = tid; e < KB * KB; e += NT) {
            const int c = e % KB, b = e / KB;
            if (c < kbs && b < kbs) {
                double v = G[(i0 + c) + (size_t)(i0 + b) * n];
                for (int k = 0; k < mA; ++k) v = fma(-ZA[c * LD + k], YA[k * LD + b], v);
                Tu[c * LD + b] = v;
            }
        }
        __syncthreads();
    }
    if (warp == 0) {
        double col[KB], cold[NS == 2 ? KB : 1];
        const bool mine = lane < kbs;
#pragma unroll
        for (int c = 0; c < KB; ++c)
            col[c] = (mine && c < kbs) ? (mA > 0 ? Tu[c * LD + lane]
                                                 : G[(i0 + c) + (size_t)(i0 + lane) * n])
                                       : 0.0;
        if constexpr (NS == 2) {
#pragma unroll
            for (int c = 0; c < KB; ++c)
                cold[c] = (mine && c < kbs) ? Gd[(i0 + c) + (size_t)(i0 + lane) * n] : 0.0;
        }
        int neg = 0;   /* accepted flips with R < 0 (dqmc.c:672-674) */
        int fvl = mine ? (int)fl[i0 + lane] : 1;
        const double Nu0 = md.Nup[0], Nu1 = md.Nup[1], Nd0 = md.Ndn[0], Nd1 = md.Ndn[1];
        uint64_t r4[4] = {0, 0, 0, 0};
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) r4[q] = rng[q];
        }
        unsigned long long nacc = 0;
        int m = 0;
#pragma unroll
        for (int a = 0; a < KB; ++a) {
            if (a < kbs) {
                const int sv = __shfl_sync(FULL, fvl, a);
                const double gii = __shfl_sync(FULL, col[a], a);
                const bool up = sv > 0;
                const double Nu = up ? Nu1 : Nu0, Nd = up ? Nd1 : Nd0;
                const double Ru = 1.0 + (1.0 - gii) * Nu;
                /* green_ph_down_ratio_N, or green_delay_ratio_N on G_down
                 * (green.c:402-416) */
                double giid = 0.0;
                if constexpr (NS == 2) giid = __shfl_sync(FULL, cold[a], a);
                const double Rd = NS == 2 ? 1.0 + (1.0 - giid) * Nd : 1.0 + gii * Nd;
                const double R = Ru * Rd;
                double u = 0.0;
                if (lane == 0) u = rng_next(r4);
                u = __shfl_sync(FULL, u, 0);
                if (u < fabs(R)) {
                    const double fac = Nu / Ru;
                    const double ra = col[a];        /* G~[a, lane] */
                    double mycol = 0.0;              /* G~[lane, a] */
                    const double fra = fac * ra;
#pragma unroll
                    for (int c = a + 1; c < KB; ++c) {
                        const double vc = __shfl_sync(FULL, col[c], a);
                        if (c == lane) mycol = vc;
                        col[c] = fma(vc, fra, col[c]);
                    }
                    Rrow[m * LD + lane] = ra;
                    Ccol[m * LD + lane] = mycol;
                    if constexpr (NS == 2) {
                        const double facd = Nd / Rd;
                        const double rad = cold[a];
                        double mycold = 0.0;
                        const double frad = facd * rad;
#pragma unroll
                        for (int c = a + 1; c < KB; ++c) {
                            const double vc = __shfl_sync(FULL, cold[c], a);
                            if (c == lane) mycold = vc;
                            cold[c] = fma(vc, frad, cold[c]);
                        }
                        RrowD[m * LD + lane] = rad;
                        CcolD[m * LD + lane] = mycold;
                        if (lane == 0) facsD[m] = facd;
                        if (R < 0.0) neg ^= 1;
                    }
                    if (lane == a) fvl = -sv;
                    if (lane == 0) {
                        facs[m] = fac;
                        alist[m] = a;
                        ++nacc;
                    }
                    ++m;
                }
            }
        }
        if (mine) fl[i0 + lane] = (signed char)fvl;
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) rng[q] = r4[q];
            *att += (unsigned long long)kbs;
            *acc += nacc;
            ch->pcalls[DQMC_PH_PROPOSE] += NS * nacc;   /* green_delay_accept calls */
            s.iscr[2 * DQMC_MAX_KB] = m;
            if (neg) ch->sign = -ch->sign;
        }
    }
    __syncthreads();
    pc.charge(ch, DQMC_PH_PROPOSE);
    const int m = s.iscr[2 * DQMC_MAX_KB];
    if constexpr (NS == 2) {
        if (m > 0)
            block_flush(n, kb, i0, m, Gd, Zsd, Ysd, 0, true, RrowD, CcolD, facsD, RrowD, s, ch,
                        pc);
    }
    return block_flush(n, kb, i0, m, G, Zs, Ys, mA, flush, Rrow, Ccol, facs, Rrow, s, ch, pc);
}

/* max|G - Gn| and G <- Gn */
__device__ double adopt_green(int n, double *G, const double *Gn, Smem &s)
{
    double mx = 0.0, bad = 0.0;
    for (int e0 = threadIdx.x; e0 < n * n; e0 += NT * 8) {
        double a[8], b[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * NT;
            a[u] = e < n * n ? G[e] : 0.0;
            b[u] = e < n * n ? Gn[e] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * NT;
            if (e < n * n) {
                const double d = fabs(a[u] - b[u]);
                if (d <= 1.7976931348623157e308)
                    mx = fmax(mx, d);
                else
                    bad += 1.0;             /* NaN or inf: counted, not maxed */
                G[e] = b[u];
            }
        }
    }
    mx = block_reduce<true>(mx, s.red);
    bad = block_reduce<false>(bad, s.red);
    return bad != 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : mx;
}

__device__ double max_diff(int n, const double *A, const double *B, Smem &s)
{
    double mx = 0.0;
    for (int e = threadIdx.x; e < n * n; e += NT) mx = fmax(mx, fabs(A[e] - B[e]));
    return block_reduce<true>(mx, s.red);
}

/* G(l0) from scratch: L single-slice lmuls then (1+UDT)^{-1} (green.c:262).
 * Uses the chain's scr UDV slot; returns det sign (0 on failure). */
__device__ __noinline__ int green_scratch(DqmcChainDev *ch, const DqmcModelDev &md, int l0, double *Gout,
                             double *slot, Smem &s, int *flag, int spin = 0)
{
    const int n = ch->n, L = ch->L;
    const double *v = spin ? md.expvd : md.expv;
    Udv u = udv_at(slot, n);
    udv_identity(u, n);
    for (int k = 0; k < L; ++k) {
        const int l = (l0 + k) % L;
        udv_lmul(n, u, nullptr, md.expK, ch->field + (size_t)l * n, v[0], v[1],
                 chain_scr(ch), s, flag);
        if (*flag) return 0;
    }
    const int ds = udv_green(n, u, Gout, chain_scr(ch), s, flag);
    return *flag ? 0 : ds;
}

/* Statistics of log|D| of one UDV factor (udv_scale_stats, dqmc.c:108-142,
 * on the log-scale D held here: ell = -inf is a zero entry, +inf or NaN a
 * non-finite one): o = {min, max over finite entries (NaN if none),
 * finite, zero, non-finite counts}, valid in thread 0.  All threads call. */
__device__ void ell_stats(int n, const double *ell, double *o, Smem &s)
{
    static_assert(5 * NW <= 40, "reduction slots");
    double mn = INFINITY, mx = -INFINITY, fin = 0.0, zero = 0.0, bad = 0.0;
    for (int e = threadIdx.x; e < n; e += NT) {
        const double x = ell[e];
        if (x == -INFINITY) {
            zero += 1.0;
        } else if (isfinite(x)) {
            fin += 1.0;
            mn = fmin(mn, x);
            mx = fmax(mx, x);
        } else {
            bad += 1.0;
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(FULL, mn, d));
        mx = fmax(mx, __shfl_xor_sync(FULL, mx, d));
        fin += __shfl_xor_sync(FULL, fin, d);
        zero += __shfl_xor_sync(FULL, zero, d);
        bad += __shfl_xor_sync(FULL, bad, d);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        double *r = s.red + 5 * warp;
        r[0] = mn;
        r[1] = mx;
        r[2] = fin;
        r[3] = zero;
        r[4] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NW; ++w) {
            const double *r = s.red + 5 * w;
            mn = fmin(mn, r[0]);
            mx = fmax(mx, r[1]);
            fin += r[2];
            zero += r[3];
            bad += r[4];
        }
        o[0] = fin > 0.0 ? mn : NAN;
        o[1] = fin > 0.0 ? mx : NAN;
        o[2] = fin;
        o[3] = zero;
        o[4] = bad;
    }
    __syncthreads();
}

/* One UDV scale record (dqmc_record_udv_scale_diag / _single_, dqmc.c:
 * 196-230) of the factor L (and R for a boundary pair) into the chain's
 * record buffer; a no-op unless the engine enabled the records. */
__device__ __noinline__ void udv_record(DqmcChainDev *ch, int kind, int tau, int boundary, int n,
                                        const double *ellL, const double *ellR, Smem &s,
                                        int spin = 0)
{
    if (!ch->udvrec) return;
    double a[5], b[5] = {NAN, NAN, 0.0, 0.0, 0.0};
    ell_stats(n, ellL, a, s);
    if (ellR) ell_stats(n, ellR, b, s);
    if (threadIdx.x == 0) {
        if (ch->udv_n < ch->udv_cap) {
            double *r = ch->udvrec + (size_t)ch->udv_n * DQMC_UDV_RECORD_DOUBLES;
            r[DQMC_UDV_R_KIND] = kind;
            r[DQMC_UDV_R_TAU] = tau;
            r[DQMC_UDV_R_BOUNDARY] = boundary;
            r[DQMC_UDV_R_SWEEP] = (double)ch->sweeps;
            for (int k = 0; k < 5; ++k) {
                r[DQMC_UDV_R_LEFT + k] = a[k];
                r[DQMC_UDV_R_RIGHT + k] = b[k];
            }
            r[DQMC_UDV_R_HAS_RIGHT] = ellR ? 1.0 : 0.0;
            r[DQMC_UDV_R_SPIN] = spin;
            ch->udv_n++;
        } else {
            ch->udv_lost++;
        }
    }
}

/* Snapshot of G as wrapped, just before a stabilization point replaces it
 * (opt-in diagnostic: max|G_mixed - G_FP64| between engines run in lock
 * step, and the wrapped G the reference's drift diagnostic compares,
 * dqmc.c:64-98). */
__device__ __noinline__ void glog_take(DqmcChainDev *ch, const double *G, int n)
{
    if (!ch->glog) return;
    const int k = ch->glog_n;
    if (k < ch->glog_cap) {
        double *dst = ch->glog + (size_t)k * n * n;
        ew_batched(n * n, [=](int e) { return G[e]; }, [=](int e, double x) { dst[e] = x; });
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (k < ch->glog_cap) ch->glog_n = k + 1;
        else ch->glog_lost++;
    }
    __syncthreads();
}

/* The forward sweep, dqmc_sweep_forward (dqmc.c:609-813) with
 * carry_prefix = 0, use_ph = 1 and the combine rebuild.  Returns false on a
 * numerical failure (flag holds the reason). */
/* One evolved spin's state: G_up (sigma = +1) or, on the two-spin path,
 * G_down (sigma = -1) with its own B factors (green_alloc, green.c:54-86). */
struct Spin {
    double *G, *S, *left, *comb, *bcache;
    double v0, v1, vi0, vi1;
};

__device__ __forceinline__ Spin spin_of(DqmcChainDev *ch, const DqmcModelDev &md, int q)
{
    if (q == 0)
        return Spin{ch->G, ch->S, ch->left, ch->comb, ch->bcache, md.expv[0], md.expv[1],
                    md.expvinv[0], md.expvinv[1]};
    return Spin{ch->Gd, ch->Sd, ch->leftd, ch->combd, ch->bcached, md.expvd[0], md.expvd[1],
                md.expvinvd[0], md.expvinvd[1]};
}

__device__ __noinline__ bool sweep_body(DqmcChainDev *ch, const DqmcModelDev &md, int kflags, Smem &s,
                           int *flag, uint64_t *rng, unsigned long long *att,
                           unsigned long long *acc, double *slot_scr)
{
    const int n = ch->n, L = ch->L, stab = ch->stab, M = ch->M, kb = ch->kb;
    const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
    const Scr w = chain_scr(ch);
    double *Gn = ch->w[3], *tmp = ch->w[4], *tmp2 = ch->w[5];
    const int ns = ch->ns;   /* 1: PH path; 2: G_up and G_down (dqmc.c:641-683) */
    auto Pj = [&](int j) { return udv_at(ch->P + (size_t)j * usz, n); };
    const bool alt = ch->alt != 0;
    PhaseClock pc;
    pc.mark();

    /* alternating order with a suffix stack carried from the backward sweep
     * before (dqmc.c:622-629): no stack build */
    if (!(alt && ch->svalid)) {
        for (int q = 0; q < ns; ++q) {   /* G_up's stack, then G_down's (dqmc.c:630-646) */
            const Spin sp = spin_of(ch, md, q);
            auto Sj = [&](int j) { return udv_at(sp.S + (size_t)j * usz, n); };
            /* Block products B(b_{j+1}, b_j) of the current field.  After the
             * first sweep they are the ones the previous sweep computed. */
            if (!ch->bvalid) {
                for (int j = 1; j < M; ++j) {
                    const int b0 = j * stab, b1 = min((j + 1) * stab, L);
                    bblock(n, b0, b1 - b0, ch->field, md.expK, sp.v0, sp.v1,
                           sp.bcache + j * nn, tmp, tmp2, s);
                }
            }
            pc.charge(ch, DQMC_PH_BCACHE, 1);
            /* suffix stack (green_stack_build_suffix, green.c:203-226) */
            udv_identity(Sj(M), n);
            for (int j = M - 1; j >= 1; --j) {
                udv_copy(Sj(j), Sj(j + 1), n);
                udv_record(ch, DQMC_UDV_STACK_SUFFIX_PRE_RMUL, min(j * stab, L), j, n, Sj(j).ell,
                           nullptr, s, q);
                if (threadIdx.x == 0) ch->pcalls[DQMC_PH_STACK]++;   /* udv_rmul calls */
                udv_rmul(n, Sj(j), sp.bcache + j * nn, w, s, flag);
                if (*flag) return false;
            }
        }
    }
    for (int q = 0; q < ns; ++q) udv_identity(udv_at(spin_of(ch, md, q).left, n), n);
    if (alt) udv_copy(Pj(0), udv_at(ch->left, n), n);   /* prefix stack (dqmc.c:648-650) */
    pc.charge(ch, DQMC_PH_STACK);
    int tau_left = 0;
    for (int l = 0; l < L; ++l) {
        signed char *fl = ch->field + (size_t)l * n;
        if (ns == 2) {
            for (int i0 = 0; i0 < n; i0 += kb)
                site_block<2>(n, kb, min(kb, n - i0), i0, ch->G, fl, md, rng, att, acc, ch->Zs,
                              ch->Ys, 0, true, s, ch, pc, ch->Gd, ch->Zsd, ch->Ysd);
        } else {
            for (int i0 = 0, mA = 0; i0 < n; i0 += kb)
                mA = site_block<1>(n, kb, min(kb, n - i0), i0, ch->G, fl, md, rng, att, acc,
                                   ch->Zs, ch->Ys, mA, !ch->pair || mA > 0 || i0 + kb >= n, s,
                                   ch, pc);
        }
        for (int q = 0; q < ns; ++q) {
            const Spin sp = spin_of(ch, md, q);
#if DQMC_MINB == 1
            if (s.spl)
                wrap_green_split(n, sp.G, tmp, md, ch, fl, sp.v0, sp.v1, sp.vi0, sp.vi1, false,
                                 s);
            else
#endif
                wrap_green(n, sp.G, tmp, md.expK, md.expKinv, fl, sp.v0, sp.v1, sp.vi0, sp.vi1,
                           s);
            pc.charge(ch, DQMC_PH_WRAP, 1);
        }
        const bool boundary = ((l + 1) % stab == 0) && (l + 1 < L);
        const bool last = (l + 1 == L);
        if (!boundary && !last) continue;
        const int tau = boundary ? l + 1 : 0;
        if (kflags & KF_SDRIFT) {
            /* dqmc_record_stab_drift (dqmc.c:64-98): both spins, the larger */
            double d = 0.0;
            for (int q = 0; q < ns; ++q) {
                const int ds = green_scratch(ch, md, tau, Gn, slot_scr, s, flag, q);
                if (*flag || ds == 0) return false;
                d = fmax(d, max_diff(n, spin_of(ch, md, q).G, Gn, s));
                pc.charge(ch, DQMC_PH_SDRIFT, 1);
            }
            if (threadIdx.x == 0) {
                ch->sdrift_count++;
                ch->sdrift_sum += d;
                if (d > ch->sdrift_max || ch->sdrift_count == 1) {
                    ch->sdrift_max = d;
                    ch->sdrift_max_tau = tau;
                    ch->sdrift_max_sweep = ch->sweeps;
                }
            }
        }
        const int te = boundary ? l + 1 : L;
        const int jblk = (boundary ? (l + 1) / stab : M) - 1;
        for (int q = 0; q < ns; ++q) {
            const Spin sp = spin_of(ch, md, q);
            if (te > tau_left) {
                bblock(n, tau_left, te - tau_left, ch->field, md.expK, sp.v0, sp.v1,
                       sp.bcache + jblk * nn, tmp, tmp2, s);
                pc.charge(ch, DQMC_PH_BBLOCK, 1);
                udv_lmul(n, udv_at(sp.left, n), sp.bcache + jblk * nn, nullptr, nullptr, 0.0, 0.0,
                         w, s, flag);
                if (*flag) return false;
                pc.charge(ch, DQMC_PH_LMUL, 1);
            }
        }
        tau_left = te;
        if (alt)   /* dqmc.c:704-706,767 */
            udv_copy(Pj(boundary ? (l + 1) / stab : M), udv_at(ch->left, n), n);
        for (int q = 0; q < ns; ++q) {   /* dqmc.c:707-724, 772-789 */
            const Spin sp = spin_of(ch, md, q);
            if (boundary)
                udv_record(ch, DQMC_UDV_FORWARD, l + 1, (l + 1) / stab, n, udv_at(sp.left, n).ell,
                           udv_at(sp.S + (size_t)((l + 1) / stab) * usz, n).ell, s, q);
            else
                udv_record(ch, DQMC_UDV_LEFT_FORWARD, L, M, n, udv_at(sp.left, n).ell, nullptr, s,
                           q);
        }
        double d = 0.0;
        int sgn = 1;
        for (int q = 0; q < ns; ++q) {   /* green_from_stack / _left_udv per spin */
            const Spin sp = spin_of(ch, md, q);
            Udv left = udv_at(sp.left, n), comb = udv_at(sp.comb, n);
            Udv Sb = udv_at(sp.S + (size_t)((l + 1) / stab) * usz, n);
            int ds;
            if (boundary && ch->rebuild) {
                ds = udv_green2(n, left, Sb, Gn, tmp2, w, s, flag);
            } else if (boundary) {
                udv_combine(n, left, Sb, comb, w, s, flag);
                if (*flag) return false;
                pc.charge(ch, DQMC_PH_COMBINE, 1);
                ds = udv_green(n, comb, Gn, w, s, flag);
            } else {
                ds = udv_green(n, left, Gn, w, s, flag);
            }
            pc.charge(ch, DQMC_PH_GREEN, 1);
            if (ds == 0) raise_flag(flag, DQMC_ST_DETSIGN);
            __syncthreads();
            if (*flag) return false;
            sgn *= ds;
            if (q == 0) glog_take(ch, sp.G, n);
            const double dq = adopt_green(n, sp.G, Gn, s);
            /* a wrapped G that is not finite means the chain's state was lost
             * since the last rebuild: stop the chain (sticky status) */
            if (!(dq == dq) || isinf(dq)) {
                raise_flag(flag, DQMC_ST_NONFINITE);
                return false;
            }
            d = fmax(d, dq);
            pc.charge(ch, DQMC_PH_ADOPT, 1);
        }
        if (threadIdx.x == 0) {
            ch->drift_count++;
            ch->drift_sum += d;
            if (d > ch->drift_max || ch->drift_count == 1) ch->drift_max = d;
            /* the running sign reset to the stabilized exact value
             * (dqmc.c:740-745): 1 on the PH path, det_up * det_down else */
            ch->sign = ns == 2 ? (double)sgn : 1.0;
        }
    }
    return true;
}

/* Backward sweep of the alternating order, dqmc_sweep_backward
 * (dqmc.c:815-950): slices L-1 .. 0 with B^-1 G B wraps (green.c:529-548);
 * the suffix product is accumulated by rmul and stored as the next forward
 * sweep's suffix stack; at a boundary G comes from the forward sweep's
 * prefix and this suffix (green_from_boundary_factors, green.c:308-341). */
__device__ __noinline__ bool sweep_body_back(DqmcChainDev *ch, const DqmcModelDev &md, int kflags,
                                             Smem &s, int *flag, uint64_t *rng,
                                             unsigned long long *att, unsigned long long *acc,
                                             double *slot_scr)
{
    const int n = ch->n, L = ch->L, stab = ch->stab, M = ch->M, kb = ch->kb;
    const size_t nn = (size_t)n * n, usz = DQMC_UDV_SIZE(n);
    const Scr w = chain_scr(ch);
    double *G = ch->G, *Gn = ch->w[3], *tmp = ch->w[4], *tmp2 = ch->w[5];
    const double v0 = md.expv[0], v1 = md.expv[1];
    auto Sj = [&](int j) { return udv_at(ch->S + (size_t)j * usz, n); };
    auto Pj = [&](int j) { return udv_at(ch->P + (size_t)j * usz, n); };
    Udv left = udv_at(ch->left, n), comb = udv_at(ch->comb, n);
    PhaseClock pc;
    pc.mark();
    if (!ch->pvalid) {
        if (threadIdx.x == 0) ch->pcalls[DQMC_PH_BCACHE]++;
        /* green_stack_build_prefix (green.c:228-250) */
        udv_identity(Pj(0), n);
        for (int j = 1; j <= M; ++j) {
            const int b0 = (j - 1) * stab, b1 = min(j * stab, L);
            bblock(n, b0, b1 - b0, ch->field, md.expK, v0, v1, ch->bcache + (j - 1) * nn, tmp,
                   tmp2, s);
            udv_copy(Pj(j), Pj(j - 1), n);
            udv_record(ch, DQMC_UDV_STACK_PREFIX_PRE_LMUL, b1, j, n, Pj(j).ell, nullptr, s);
            udv_lmul(n, Pj(j), ch->bcache + (j - 1) * nn, nullptr, nullptr, 0.0, 0.0, w, s,
                     flag);
            if (*flag) return false;
        }
    }
    udv_identity(left, n);
    udv_identity(Sj(M), n);
    pc.charge(ch, DQMC_PH_STACK);
    auto back_wrap = [&](int l) {
#if DQMC_MINB == 1
        if (s.spl)
            wrap_green_split(n, G, tmp, md, ch, ch->field + (size_t)l * n, v0, v1,
                             md.expvinv[0], md.expvinv[1], true, s);
        else
#endif
            wrap_green_back(n, G, tmp, md.expK, md.expKinv, ch->field + (size_t)l * n, v0, v1,
                            md.expvinv[0], md.expvinv[1], s);
        pc.charge(ch, DQMC_PH_WRAP, 1);
    };
    auto rebuild = [&](int tau, Udv u, bool boundary, int j) {
        if (kflags & KF_SDRIFT) {
            const int ds = green_scratch(ch, md, tau, Gn, slot_scr, s, flag);
            if (*flag || ds == 0) return false;
            const double d = max_diff(n, G, Gn, s);
            if (threadIdx.x == 0) {
                ch->sdrift_count++;
                ch->sdrift_sum += d;
                if (d > ch->sdrift_max || ch->sdrift_count == 1) {
                    ch->sdrift_max = d;
                    ch->sdrift_max_tau = tau;
                    ch->sdrift_max_sweep = ch->sweeps;
                }
            }
            pc.charge(ch, DQMC_PH_SDRIFT, 1);
        }
        const int b1 = min(tau + stab, L);
        bblock(n, tau, b1 - tau, ch->field, md.expK, v0, v1, ch->bcache + j * nn, tmp, tmp2, s);
        pc.charge(ch, DQMC_PH_BBLOCK, 1);
        udv_rmul(n, u, ch->bcache + j * nn, w, s, flag);
        if (*flag) return false;
        pc.charge(ch, DQMC_PH_LMUL, 1);
        int ds;
        if (boundary) {
            udv_copy(Sj(j), u, n);
            udv_record(ch, DQMC_UDV_BACKWARD, tau, j, n, Pj(j).ell, u.ell, s);   /* dqmc.c:831 */
            if (ch->rebuild) {
                ds = udv_green2(n, Pj(j), u, Gn, tmp2, w, s, flag);
            } else {
                udv_combine(n, Pj(j), u, comb, w, s, flag);
                if (*flag) return false;
                pc.charge(ch, DQMC_PH_COMBINE, 1);
                ds = udv_green(n, comb, Gn, w, s, flag);
            }
        } else {
            udv_record(ch, DQMC_UDV_LEFT_BACKWARD, 0, 0, n, u.ell, nullptr, s);   /* dqmc.c:926 */
            ds = udv_green(n, u, Gn, w, s, flag);
        }
        pc.charge(ch, DQMC_PH_GREEN, 1);
        if (ds == 0) raise_flag(flag, DQMC_ST_DETSIGN);
        __syncthreads();
        if (*flag) return false;
        glog_take(ch, G, n);
        const double d = adopt_green(n, G, Gn, s);
        /* a wrapped G that is not finite means the chain's state was lost
         * since the last rebuild: stop the chain (sticky status) */
        if (!(d == d) || isinf(d)) {
            raise_flag(flag, DQMC_ST_NONFINITE);
            return false;
        }
        if (threadIdx.x == 0) {
            ch->drift_count++;
            ch->drift_sum += d;
            if (d > ch->drift_max || ch->drift_count == 1) ch->drift_max = d;
            ch->sign = 1.0;
        }
        pc.charge(ch, DQMC_PH_ADOPT, 1);
        return true;
    };
    back_wrap(L - 1);
    for (int l = L - 1; l >= 0; --l) {
        signed char *fl = ch->field + (size_t)l * n;
        for (int i0 = 0, mA = 0; i0 < n; i0 += kb)
            mA = site_block<1>(n, kb, min(kb, n - i0), i0, G, fl, md, rng, att, acc, ch->Zs,
                               ch->Ys, mA, !ch->pair || mA > 0 || i0 + kb >= n, s, ch, pc);
        if (l == 0) break;
        if (l % stab == 0 && !rebuild(l, left, true, l / stab)) return false;
        back_wrap(l - 1);
    }
    return rebuild(0, left, false, 0);
}

/* One CTA per chain, or thread-block clusters: cluster b < ncoop advances
 * chain order[b] with all its CTAs (cl_serve); each later cluster runs cc
 * chains, one per CTA, order[ncoop + (b - ncoop) cc + rank] (CTAs past
 * nchains return).  order lists the chains most expensive first, so a batch
 * of uneven chains gives its longest chains the clusters and does not end
 * on a late-starting long one. */
__global__ void __launch_bounds__(NT, DQMC_MINB)
    k_sweep(DqmcChainDev *chains, const DqmcModelDev *models, int kflags, int nsweeps,
            const int *order, int ncoop, int nchains)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    __shared__ uint64_t rng[4];
    __shared__ unsigned long long att, acc;
    /* a launch without clusters is a launch of one-CTA clusters */
    const int csz = max(1, (int)cl_size_hw()), crk = csz > 1 ? (int)cl_rank_hw() : 0;
    const int slot = (int)(blockIdx.x / (unsigned)csz);
    const bool coop = slot < ncoop;
    const int cidx = coop ? slot : ncoop + (slot - ncoop) * csz + crk;
    if (cidx >= nchains) return;
    const int cc = coop ? csz : 1, cr = coop ? crk : 0;
    DqmcChainDev *ch = &chains[order ? order[cidx] : cidx];
    const DqmcModelDev &md = models[ch->model];
    Smem s = carve(smraw, ch->n, ch->kb);
    s.cl = Part{cr, cc};
    s.cmd = &ch->cl;
    s.stage = ch->clstage;
#if DQMC_MINB == 1
    __shared__ SplCtx spl;
#endif
    if (cr > 0) {
#if DQMC_MINB == 1
        if (kflags & KF_MIXED) {   /* this rank's own tensor memory */
            spl_setup(&spl);
            s.spl = &spl;
        }
#endif
        cl_serve(s);
#if DQMC_MINB == 1
        if (s.spl) spl_teardown(&spl);
#endif
        return;
    }
    if (threadIdx.x == 0) {
        flag = ch->status;
        ch->cl.err = 0;
    }
    __syncthreads();
    if (!flag) {
#if DQMC_MINB == 1
        if (kflags & KF_MIXED) {
            spl_setup(&spl);
            s.spl = &spl;
        }
#endif
        for (int sw = 0; sw < nsweeps; ++sw) {
            if (threadIdx.x == 0) {
                for (int i = 0; i < 4; ++i) rng[i] = ch->rng[i];
                att = 0;
                acc = 0;
                ch->meas_accepted = ch->accepted;
                ch->meas_attempts = ch->attempts;
            }
            __syncthreads();
            const bool back = ch->alt && ch->dir;
            bool ok = back ? sweep_body_back(ch, md, kflags, s, &flag, rng, &att, &acc, ch->scr)
                           : sweep_body(ch, md, kflags, s, &flag, rng, &att, &acc, ch->scr);
            __syncthreads();
#if DQMC_MINB == 1
            if (s.spl && spl.err) {   /* a split product was abandoned */
                ok = false;
                if (threadIdx.x == 0) flag |= DQMC_ST_TIMEOUT;
                __syncthreads();
            }
#endif
            if (threadIdx.x == 0) {
                for (int i = 0; i < 4; ++i) ch->rng[i] = rng[i];
                ch->attempts += att;
                ch->accepted += acc;
                if (ok && !flag) {
                    ch->sweeps++;
                    ch->bvalid = 1;
                    if (ch->alt) {   /* dqmc.c:806-810, 943-946 */
                        ch->dir = back ? 0 : 1;
                        ch->pvalid = back ? 0 : 1;
                        ch->svalid = back ? 1 : 0;
                    }
                } else {
                    ch->status = flag ? flag : DQMC_ST_NONFINITE;
                    ch->sign = 0.0;
                    ch->bvalid = 0;
                    ch->pvalid = 0;
                    ch->svalid = 0;
                }
            }
            __syncthreads();
            if (!ok || flag) break;
        }
#if DQMC_MINB == 1
        if (s.spl) spl_teardown(&spl);
#endif
    }
    /* the one exit of rank 0: release the other ranks */
    if (cc > 1) {
        if (threadIdx.x == 0) ch->cl.op = CL_EXIT;
        cl_sync();
    }
}

/* G from scratch at l0 = 0 for every chain (dqmc_init_modes, dqmc.c:466-483). */
/* G at slice 0 for a new or rewritten field: the UDV of B_{L-1} ... B_0
 * accumulated from the stabilization blocks B(b_{j+1}, b_j) (stab slices
 * per QR-based lmul, as the sweep's stack is) instead of one lmul per slice
 * (green_from_scratch, green.c:262-306, which the reference-definition
 * drift diagnostic keeps using): the same product, M instead of L
 * factorizations. */
__device__ __noinline__ int green_init(DqmcChainDev *ch, const DqmcModelDev &md, double *Gout,
                                       double *slot, Smem &s, int *flag, int spin)
{
    const int n = ch->n, L = ch->L, stab = ch->stab, M = ch->M;
    const double *v = spin ? md.expvd : md.expv;
    Udv u = udv_at(slot, n);
    udv_identity(u, n);
    for (int j = 0; j < M; ++j) {
        const int b0 = j * stab, len = min(stab, L - b0);
        bblock(n, b0, len, ch->field, md.expK, v[0], v[1], ch->w[3], ch->w[4], ch->w[5], s);
        udv_lmul(n, u, ch->w[3], nullptr, nullptr, 0.0, 0.0, chain_scr(ch), s, flag);
        if (*flag) return 0;
    }
    const int ds = udv_green(n, u, Gout, chain_scr(ch), s, flag);
    return *flag ? 0 : ds;
}

__global__ void __launch_bounds__(NT, DQMC_MINB) k_init(DqmcChainDev *chains, const DqmcModelDev *models)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    DqmcChainDev *ch = &chains[blockIdx.x];
    const DqmcModelDev &md = models[ch->model];
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    Smem s = carve(smraw, ch->n, ch->kb);
    int ds = green_init(ch, md, ch->G, ch->scr, s, &flag, 0);
    /* the two-spin path starts with the sign det_up * det_down
     * (dqmc.c:467-481) */
    if (ch->ns == 2 && !flag) ds *= green_init(ch, md, ch->Gd, ch->scr, s, &flag, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        ch->status = flag ? flag : (ds == 0 ? DQMC_ST_DETSIGN : 0);
        ch->sign = ch->status ? 0.0 : (ch->ns == 2 ? (double)ds : 1.0);
        ch->bvalid = 0;
        ch->dir = 0;
        ch->pvalid = 0;
        ch->svalid = 0;
    }
}

/* Test kernels: rebuild from scratch into out; wrap a caller G. */
__global__ void __launch_bounds__(NT, DQMC_MINB)
    k_scratch(DqmcChainDev *chains, const DqmcModelDev *models, int c, int l0, double *out,
              int *det)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    DqmcChainDev *ch = &chains[c];
    const DqmcModelDev &md = models[ch->model];
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    Smem s = carve(smraw, ch->n, ch->kb);
    const int ds = green_scratch(ch, md, l0, out, ch->scr, s, &flag);
    if (threadIdx.x == 0) *det = flag ? 0 : ds;
}

__global__ void __launch_bounds__(NT, DQMC_MINB)
    k_wrap(DqmcChainDev *chains, const DqmcModelDev *models, int c, int l, double *Gio,
           int kflags)
{
    extern __shared__ __align__(16) double smraw[];
    DqmcChainDev *ch = &chains[c];
    const DqmcModelDev &md = models[ch->model];
    Smem s = carve(smraw, ch->n, ch->kb);
    const int n = ch->n;
#if DQMC_MINB == 1
    if (kflags & KF_MIXED) {
        __shared__ SplCtx spl;
        spl_setup(&spl);
        s.spl = &spl;
        wrap_green_split(n, Gio, ch->w[4], md, ch, ch->field + (size_t)l * n, md.expv[0],
                         md.expv[1], md.expvinv[0], md.expvinv[1], false, s);
        spl_teardown(&spl);
        return;
    }
#endif
    (void)kflags;
    wrap_green(n, Gio, ch->w[4], md.expK, md.expKinv, ch->field + (size_t)l * n, md.expv[0],
               md.expv[1], md.expvinv[0], md.expvinv[1], s);
}

/* Caller UDV -> G (fixture parity).  ws: 4 n*n scratch + tw + UDV slot. */
__global__ void __launch_bounds__(NT, DQMC_MINB)
    k_udv_green(int n, double *slot, double *ws, double *G, int *det)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    Smem s = carve(smraw, n, 1);
    const size_t nn = (size_t)n * n;
    Scr w{ws, ws + nn, ws + 2 * nn, ws + 3 * nn};
    const int ds = udv_green(n, udv_at(slot, n), G, w, s, &flag);
    if (threadIdx.x == 0) *det = flag ? 0 : ds;
}

/* Two caller UDV slots -> G by the two-sided reconstruction (fixture
 * parity).  ws: 4 n*n scratch + tw. */
__global__ void __launch_bounds__(NT, DQMC_MINB)
    k_udv_green2(int n, double *lslot, double *rslot, double *ws, double *G, int *det)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ int flag;
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    Smem s = carve(smraw, n, 1);
    const size_t nn = (size_t)n * n;
    Scr w{ws, ws + nn, ws + 2 * nn, ws + 4 * nn};
    const int ds = udv_green2(n, udv_at(lslot, n), udv_at(rslot, n), G, ws + 3 * nn, w, s, &flag);
    if (threadIdx.x == 0) *det = flag ? 0 : ds;
}

/* Equal-time measurements on G_up at slice 0, fused: one read of G gives
 * measure_sample (measure.c:6-39) with G_down = I - P G_up^T P, the spin
 * correlations by displacement (structure_factor.c:258-297, 328-392) and the
 * cosine transforms (finish_fourier, structure_factor.c:311-326); the
 * sample is added to bin `bin` (replica_bin_add, replica.c:48-71;
 * q_add, replica.c:219-226).  Per displacement the i order matches the
 * reference's loop, so the sums are formed in the same order. */
__global__ void __launch_bounds__(NT)
    k_measure(DqmcChainDev *chains, const DqmcModelDev *models, int bin)
{
    extern __shared__ __align__(16) double smraw[];
    __shared__ double red[40];
    DqmcChainDev *ch = &chains[blockIdx.x];
    if (ch->status) return;
    PhaseClock pc;
    pc.mark();
    const DqmcModelDev &md = models[ch->model];
    const int n = ch->n;
    const double *G = ch->G;
    const double *t = md.thop;
    const int *p = md.bipart;
    /* G_down: the PH map of G_up (dqmc_map_ph_down, dqmc.c:9-17), or the
     * evolved G_down of the two-spin path */
    const double *Gd = ch->Gd;
    const bool two = ch->ns == 2;
    double ek = 0.0, ei = 0.0, nt = 0.0, bad = 0.0;
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e % n, j = e / n;
        const double dij = (i == j) ? 1.0 : 0.0;
        const double gu_ji = G[j + (size_t)i * n];
        const double gd_ji = two ? Gd[j + (size_t)i * n]
                                 : dij - (double)(p[j] * p[i]) * G[i + (size_t)j * n];
        const double tij = t[i + (size_t)j * n];
        ek += tij * (dij - gu_ji);
        ek += tij * (dij - gd_ji);
        bad += isfinite(gu_ji) && isfinite(gd_ji) ? 0.0 : 1.0;
    }
    for (int i = threadIdx.x; i < n; i += NT) {
        const double gu = G[i + (size_t)i * n];
        const double gd = two ? Gd[i + (size_t)i * n] : 1.0 - (double)(p[i] * p[i]) * gu;
        const double nu = 1.0 - gu, nd = 1.0 - gd;
        ei += nu * nd;
        nt += nu + nd;
    }
    ek = block_reduce<false>(ek, red);
    ei = block_reduce<false>(ei, red);
    nt = block_reduce<false>(nt, red);
    bad = block_reduce<false>(bad, red);
    if (bad != 0.0) {
        if (threadIdx.x == 0) ch->status |= DQMC_ST_NONFINITE;
        return;
    }
    double *cz = smraw, *cp = smraw + n;
    const int Lx = md.Lx > 0 ? md.Lx : n, Ly = md.Ly > 0 ? md.Ly : 1;
    const bool spin = (md.nq_zz > 0 || md.nq_perp > 0);
    if (spin) {
        for (int d = threadIdx.x; d < n; d += NT) {
            const int dx = d % Lx, dy = d / Lx;
            double sz = 0.0, sp = 0.0;
            for (int i = 0; i < n; ++i) {
                const int xi = i % Lx, yi = i / Lx;
                const int xj = (xi - dx + Lx) % Lx, yj = (yi - dy + Ly) % Ly;
                const int j = xj + yj * Lx;
                const double delta = (i == j) ? 1.0 : 0.0;
                const double pij = (double)(p[i] * p[j]);
                const double gu_ii = G[i + (size_t)i * n], gu_jj = G[j + (size_t)j * n];
                const double gu_ij = G[i + (size_t)j * n], gu_ji = G[j + (size_t)i * n];
                const double gd_ii = two ? Gd[i + (size_t)i * n] : 1.0 - (double)(p[i] * p[i]) * gu_ii;
                const double gd_jj = two ? Gd[j + (size_t)j * n] : 1.0 - (double)(p[j] * p[j]) * gu_jj;
                const double gd_ij = two ? Gd[i + (size_t)j * n] : delta - pij * gu_ji;
                const double gd_ji = two ? Gd[j + (size_t)i * n] : delta - pij * gu_ij;
                const double spin_i = gd_ii - gu_ii, spin_j = gd_jj - gu_jj;
                sz += 0.25 * (spin_i * spin_j + (delta - gu_ji) * gu_ij + (delta - gd_ji) * gd_ij);
                sp += 0.5 * ((delta - gu_ji) * gd_ij + (delta - gd_ji) * gu_ij);
            }
            cz[d] = sz;
            cp[d] = sp;
        }
        __syncthreads();
    }
    double *bins = ch->bins + (size_t)bin * DQMC_BIN_FIELDS;
    if (threadIdx.x == 0) {
        const double U = md.U, mu = md.mu, sign = ch->sign;
        const double ekin = ek, eint = U * ei, ntot = nt, dbl = ei / n;
        const double E = ekin + eint;
        bins[DQMC_BIN_EHUB] += sign * E;
        bins[DQMC_BIN_EGC] += sign * (E - mu * ntot);
        bins[DQMC_BIN_EPH] += sign * (E - 0.5 * U * ntot + 0.25 * U * (double)n);
        bins[DQMC_BIN_N] += sign * ntot;
        bins[DQMC_BIN_D] += sign * dbl;
        bins[DQMC_BIN_SIGN] += sign;
        bins[DQMC_BIN_COUNT] += 1.0;
        bins[DQMC_BIN_ACCEPTED] += (double)(ch->accepted - ch->meas_accepted);
        bins[DQMC_BIN_ATTEMPTS] += (double)(ch->attempts - ch->meas_attempts);
    }
    if (spin) {
        const double sign = ch->sign;
        for (int q = threadIdx.x; q < md.nq_zz; q += NT) {
            double sum = 0.0;
            for (int d = 0; d < n; ++d) sum += md.cos_zz[d + (size_t)q * n] * cz[d];
            ch->bins_zz[(size_t)bin * md.nq_zz + q] += sign * (sum / (double)n);
        }
        for (int q = threadIdx.x; q < md.nq_perp; q += NT) {
            double sum = 0.0;
            for (int d = 0; d < n; ++d) sum += md.cos_perp[d + (size_t)q * n] * cp[d];
            ch->bins_perp[(size_t)bin * md.nq_perp + q] += sign * (sum / (double)n);
        }
    }
    __syncthreads();
    pc.charge(ch, DQMC_PH_MEASURE, 1);
}

/* ---------------------------------------------------------- launchers */
inline size_t smem_bytes(int n, int kb) { return smem_doubles(n, kb) * sizeof(double); }

inline cudaError_t set_attrs(size_t smem, size_t msmem)
{
    cudaError_t e = cudaFuncSetAttribute(k_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_scratch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_wrap, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_measure, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)msmem);
    return e;
}

inline void launch_sweep(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                         const DqmcModelDev *m, int flags, int nsweeps, const int *order)
{
    k_sweep<<<nc, NT, smem, st>>>(c, m, flags, nsweeps, order, (int)nc, (int)nc);
}

/* The sweep kernel with one cluster of cc CTAs per chain (cl_serve). */
inline cudaLaunchConfig_t cluster_config(unsigned nc, int cc, size_t smem, cudaStream_t st,
                                         cudaLaunchAttribute *at)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nc * (unsigned)cc, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cc;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

/* How many clusters of cc CTAs (smem bytes each) the device holds at once
 * (0: such a cluster cannot be resident). */
inline cudaError_t cluster_fit(int cc, size_t smem, int *nclusters)
{
    *nclusters = 0;
    cudaError_t e = cudaSuccess;
    if (cc > 8)
        e = cudaFuncSetAttribute(k_sweep, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = cluster_config(1, cc, smem, nullptr, at);
    return cudaOccupancyMaxActiveClusters(nclusters, (void *)k_sweep, &cfg);
}

/* nclus clusters of cc CTAs: the first ncoop advance one chain each, the
 * others run up to cc of the remaining chains, one per CTA. */
inline cudaError_t launch_sweep_cluster(unsigned nclus, int cc, size_t smem, cudaStream_t st,
                                        DqmcChainDev *c, const DqmcModelDev *m, int flags,
                                        int nsweeps, const int *order, int ncoop, int nchains)
{
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = cluster_config(nclus, cc, smem, st, at);
    return cudaLaunchKernelEx(&cfg, k_sweep, c, m, flags, nsweeps, order, ncoop, nchains);
}

inline void launch_measure(unsigned nc, size_t msmem, cudaStream_t st, DqmcChainDev *c,
                           const DqmcModelDev *m, int bin)
{
    k_measure<<<nc, NT, msmem, st>>>(c, m, bin);
}

inline void launch_init(unsigned nc, size_t smem, cudaStream_t st, DqmcChainDev *c,
                        const DqmcModelDev *m)
{
    k_init<<<nc, NT, smem, st>>>(c, m);
}

}  // namespace DQMC_NS
