/* Mixed-precision wrap: FP64 products emulated on the int8 tensor cores.
 *
 * Split-product scheme (integer Ozaki scheme: Ootomo, Ozaki and Yokota,
 * "DGEMM on integer matrix multiplication unit", 2024): each row of A and
 * each column of B is scaled by a power of two 2^e with max|x| < 2^e and
 * written as the fixed-point integer X = trunc(x 2^(7S-e)), |X| < 2^7S,
 * in base-128 digits: a signed top digit X >> 7(S-1) in [-128, 127] and
 * S-1 lower digits in [0, 127] (two's-complement arithmetic shifts, so the
 * digits reproduce X exactly; |x 2^-e - X 2^-7S| < 2^-7S).  A B is then
 *     2^(e_i + f_j) sum_{p+q < S} 2^-7(p+q+2) (A_p B_q)_ij,
 * the digit products run as mma.sync m16n8k32 s8 x s8 -> s32 (exact: at
 * most S products of |128^2 k| per accumulator, below 2^31 for k <= 21000)
 * and are converted and scaled in FP64.  Dropped terms and the truncation
 * leave about 2^-7S n max_k|a_ik| max_k|b_kj| per entry (S = 6: 2^-42):
 * one wrap stays within 1e-11 of FP64 on the benchmark lattices, far inside
 * the 1e-9 the stabilization tolerates; the pivoted QR, G-from-UDV,
 * B-block products and the acceptance ratios stay FP64.
 *
 * Layouts: digit slice p of an operand is n lines x kp bytes (kp =
 * round64(n), zero padded), line = a row of A or a column of B, so both
 * are contiguous along the summation index, as m16n8k32 row.col reads
 * them.  Only the one-CTA-per-SM build carries this path. */
#pragma once
#include "dqmc_device.cuh"

namespace DQMC_NS {

#if DQMC_MINB == 1

constexpr int MIX_S = DQMC_MIX_DIGITS;
constexpr int MIX_PITCH = 80;                  /* bytes per staged line (64 + 16 pad) */
constexpr int MIX_TILE = 64 * MIX_PITCH;       /* one 64-line x 64-byte slice tile   */
constexpr int MIX_STAGE = 2 * MIX_S * MIX_TILE;
static_assert(2 * MIX_STAGE <= (int)MIX_SMEM_DOUBLES * 8, "mixed staging fits the union");

__host__ __device__ inline int mix_kp(int n) { return ((n + 63) / 64) * 64; }

__device__ __forceinline__ void mix_imma(int *c, const unsigned *a, const unsigned *b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void mix_cp16(void *dst, const void *src, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes));
}

/* Digits of n lines of M (element k of line l at M[k + l*ldm], value
 * rs[k] * M * cs[l] when the scalings are given) into out (S slices of
 * n x kp bytes) and the line exponents into ex. */
__device__ __noinline__ void mix_split(int n, int kp, const double *M, int ldm, const double *rs,
                                       const double *cs, signed char *out, int *ex)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto val = [=](int k, int l) {
        double v = M[k + (size_t)l * ldm];
        if (rs) v = (rs[k] * v) * cs[l];
        return v;
    };
    /* line maxima: a warp takes four lines at a time (independent loads) */
    for (int l0 = 4 * warp; l0 < n; l0 += 4 * NW) {
        double m[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = lane; k < n; k += 32) {
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (l0 + u < n) m[u] = fmax(m[u], fabs(val(k, l0 + u)));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double mu = warp_max(m[u]);
            if (lane == 0 && l0 + u < n) {
                int e = 0;
                if (mu > 0.0) frexp(mu, &e);
                ex[l0 + u] = e;
            }
        }
    }
    __syncthreads();
    const size_t sstride = (size_t)n * kp;
    const int q4 = kp / 4;
    for (int e0 = threadIdx.x; e0 < n * q4; e0 += NT) {
        const int l = e0 / q4, k0 = (e0 - l * q4) * 4;
        const double sc = ldexp(1.0, 7 * MIX_S - ex[l]);   /* exact power of two */
        unsigned w[MIX_S];
#pragma unroll
        for (int p = 0; p < MIX_S; ++p) w[p] = 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u;
            const long long X = k < n ? (long long)(val(k, l) * sc) : 0;
#pragma unroll
            for (int p = 0; p < MIX_S; ++p) {
                const int sh = 7 * (MIX_S - 1 - p);
                const unsigned d = p == 0 ? (unsigned)(X >> sh) & 255u : (unsigned)(X >> sh) & 127u;
                w[p] |= d << (8 * u);
            }
        }
#pragma unroll
        for (int p = 0; p < MIX_S; ++p)
            *(unsigned *)(out + p * sstride + (size_t)l * kp + k0) = w[p];
    }
    __syncthreads();
}

/* C = A B (n x n) from digit slices: A by rows (a, exponents aex), B by
 * columns (b, bex); st(i, j, value).  64 x 64 output tiles, 8 warps as
 * 2 x 4 (warp tile 32 x 16), 64-byte k stages double-buffered by cp.async;
 * per stage and warp the S(S+1)/2 digit products accumulate per diagonal
 * p + q in int32.  sm: 2 * MIX_STAGE bytes, 16-byte aligned. */
template <class ST>
__device__ __forceinline__ void mix_gemm(int n, int kp, const signed char *a, const int *aex,
                                         const signed char *b, const int *bex, ST st,
                                         unsigned char *sm)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    const size_t sstride = (size_t)n * kp;
    const int tm = (n + 63) / 64, nk = kp / 64, total = tm * tm * nk;
    auto advance = [&](int &m0, int &n0, int &k0) {
        k0 += 64;
        if (k0 >= kp) {
            k0 = 0;
            m0 += 64;
            if (m0 >= tm * 64) {
                m0 = 0;
                n0 += 64;
            }
        }
    };
    /* one 16-byte chunk per thread per slice tile: line tid/4, bytes 16*(tid%4) */
    const int cl = tid >> 2, cc = (tid & 3) * 16;
    auto issue = [&](int stg, int m0, int n0, int k0) {
        unsigned char *base = sm + stg * MIX_STAGE;
        const bool va = m0 + cl < n, vb = n0 + cl < n;
#pragma unroll
        for (int p = 0; p < MIX_S; ++p) {
            mix_cp16(base + p * MIX_TILE + cl * MIX_PITCH + cc,
                     va ? a + p * sstride + (size_t)(m0 + cl) * kp + k0 + cc : a, va ? 16 : 0);
            mix_cp16(base + (MIX_S + p) * MIX_TILE + cl * MIX_PITCH + cc,
                     vb ? b + p * sstride + (size_t)(n0 + cl) * kp + k0 + cc : b, vb ? 16 : 0);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int acc[MIX_S][2][2][4];
#pragma unroll
    for (int d = 0; d < MIX_S; ++d)
#pragma unroll
        for (int fm = 0; fm < 2; ++fm)
#pragma unroll
            for (int fn = 0; fn < 2; ++fn)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[d][fm][fn][c] = 0;
    __syncthreads();
    int fm0 = 0, fn0 = 0, fk0 = 0, cm0 = 0, cn0 = 0, ck0 = 0;
    issue(0, fm0, fn0, fk0);
    advance(fm0, fn0, fk0);
    for (int it = 0; it < total; ++it) {
        asm volatile("cp.async.wait_group 0;\n" ::);
        __syncthreads();
        if (it + 1 < total) {
            issue((it + 1) & 1, fm0, fn0, fk0);
            advance(fm0, fn0, fk0);
        }
        const unsigned char *As = sm + (it & 1) * MIX_STAGE, *Bs = As + MIX_S * MIX_TILE;
#pragma unroll
        for (int ks = 0; ks < 64; ks += 32) {
            unsigned bf[MIX_S][2][2];
#pragma unroll
            for (int q = 0; q < MIX_S; ++q)
#pragma unroll
                for (int fn = 0; fn < 2; ++fn) {
                    const unsigned char *r =
                        Bs + q * MIX_TILE + (wn * 16 + fn * 8 + gid) * MIX_PITCH + ks + tig * 4;
                    bf[q][fn][0] = *(const unsigned *)r;
                    bf[q][fn][1] = *(const unsigned *)(r + 16);
                }
#pragma unroll
            for (int p = 0; p < MIX_S; ++p) {
                unsigned af[2][4];
#pragma unroll
                for (int fm = 0; fm < 2; ++fm) {
                    const unsigned char *r =
                        As + p * MIX_TILE + (wm * 32 + fm * 16 + gid) * MIX_PITCH + ks + tig * 4;
                    af[fm][0] = *(const unsigned *)r;
                    af[fm][1] = *(const unsigned *)(r + 8 * MIX_PITCH);
                    af[fm][2] = *(const unsigned *)(r + 16);
                    af[fm][3] = *(const unsigned *)(r + 8 * MIX_PITCH + 16);
                }
#pragma unroll
                for (int q = 0; q < MIX_S; ++q)
                    if (p + q < MIX_S) {
#pragma unroll
                        for (int fm = 0; fm < 2; ++fm)
#pragma unroll
                            for (int fn = 0; fn < 2; ++fn)
                                mix_imma(acc[p + q][fm][fn], af[fm], bf[q][fn]);
                    }
            }
        }
        if (ck0 + 64 >= kp) {
#pragma unroll
            for (int fm = 0; fm < 2; ++fm)
#pragma unroll
                for (int fn = 0; fn < 2; ++fn)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int i = cm0 + wm * 32 + fm * 16 + gid + (c >> 1) * 8;
                        const int j = cn0 + wn * 16 + fn * 8 + 2 * tig + (c & 1);
                        double v = 0.0, w = 1.0;
#pragma unroll
                        for (int d = 0; d < MIX_S + 1; ++d) w *= (1.0 / 128.0);
                        /* smallest diagonal first: weight 2^-7(d+2) */
#pragma unroll
                        for (int d = MIX_S - 1; d >= 0; --d) {
                            v += (double)acc[d][fm][fn][c] * w;
                            w *= 128.0;
                            acc[d][fm][fn][c] = 0;
                        }
                        if (i < n && j < n) st(i, j, ldexp(v, aex[i] + bex[j]));
                    }
        }
        advance(cm0, cn0, ck0);
    }
    __syncthreads();
}

/* G <- B_l G B_l^{-1} as wrap_green, both products split: tmp (row-major)
 * = expK [diag(v) G diag(1/v)], G = tmp expKinv. */
__device__ __noinline__ void wrap_green_mixed(int n, double *G, double *tmp, const DqmcModelDev &md,
                                              const signed char *fl, double v0, double v1,
                                              double vi0, double vi1, signed char *mix,
                                              int *mix_ex, Smem &s)
{
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    __syncthreads();
    const int kp = md.mix_kp;
    unsigned char *sm = (unsigned char *)s.q.X;
    mix_split(n, kp, G, n, vv, vi, mix, mix_ex);
    mix_gemm(n, kp, md.mixK, md.mixK_ex, mix, mix_ex,
             [=](int i, int j, double v) { tmp[(size_t)i * n + j] = v; }, sm);
    mix_split(n, kp, tmp, n, nullptr, nullptr, mix, mix_ex);
    mix_gemm(n, kp, mix, mix_ex, md.mixKinv, md.mixKinv_ex,
             [=](int i, int j, double v) { G[i + (size_t)j * n] = v; }, sm);
}

#endif  /* DQMC_MINB == 1 */

}  // namespace DQMC_NS
