/* Mixed precision: FP64 products emulated on the int8 tensor cores
 * (tcgen05.mma kind::i8, accumulators in tensor memory).
 *
 * Split-product scheme (integer Ozaki scheme: Ootomo, Ozaki and Yokota,
 * "DGEMM on integer matrix multiplication unit", 2024), with balanced
 * digits.  Every line of an operand (a row of A or a column of B) is scaled
 * by 2^(NB - e), e the binary exponent of the line's largest magnitude, and
 * rounded to the nearest integer X, |X| <= 2^NB, NB = 8 S - 2.  X is written
 * in S signed base-256 digits taken from the bottom, each in [-128, 127]
 * ("balanced": d = ((X + 128) mod 256) - 128, X <- (X - d) / 256), so the
 * digits reproduce X exactly and the top digit stays within [-65, 65].
 * Then, with a_p, b_q the digit matrices,
 *     (A B)_ij = 2^(e_i + f_j - 2 NB) sum_{p+q <= S-1} 2^(8 (2S-2-p-q)) (A_p B_q)_ij
 * up to the dropped diagonals p + q >= S and the rounding of X.  Each digit
 * product is exact in int32 (|a_p b_q| <= 2^14 per term, K <= 2^14 terms
 * would still fit; the engine's K is n <= 1024) and the S diagonal sums
 * d = p + q accumulate in S int32 accumulators.
 *
 * Balanced, rounded digits matter: with truncated digits and unsigned lower
 * digits every dropped term has the same sign and the error of the wrapped G
 * grows coherently over a stabilization interval.  A CPU emulation of this
 * exact arithmetic in the reference's forward sweep (16x16, U=4, beta=8,
 * stab=8, delay 32, wrap and flush split) gives max|G - G_FP64| before each
 * rebuild of 1.2e-6 for S = 6, 2.9e-9 for S = 7 and 4.1e-11 for S = 8.  On
 * the GPU, S = 7 reached 2.2e-8 over three chains of that lattice, so the
 * engine uses S = DQMC_MIX_DIGITS = 8 (36 digit products per FP64 product,
 * all 512 tensor-memory columns).
 *
 * Data path (one CTA = one chain, 256 threads):
 *  - operands are split into a tiled global buffer: block (128 lines, 32 k)
 *    = S digit slices of 128 lines x 32 bytes, each slice already in the
 *    tensor core's K-major no-swizzle canonical layout (8-line x 16-byte
 *    core matrices; the two 16-byte k halves 2 KB apart), so the operand
 *    data of one pipeline stage is one contiguous bulk copy per operand
 *    (cp.async.bulk, completing on an mbarrier);
 *  - output tiles are 128 x 128 (tcgen05.mma M = 128, N = 128, K = 32,
 *    s8 x s8 -> s32) in two passes over k: pass 0 accumulates the digit
 *    diagonals d = p + q = 0..3 (slices 0..3, 10 MMAs per chunk), pass 1
 *    the diagonals 4..7 (26 MMAs), four accumulators of 128 tensor-memory
 *    columns each.  A microbenchmark on B200 measured about 104 cycles per
 *    M = 128 kind::i8 MMA for N <= 128 and 129 cycles for N = 256, so wide
 *    tiles matter more than the number of accumulators;
 *  - thread 0 issues the copies (one stage ahead) and the MMAs, then
 *    tcgen05.commit to the stage's "empty" barrier and, after a pass's
 *    last chunk, to the "accum" barrier that releases the epilogue: every
 *    warp reads its 32 tensor-memory lanes (tile rows) with tcgen05.ld,
 *    combines the pass's four diagonals exactly in int64 and scales by the
 *    two lines' powers of two; pass 1 adds to pass 0's result.
 * Every wait is bounded (about two seconds); a wait that runs out sets the
 * context's error flag, the product is abandoned and the chain stops with
 * DQMC_ST_TIMEOUT.  Only the one-CTA-per-SM build carries this path (the
 * accumulators take all 512 tensor-memory columns of the SM).  TMA loads
 * here never use cluster multicast: every operand is this GPU's memory. */
#pragma once
#include "dqmc_device.cuh"

namespace DQMC_NS {

#if DQMC_MINB == 1

constexpr int SPL_S = DQMC_MIX_DIGITS;
static_assert(SPL_S == 8, "the GEMM runs two passes of four digit diagonals");
constexpr int SPL_NB = 8 * SPL_S - 2;            /* bits of a line's fixed point       */
constexpr int SPL_LB = 128;                       /* lines per block: A rows, B columns */
constexpr int SPL_KC = 32;                        /* bytes (= k) per chunk               */
constexpr int SPL_SLICE = SPL_LB * SPL_KC;        /* one digit slice of a block chunk    */
constexpr int SPL_TILE = SPL_S * SPL_SLICE;       /* all digits of a block chunk (32 KB) */
constexpr int SPL_STAGE = 2 * SPL_TILE;           /* A and B                             */
constexpr int SPL_NSTAGE = DQMC_SPL_STAGES;
constexpr int SPL_N = 128;                        /* tile columns (MMA N)                */
constexpr int SPL_ACC = 4;                        /* accumulators (diagonals) per pass   */
constexpr int SPL_TMEM_COLS = 512;
constexpr long long SPL_WAIT_CYCLES = 4000000000ll;   /* about 2 s at 1.9 GHz */
static_assert(SPL_ACC * SPL_N == SPL_TMEM_COLS, "four 128-column accumulators");
static_assert((size_t)SPL_NSTAGE * SPL_STAGE <= MIX_SMEM_DOUBLES * 8, "stages fit the union");

/* instruction descriptor: D s32 (bits 4-5 = 2), A and B signed 8-bit (bits
 * 7-9, 10-12 = 1), both K-major, N = 128 (bits 17-22 = N/8), M = 128 (bits
 * 24-28 = M/16) */
constexpr uint32_t SPL_IDESC =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SPL_N >> 3) << 17) | ((128u >> 4) << 24);

/* Per-CTA state of the split GEMM (shared memory). */
struct SplCtx {
    unsigned long long full[SPL_NSTAGE], empty[SPL_NSTAGE], accum;
    uint32_t tmem;     /* tensor-memory base address of the accumulators */
    int err;           /* a bounded wait ran out                          */
    unsigned seq;      /* k chunks consumed so far (stage ring position)  */
    unsigned tiles;    /* accumulator phases so far                       */
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity)
{
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > SPL_WAIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* Kernel entry: barriers, tensor memory (warp 0 allocates all 512 columns;
 * the CTA's shared-memory size keeps it alone on its SM). */
__device__ __forceinline__ void spl_setup(SplCtx *cx)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s < SPL_NSTAGE; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cx->full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cx->empty[s])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cx->accum)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        cx->err = 0;
        cx->seq = 0;
        cx->tiles = 0;
    }
    __syncwarp();
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&cx->tmem)),
                     "r"(SPL_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

/* Kernel exit: every tcgen05 operation of the CTA has completed (each GEMM
 * waits for its last accumulator phase; after a timeout a final commit is
 * awaited, bounded), then warp 0 frees the tensor memory. */
__device__ __forceinline__ void spl_teardown(SplCtx *cx)
{
    __syncthreads();
    if (threadIdx.x == 0 && cx->err) {
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&cx->accum)));
        mbar_wait(&cx->accum, cx->tiles & 1);
    }
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(cx->tmem),
                     "r"(SPL_TMEM_COLS));
    }
}

/* A split operand (DqmcSplitDev): blocks (lb, kc) of 128 lines x 32 k at
 * t + (lb * nkc + kc) * SPL_TILE, digit slice p of a block at p * SPL_SLICE
 * (the top digit first), and the per-line scale
 * sc[l] = 2^(e_l - NB + 4 (S - 1)). */
using SplitOp = DqmcSplitDev;

/* byte offset of digit slice p of entry (line l, k) in a split buffer: the
 * tensor core's K-major no-swizzle layout, 8-line x 16-byte core matrices,
 * the two 16-byte k halves of a chunk LB * 16 bytes apart */
__host__ __device__ inline size_t spl_offset(int nkc, int l, int k, int p)
{
    return ((size_t)(l / SPL_LB) * nkc + k / SPL_KC) * SPL_TILE + (size_t)p * SPL_SLICE +
           ((k >> 4) & 1) * (SPL_LB * 16) + ((l % SPL_LB) >> 3) * 128 + (l & 7) * 16 + (k & 15);
}

__host__ __device__ inline int spl_nlb(int lines) { return (lines + SPL_LB - 1) / SPL_LB; }
__host__ __device__ inline int spl_nkc(int k) { return (k + SPL_KC - 1) / SPL_KC; }
/* bytes of a split buffer with room for `lines` lines and K <= kmax */
__host__ __device__ inline size_t spl_tile_bytes(int lines, int kmax)
{
    return (size_t)spl_nlb(lines) * spl_nkc(kmax) * SPL_TILE;
}

/* Exact conversions between doubles and 64-bit integers below 2^51 in
 * magnitude with FP64 adds (the integer conversion instructions are slow):
 * 1.5 * 2^52 + x has unit spacing, so adding it rounds x to the nearest
 * integer and leaves that integer in the low bits of the word. */
constexpr double SPL_MAGIC = 6755399441055744.0;          /* 1.5 * 2^52 */
constexpr long long SPL_MAGIC_BITS = 0x4338000000000000ll;
__device__ __forceinline__ double spl_i2d(long long h)     /* |h| < 2^51 */
{
    return __longlong_as_double(h + SPL_MAGIC_BITS) - SPL_MAGIC;
}

/* The digits of X = round(x f) (|X| <= 2^62) as the bytes of one word:
 * adding 128 to each of the seven lower balanced digits makes them the
 * plain bytes of X + 0x0080..80, so (X + B) ^ B, B = 0x0080808080808080,
 * holds digit byte 7 - p of slice p (slice 0 = the top digit). */
__device__ __forceinline__ unsigned long long spl_digits(double x, double f)
{
    const long long X = __double2ll_rn(x * f);
    return (unsigned long long)(X + 0x0080808080808080ll) ^ 0x0080808080808080ull;
}

/* 4 x 4 byte transpose: o[k] = byte k of a, b, c, d */
__device__ __forceinline__ void spl_tr4(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                        uint32_t (&o)[4])
{
    const uint32_t ab0 = __byte_perm(a, b, 0x5140), ab1 = __byte_perm(a, b, 0x7362);
    const uint32_t cd0 = __byte_perm(c, d, 0x5140), cd1 = __byte_perm(c, d, 0x7362);
    o[0] = __byte_perm(ab0, cd0, 0x5410);
    o[1] = __byte_perm(ab0, cd0, 0x7632);
    o[2] = __byte_perm(ab1, cd1, 0x5410);
    o[3] = __byte_perm(ab1, cd1, 0x7632);
}

/* Digits of the lines of an operand into op: line l < lines holds ld(k, l)
 * for k < K; lines and k are zero-padded to whole blocks.  KCONTIG: a
 * line's entries are contiguous in memory, otherwise consecutive lines are;
 * the maxima take a thread per line, sixteen loads in flight.  The digit
 * pass gives consecutive threads consecutive lines of one 16-entry k group
 * (coalesced 16-byte stores), two groups in flight per thread. */
template <bool KCONTIG, class LD>
__device__ __noinline__ void spl_split(int lines, int K, LD ld, SplitOp op, Part pt = Part())
{
    const int tid = threadIdx.x;
    const int lpad_all = op.nlb * SPL_LB;
    /* this CTA's lines [l0, l0 + lpad) (all of them unless a cluster shares
     * the split; each line's scale and digits depend on that line alone) */
    const int per = (lpad_all + pt.c - 1) / pt.c;
    const int l0 = min(lpad_all, pt.r * per);
    const int lpad = min(lpad_all, l0 + per) - l0;
    auto set_line = [&](int l, double m) {
        int e = 0;
        if (m > 0.0 && isfinite(m)) frexp(m, &e);
        /* a non-finite line poisons its products (NaN scale) so that the
         * stabilization check sees it */
        op.sc[l] = isfinite(m) ? ldexp(1.0, e - SPL_NB + 4 * (SPL_S - 1))
                               : __longlong_as_double(0x7ff8000000000000ll);
    };
    if (KCONTIG) {
        /* a thread per line; 16 entries (128 contiguous bytes) per step */
        for (int l = l0 + tid; l < l0 + lpad; l += NT) {
            double m = 0.0;
            if (l < lines) {
                int k = 0;
                for (; k + 16 <= K; k += 16) {
                    double x[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) x[u] = fabs(ld(k + u, l));
#pragma unroll
                    for (int u = 0; u < 16; ++u) m = (x[u] > m || x[u] != x[u]) ? x[u] : m;
                }
                for (; k < K; ++k) {
                    const double x = fabs(ld(k, l));
                    m = (x > m || x != x) ? x : m;
                }
            }
            set_line(l, m);
        }
    } else {
        for (int l = l0 + tid; l < l0 + lpad; l += NT) {
            double m = 0.0;
            if (l < lines) {
                /* sixteen independent loads in flight per step */
                int k = 0;
                for (; k + 16 <= K; k += 16) {
                    double x[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) x[u] = fabs(ld(k + u, l));
#pragma unroll
                    for (int u = 0; u < 16; ++u) m = (x[u] > m || x[u] != x[u]) ? x[u] : m;
                }
                for (; k < K; ++k) {
                    const double x = fabs(ld(k, l));
                    m = (x > m || x != x) ? x : m;
                }
            }
            set_line(l, m);
        }
    }
    __syncthreads();
    const int items = lpad * op.nkc * 2;   /* (line, 16-entry k group) */
    /* 2^(NB - e) = 2^(4 (S - 1)) / sc, exact for powers of two */
    const double f0 = ldexp(1.0, 4 * (SPL_S - 1));
    for (int it0 = tid; it0 < items; it0 += 2 * NT) {
        double x[2][16];
        int ll[2], gg[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int it = it0 + h * NT;
            ll[h] = l0 + (lpad > 0 ? it % lpad : 0);
            gg[h] = it < items ? it / lpad : -1;
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int k = gg[h] * 16 + u;
                x[h][u] = (gg[h] >= 0 && ll[h] < lines && k < K) ? ld(k, ll[h]) : 0.0;
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (gg[h] < 0) continue;
            const int l = ll[h], g = gg[h];
            const double f = f0 / op.sc[l];
            uint32_t w[SPL_S][4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                unsigned long long z[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) z[u] = spl_digits(x[h][4 * q + u], f);
                uint32_t lo[4], hi[4];
                spl_tr4((uint32_t)z[0], (uint32_t)z[1], (uint32_t)z[2], (uint32_t)z[3], lo);
                spl_tr4((uint32_t)(z[0] >> 32), (uint32_t)(z[1] >> 32), (uint32_t)(z[2] >> 32),
                        (uint32_t)(z[3] >> 32), hi);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    w[7 - b][q] = lo[b];   /* byte b: slice 7 - b  */
                    w[3 - b][q] = hi[b];   /* byte 4 + b: slice 3 - b */
                }
            }
            signed char *dst = op.t + spl_offset(op.nkc, l, g * 16, 0);
#pragma unroll
            for (int p = 0; p < SPL_S; ++p)
                *reinterpret_cast<uint4 *>(dst + (size_t)p * SPL_SLICE) =
                    make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
        }
    }
    /* the digits are read next by bulk copies (the async proxy) */
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
}

/* shared-memory matrix descriptor, K-major, no swizzle: start, leading
 * byte offset (between the two 16-byte k halves), stride byte offset
 * (between 8-line groups), version 1 (bit 46) */
__device__ __forceinline__ uint64_t spl_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void spl_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc)
{
    const uint32_t z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(SPL_IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void spl_bulk(uint32_t dst, const void *src, uint32_t bytes,
                                         unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];\n" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
}

/* Epilogues: a thread gets row i and eight consecutive columns j0..j0+7
 * (nj of them inside the matrix) of one pass: pass 0 carries the four top
 * digit diagonals, pass 1 the four lower ones, added to pass 0's result.
 * load() runs before the accumulators are read, so a read-modify-write's
 * loads overlap the tensor-memory reads. */
struct EpiStore {     /* C = A B */
    double *C;
    int ldc;
    __device__ __forceinline__ void load(int i, int j0, int nj, int pass, double (&o)[8]) const
    {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            o[c] = (pass && c < nj) ? C[i + (size_t)(j0 + c) * ldc] : 0.0;
    }
    __device__ __forceinline__ void store(int i, int j0, int nj, int, const double (&v)[8],
                                          const double (&o)[8]) const
    {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c < nj) C[i + (size_t)(j0 + c) * ldc] = o[c] + v[c];
    }
};
struct EpiSub {       /* C -= A B */
    double *C;
    int ldc;
    __device__ __forceinline__ void load(int i, int j0, int nj, int, double (&o)[8]) const
    {
#pragma unroll
        for (int c = 0; c < 8; ++c) o[c] = c < nj ? C[i + (size_t)(j0 + c) * ldc] : 0.0;
    }
    __device__ __forceinline__ void store(int i, int j0, int nj, int, const double (&v)[8],
                                          const double (&o)[8]) const
    {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c < nj) C[i + (size_t)(j0 + c) * ldc] = o[c] - v[c];
    }
};
struct EpiDiag {      /* C = diag(r) (A B) diag(q) */
    double *C;
    int ldc;
    const double *r, *q;
    __device__ __forceinline__ void load(int i, int j0, int nj, int pass, double (&o)[8]) const
    {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            o[c] = (pass && c < nj) ? C[i + (size_t)(j0 + c) * ldc] : 0.0;
    }
    __device__ __forceinline__ void store(int i, int j0, int nj, int, const double (&v)[8],
                                          const double (&o)[8]) const
    {
        const double ri = r[i];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c < nj) C[i + (size_t)(j0 + c) * ldc] = o[c] + (ri * v[c]) * q[j0 + c];
    }
};

/* C = A B (M x N) from split operands (A by rows, B by columns, the same
 * nkc); the epilogue object writes the result (EpiStore, EpiSub, EpiDiag).
 * Output tiles of 128 x 128 in two passes over k: pass 0 accumulates the
 * digit diagonals d = p + q = 0..3 (10 MMAs per chunk, slices 0..3 of each
 * operand), pass 1 the diagonals 4..7 (26 MMAs, all slices); the epilogue
 * of a pass combines its four diagonals exactly in int64.  sm:
 * SPL_NSTAGE * SPL_STAGE bytes of shared memory, 16-byte aligned.  Returns
 * false when a wait ran out (cx->err set; nothing further is issued). */
template <class EPI>
__device__ __noinline__ bool spl_gemm(int M, int N, SplitOp A, SplitOp B, EPI epi,
                                      unsigned char *sm, SplCtx *cx, Part pt = Part())
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tm = (M + SPL_LB - 1) / SPL_LB, tn = (N + SPL_N - 1) / SPL_N, nk = A.nkc;
    /* this CTA's tiles pt.r, pt.r + pt.c, ... (all of them by default) */
    const int ntile = tm * tn > pt.r ? (tm * tn - pt.r + pt.c - 1) / pt.c : 0;
    const unsigned total = (unsigned)ntile * 2 * nk;
    /* earlier generic-proxy use of the staging area is ordered before the
     * bulk copies that overwrite it; operands split by other CTAs of a
     * cluster (published by the cluster barrier) before the bulk reads */
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    if (cx->err) return false;
    const uint32_t sbase = smem_u32(sm);
    const unsigned seq0 = cx->seq;
    unsigned tiles = cx->tiles;
    /* thread 0: stage ring position g = seq0 + chunk; chunk x = (tile, pass,
     * kc); a stage is refilled once the MMAs of its previous chunk have
     * completed ("empty"); pass 0 needs the top four digit slices only */
    auto issue = [&](unsigned x) {
        const unsigned g = seq0 + x, st = g % SPL_NSTAGE, u = g / SPL_NSTAGE;
        if (u >= 1 && !mbar_wait(&cx->empty[st], (u - 1) & 1)) {
            cx->err = 1;
            return;
        }
        const int it = pt.r + pt.c * (int)(x / (2 * nk)), pass = (int)((x / nk) & 1),
                  ik = (int)(x % nk);
        const uint32_t bytes = (pass ? SPL_S : SPL_ACC) * SPL_SLICE;
        const signed char *ga = A.t + ((size_t)(it % tm) * A.nkc + ik) * (size_t)SPL_TILE;
        const signed char *gb = B.t + ((size_t)(it / tm) * B.nkc + ik) * (size_t)SPL_TILE;
        const uint32_t sa = sbase + st * SPL_STAGE;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_u32(&cx->full[st])),
                     "r"(2 * bytes)
                     : "memory");
        spl_bulk(sa, ga, bytes, &cx->full[st]);
        spl_bulk(sa + SPL_TILE, gb, bytes, &cx->full[st]);
    };
    if (tid == 0)
        for (unsigned x = 0; x + 1 < SPL_NSTAGE && x < total && !cx->err; ++x) issue(x);
    for (int t = 0; t < ntile; ++t) {
        const int gt = pt.r + pt.c * t, mb = gt % tm, nb = gt / tm;
        for (int pass = 0; pass < 2; ++pass) {
            if (tid == 0) {
                tc_fence_after();
                for (int kc = 0; kc < nk && !cx->err; ++kc) {
                    const unsigned c = ((unsigned)t * 2 + pass) * nk + kc;
                    const unsigned g = seq0 + c, st = g % SPL_NSTAGE, u = g / SPL_NSTAGE;
                    if (!mbar_wait(&cx->full[st], u & 1)) {
                        cx->err = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = sbase + st * SPL_STAGE, sb = sa + SPL_TILE;
#pragma unroll
                    for (int a = 0; a < SPL_ACC; ++a) {
                        const int d = SPL_ACC * pass + a;
                        for (int p = 0; p <= d; ++p)
                            spl_mma(cx->tmem + (uint32_t)(SPL_N * a),
                                    spl_desc(sa + p * SPL_SLICE, SPL_LB * 16, 128),
                                    spl_desc(sb + (d - p) * SPL_SLICE, SPL_LB * 16, 128),
                                    (kc > 0 || p > 0) ? 1u : 0u);
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                        "[%0];" ::"r"(smem_u32(&cx->empty[st]))
                        : "memory");
                    /* refill the stage of chunk c + 1 - NSTAGE (its MMAs run
                     * ahead of this chunk's in the tensor pipe) */
                    if (c + SPL_NSTAGE - 1 < total) issue(c + SPL_NSTAGE - 1);
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&cx->accum))
                    : "memory");
            }
            __syncwarp();
            /* epilogue: every thread waits for the pass's accumulators */
            const bool ok = __all_sync(FULL, mbar_wait(&cx->accum, tiles & 1));
            ++tiles;
            tc_fence_after();
            if (ok) {
                const int i = mb * SPL_LB + (warp & 3) * 32 + lane;
                const int cb = (warp >> 2) * (SPL_N / 2);
                const double sa = A.sc[i];
                const double wsc = pass ? 1.0 : 4294967296.0;   /* 2^32 */
                const uint32_t taddr = cx->tmem + ((uint32_t)((warp & 3) * 32) << 16);
                /* the next group's old values and column scales are loaded
                 * one group ahead */
                auto jnj = [&](int cc, int &j0) {
                    j0 = nb * SPL_N + cb + 8 * cc;
                    return i < M ? max(0, min(8, N - j0)) : 0;
                };
                int j0n;
                int njn = jnj(0, j0n);
                double oldn[8], sbn[8];
                epi.load(i, j0n, njn, pass, oldn);
#pragma unroll
                for (int c = 0; c < 8; ++c) sbn[c] = c < njn ? B.sc[j0n + c] : 0.0;
#pragma unroll 1
                for (int cc = 0; cc < SPL_N / 16; ++cc) {
                    const int j0 = j0n, nj = njn;
                    double old[8], sb[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        old[c] = oldn[c];
                        sb[c] = sbn[c];
                    }
                    if (cc + 1 < SPL_N / 16) {
                        njn = jnj(cc + 1, j0n);
                        epi.load(i, j0n, njn, pass, oldn);
#pragma unroll
                        for (int c = 0; c < 8; ++c) sbn[c] = c < njn ? B.sc[j0n + c] : 0.0;
                    }
                    uint32_t r[SPL_ACC][8];
                    __syncwarp();
#pragma unroll
                    for (int a = 0; a < SPL_ACC; ++a)
                        tmem_ld8(taddr + SPL_N * a + cb + 8 * cc, r[a]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    double v[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        /* the pass's four diagonals in base 256, exactly
                         * (|acc| < 2^27 for K <= 1024, so |h| < 2^51): pass 0
                         * weighs 2^32 relative to pass 1 */
                        long long h = (int)r[0][c];
#pragma unroll
                        for (int a = 1; a < SPL_ACC; ++a) h = h * 256 + (int)r[a][c];
                        v[c] = ((spl_i2d(h) * wsc) * sa) * sb[c];
                    }
                    if (nj > 0) epi.store(i, j0, nj, pass, v, old);
                }
            } else if (lane == 0) {
                atomicExch(&cx->err, 1);
            }
            tc_fence_before();
            __syncthreads();
            if (cx->err) break;
        }
        if (cx->err) break;
    }
    if (tid == 0) {
        cx->seq = seq0 + total;
        cx->tiles = tiles;
    }
    __syncthreads();
    return !cx->err;
}

/* End of a split product as a command of a cluster per chain: a rank whose
 * bounded wait ran out reports it in the command block, rank 0 takes it
 * into its own error state after the last barrier. */
__device__ __forceinline__ bool spl_cl_finish(Smem &s, SplCtx *cx)
{
    if (s.cl.c > 1) {
        if (s.cl.r > 0 && threadIdx.x == 0 && cx->err) atomicOr(&s.cmd->err, 1);
        cl_done(s);
        if (s.cl.r == 0 && threadIdx.x == 0 && *(volatile int *)&s.cmd->err) cx->err = 1;
        __syncthreads();
    }
    return !cx->err;
}

/* G <- B_l G B_l^-1 (green_wrap, green.c:509-527) or, back, G <- B_l^-1
 * G B_l (green_wrap_backward, green.c:529-548), both products split:
 * forward P = [diag(v) G diag(1/v)] expK^-1, G = expK P; backward
 * P = G expK, G = diag(1/v) (expK^-1 P) diag(v).  P: n x n scratch.
 * A split command with a cluster per chain: the ranks split a range of
 * lines of each operand and form a share of the output tiles, each on its
 * own tensor memory; the per-tile arithmetic is the one-CTA product's.
 * Every rank runs every step (a failed wait makes the later products
 * return at once) so the ranks stay in step. */
__device__ __noinline__ bool wrap_green_split(int n, double *G, double *P, const DqmcModelDev &md,
                                              const DqmcChainDev *ch, const signed char *fl,
                                              double v0, double v1, double vi0, double vi1,
                                              bool back, Smem &s)
{
    cl_post(s, CL_WSPLIT, G, P, &md, ch, fl, nullptr, n, back ? 1 : 0, 0, v0, v1, vi0, vi1);
    const Part pt = s.cl;
    double *vv = s.vA, *vi = s.vB;
    for (int k = threadIdx.x; k < n; k += NT) {
        const bool up = fl[k] > 0;
        vv[k] = up ? v1 : v0;
        vi[k] = up ? vi1 : vi0;
    }
    __syncthreads();
    SplCtx *cx = (SplCtx *)s.spl;
    unsigned char *sm = (unsigned char *)s.gsm;
    SplitOp a = ch->spA, b = ch->spB;
    a.nkc = b.nkc = spl_nkc(n);
    if (!back) {
        spl_split<false>(
            n, n, [=](int k, int l) { return (vv[l] * G[l + (size_t)k * n]) * vi[k]; }, a, pt);
        part_sync(s);
        spl_gemm(n, n, a, md.spKi_c, EpiStore{P, n}, sm, cx, pt);
        part_sync(s);
        spl_split<true>(n, n, [=](int k, int l) { return P[k + (size_t)l * n]; }, b, pt);
        part_sync(s);
        spl_gemm(n, n, md.spK_r, b, EpiStore{G, n}, sm, cx, pt);
    } else {
        spl_split<false>(n, n, [=](int k, int l) { return G[l + (size_t)k * n]; }, a, pt);
        part_sync(s);
        spl_gemm(n, n, a, md.spK_c, EpiStore{P, n}, sm, cx, pt);
        part_sync(s);
        spl_split<true>(n, n, [=](int k, int l) { return P[k + (size_t)l * n]; }, b, pt);
        part_sync(s);
        spl_gemm(n, n, md.spKi_r, b, EpiDiag{G, n, vi, vv}, sm, cx, pt);
    }
    return spl_cl_finish(s, cx);
}

/* G -= Zs Ys, rank mt (green_delay_flush, green.c:462-475, through
 * la_gemm_nt_rect, linalg.c:209-219) as a split product; Zs n x mt (ld n),
 * Ys mt x n (ld ldy).  A split command with a cluster per chain (as the
 * wrap). */
__device__ __noinline__ bool flush_split(int n, int mt, double *G, const double *Zs,
                                         const double *Ys, int ldy, const DqmcChainDev *ch,
                                         Smem &s)
{
    cl_post(s, CL_FSPLIT, G, Zs, Ys, ch, nullptr, nullptr, n, mt, ldy);
    const Part pt = s.cl;
    SplitOp a = ch->spA, b = ch->spB;
    a.nkc = b.nkc = spl_nkc(mt);
    spl_split<false>(n, mt, [=](int k, int l) { return Zs[l + (size_t)k * n]; }, a, pt);
    spl_split<true>(n, mt, [=](int k, int l) { return Ys[k + (size_t)l * ldy]; }, b, pt);
    part_sync(s);
    spl_gemm(n, n, a, b, EpiSub{G, n}, (unsigned char *)s.gsm, (SplCtx *)s.spl, pt);
    return spl_cl_finish(s, (SplCtx *)s.spl);
}

#endif  /* DQMC_MINB == 1 */

}  // namespace DQMC_NS
