/* Masked coherence-matrix accumulation on the tcgen05 tensor cores:
 *
 *   C_p = sum over SHPs q of p:  s_q s_q^H          (tcoh.cl:567-602)
 *
 * written, for one tile of 128 output pixels (16 rows x 8 columns, the M
 * extent of one accumulator), as a single GEMM
 *
 *   D[p][col] = sum over k of A[p][k] B[k][col]
 *
 * - k runs over the union of the tile's windows, (16 + WA - 1) x (8 + WR - 1)
 *   candidates (36 x 14 = 504 at 21 x 7), row-major;
 * - A[p][k] is 1 where candidate k is an SHP of pixel p, else 0 (exact in
 *   BF16);
 * - a column is the real or the imaginary part of one packed upper-triangle
 *   entry (i, j), and B[k][col] the same part of the candidate's product
 *   s_k,i conj(s_k,j). The product is formed once in FP32 and split exactly
 *   into BF16 terms by rounding to nearest: hi = the product to 8
 *   significant bits, mid = the remainder to 8 bits, lo = the rest, exact
 *   (hi + mid + lo == the FP32 product, bit for bit). Each term is one MMA
 *   pass into the same FP32 accumulator, so D is an FP32 sum of the exact
 *   FP32 products. With two terms lo is dropped: a relative error of at
 *   most 2^-17 per product.
 *
 * Per CTA (256 threads, two CTAs per SM, persistent): the packed entries are
 * taken 128 at a time ("phases"); a phase's accumulator is 128 lanes x 2h
 * columns of TMEM (re of entry r in column r, im in column h + r, h =
 * entries rounded up to 16). The CTAs take (tile, phase) items in turn, so
 * that the last round of a launch is split four ways instead of leaving
 * whole tiles on a fraction of the SMs. For each block of 16 candidates
 * (one MMA K step) the CTA builds A and the B terms in the canonical
 * K-major layout without swizzle (8-row x 16-byte core matrices) into one
 * of two operand buffers, and one thread issues the MMAs (M = 128,
 * N = 2h, K = 16) and commits them to that buffer's mbarrier: block kb is
 * built while block kb - 1 multiplies, and a buffer is rebuilt once the
 * MMAs that read it (block kb - 2) have completed. The next block's samples
 * load into registers meanwhile. The epilogue reads the accumulator with
 * tcgen05.ld and writes gram[p][pidx] (float2), the layout the linking
 * kernels read.
 *
 * Candidates that are not finite contribute zero: a product with A = 0 must
 * stay zero, and a candidate with a non-finite sample is invalid and never
 * an SHP (the caller's valid mask marks it, main.c:60-111).
 *
 * Every wait on the mbarrier is bounded; a wait that runs out sets a fault
 * flag (read by tc_gram_tensor_fault), fills the tile's entries with NaN,
 * frees the tile's TMEM and returns.
 */
#include "tcoh_internal.h"

#include <math.h>

namespace {

constexpr int KB = 16;            /* candidates per K block: one MMA K step */
constexpr int KCH = KB / 8;       /* 16-byte K chunks per K block */
constexpr int STAGES = 2;         /* operand buffers */
constexpr int THREADS = 256;
constexpr int PHASE = 128;        /* packed entries per accumulator phase */
constexpr int TMEM_COLS = 256;    /* 2 x PHASE FP32 columns */
constexpr int STAGE_LD = KB + 2;  /* float2 per date row of the staged samples */
constexpr uint32_t WAIT_LIMIT = 1u << 22;
constexpr int MIN_SMEM = 80 << 10; /* keeps at most two CTAs (512 TMEM columns) per SM */
constexpr int MAX_WR = 25;        /* window row bits of one pixel, shifted by <= 7, fit 32 */
constexpr int MAX_WA = 64;

/* Shared-memory carve-up (byte offsets). */
struct GramSmem {
    int ops;     /* STAGES x (3 B terms x KCH chunks x 256 rows x 16 B, then A:
                    KCH chunks x 128 rows x 16 B) */
    int stage;   /* n x STAGE_LD float2 */
    int uyx;     /* K x u16: union row << 8 | union column of candidate u */
    int rows;    /* wa x 128 u32: SHP bits of each window row of each pixel */
    int pair;    /* npu x u16 */
    int expand;  /* 16 x uint2: four mask bits -> four BF16 0/1 */
    int bar;     /* STAGES mbarriers (16 B), TMEM address (4 B + pad), drain mbarrier (8 B) */
    int bytes;
};

constexpr int TERM_BYTES = KCH * 2 * PHASE * 16;
constexpr int OP_BYTES = 3 * TERM_BYTES + KCH * 128 * 16;
/* the epilogue stages each warp's 32 pixels x 16 entries (+1 pad) in the
   idle operand buffers */
static_assert(8 * 32 * 17 * 8 <= STAGES * OP_BYTES, "epilogue staging exceeds the operand buffers");

__host__ __device__ inline int up16(int x) { return (x + 15) & ~15; }

__host__ __device__ inline GramSmem gram_smem(int n, int wa, int wr)
{
    GramSmem g;

    g.ops = 0;
    g.stage = g.ops + STAGES * OP_BYTES;
    g.uyx = g.stage + up16(n * STAGE_LD * 8);
    g.rows = g.uyx + up16((TC_TILE_H + wa - 1) * (TC_TILE_W + wr - 1) * 2);
    g.pair = g.rows + wa * 128 * 4;
    g.expand = g.pair + up16(tc_npu(n) * 2);
    g.bar = g.expand + 16 * 8;
    g.bytes = g.bar + 32;
    return g;
}

__device__ int g_gram_fault;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* Shared-memory matrix descriptor: K-major, no swizzle. lbo = bytes between
   the two 8-element K halves of one MMA, sbo = bytes between 8-row groups. */
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3fff) | (uint64_t)((lbo >> 4) & 0x3fff) << 16 |
           (uint64_t)((sbo >> 4) & 0x3fff) << 32 | (uint64_t)1 << 46;
}

/* Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, both K-major,
   M = 128, N = n. */
__device__ __forceinline__ uint32_t instr_desc(int n)
{
    return 1u << 4 | 1u << 7 | 1u << 10 | (uint32_t)(n >> 3) << 17 | (uint32_t)(128 >> 4) << 24;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
                 "}\n" ::"r"(tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
                 "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t it = 0; it < WAIT_LIMIT; it++) {
        uint32_t ok;

        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok)
            return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* Teardown after a bounded wait ran out, by the thread that issued every MMA
   of the CTA: a commit to a fresh mbarrier tracks the completion of all the
   thread's earlier tcgen05 operations, whatever phase the working barriers
   were left in, so its arrival proves that no MMA still writes the
   accumulator. Only then may the TMEM be freed. The wait is sixteen times
   the working one; an MMA completes in bounded time once issued, so a drain
   that still runs out means the tensor pipe itself has stopped (bit 2 of
   the fault flag), and the TMEM is freed all the same: a CTA that exits
   holding it would block every later allocation on its SM. */
__device__ __forceinline__ bool drain_mmas(uint32_t bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mma_commit(bar);
    for (int k = 0; k < 16; k++)
        if (mbar_wait(bar, 0))
            return true;
    return false;
}

/* 16 consecutive FP32 columns of this warp's 32 TMEM lanes. */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr));
}

/* Splits 8 FP32 values into BF16 terms and stores each term's 16 bytes;
   term t goes to dst + t * TERM_BYTES. Rounding to nearest: hi = x to 8
   significant bits, mid = the remainder x - hi to 8 bits, lo = what is
   left, at most 8 significant bits, so exact; hi + mid + lo == x for every
   finite x whose rounding to 8 bits stays finite (|x| below 3.39e38).
   The pair conversion (cvt.rn.bf16x2.f32) packs two values at once. */
__device__ __forceinline__ uint32_t bf16x2(float lo_half, float hi_half)
{
    uint32_t d;

    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi_half), "f"(lo_half));
    return d;
}

__device__ __forceinline__ void split_store(const float (&v)[8], unsigned char *dst, int terms)
{
    uint32_t hi[4], mid[4], lo[4];

#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float a = v[2 * k], b = v[2 * k + 1];

        hi[k] = bf16x2(a, b);
        const float ra = a - __uint_as_float(hi[k] << 16);
        const float rb = b - __uint_as_float(hi[k] & 0xffff0000u);

        mid[k] = bf16x2(ra, rb);
        const float la = ra - __uint_as_float(mid[k] << 16);
        const float lb = rb - __uint_as_float(mid[k] & 0xffff0000u);

        lo[k] = bf16x2(la, lb);
    }
    *(uint4 *)dst = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4 *)(dst + TERM_BYTES) = make_uint4(mid[0], mid[1], mid[2], mid[3]);
    if (terms > 2)
        *(uint4 *)(dst + 2 * TERM_BYTES) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

/* Samples of this thread's share of K block kb: candidate t / 16 of the
   block, dates t % 16 + 16 i (16 lanes read one candidate's 128 contiguous
   bytes). Zero outside the strip and the union, and for non-finite values. */
struct Prefetch {
    float2 v[TC_MAX_DATES / 16];
};

__device__ __forceinline__ void prefetch(Prefetch &f, const TcStrip &s, const float2 *slc,
                                         const unsigned short *uyx, int kb, int K, int y0,
                                         int x0, int t)
{
    const int u = kb * KB + (t >> 4), sub = t & 15;
    const float2 *src = nullptr;

    if (u < K) {
        const int c = uyx[u], py = y0 + (c >> 8), px = x0 + (c & 255);

        if (py < s.padded_rows && px < s.W)
            src = slc + ((long long)py * s.W + px) * s.n;
    }
#pragma unroll
    for (int i = 0; i < TC_MAX_DATES / 16; i++) {
        const int d = sub + 16 * i;

        f.v[i] = src && d < s.n ? __ldg(src + d) : make_float2(0.f, 0.f);
    }
}

__device__ __forceinline__ void stage_store(const Prefetch &f, float2 *stage, int n, int t)
{
    const int kk = t >> 4, sub = t & 15;

#pragma unroll
    for (int i = 0; i < TC_MAX_DATES / 16; i++) {
        const int d = sub + 16 * i;

        if (d < n) {
            float2 v = f.v[i];

            if (!isfinite(v.x) || !isfinite(v.y))
                v = make_float2(0.f, 0.f);
            stage[d * STAGE_LD + kk] = v;
        }
    }
}

/* Bounded wait for the MMAs that last read operand buffer b (if any). */
__device__ __forceinline__ bool buffer_free(uint32_t bar0, int b, uint32_t &parity,
                                            uint32_t &pending)
{
    if (!(pending >> b & 1u))
        return true;
    if (!mbar_wait(bar0 + 8 * b, parity >> b & 1u))
        return false;
    parity ^= 1u << b;
    pending &= ~(1u << b);
    return true;
}

__global__ void __launch_bounds__(THREADS, 2)
tc_gram_tc_kernel(TcStrip s, TcChunk c, int terms, const float2 *__restrict__ slc,
                  const uint32_t *__restrict__ mask, float2 *__restrict__ gram)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int n = s.n, npu = tc_npu(n);
    const GramSmem L = gram_smem(n, s.wa, s.wr);
    float2 *stage = (float2 *)(sm + L.stage);
    unsigned short *s_uyx = (unsigned short *)(sm + L.uyx);
    uint32_t *s_rows = (uint32_t *)(sm + L.rows);
    unsigned short *s_pair = (unsigned short *)(sm + L.pair);
    uint2 *s_expand = (uint2 *)(sm + L.expand);
    uint32_t *s_taddr = (uint32_t *)(sm + L.bar + 8 * STAGES);
    const uint32_t bar0 = smem_u32(sm + L.bar);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int UW = TC_TILE_W + s.wr - 1, K = (TC_TILE_H + s.wa - 1) * UW;
    const int nkb = (K + KB - 1) / KB;
    const int nph = (npu + PHASE - 1) / PHASE;
    const int items = c.npix / TC_TILE_PIX * nph;
    const uint32_t wr_mask = (1u << s.wr) - 1u;

    for (int u = t; u < K; u += THREADS) {
        const int uy = u / UW;

        s_uyx[u] = (unsigned short)(uy << 8 | (u - uy * UW));
    }
    for (int q = t; q < npu; q += THREADS) {
        int i = 0, r = q;

        while (r >= n - i) {
            r -= n - i;
            i++;
        }
        s_pair[q] = (unsigned short)(i << 8 | (i + r));
    }
    if (t < 16)
        s_expand[t] = make_uint2((t & 1 ? 0x3f80u : 0u) | (t & 2 ? 0x3f800000u : 0u),
                                 (t & 4 ? 0x3f80u : 0u) | (t & 8 ? 0x3f800000u : 0u));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(s_taddr)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        for (int b = 0; b < STAGES; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0 + 8 * b), "r"(1)
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_taddr;
    uint32_t parity = 0u, pending = 0u; /* bit b: operand buffer b */
    bool ok = true;
    int it = 0; /* K blocks issued by this CTA: block it uses buffer it % 2 */
    /* this thread's A row and B item: pixel / entry t % 128, chunk t / 128 */
    const int m = t & 127, py = m >> 3, px = m & 7, g = t >> 7;
    Prefetch pf;
    int item = blockIdx.x;

    for (; item < items; item += gridDim.x) {
        const int tile = item / nph, P0 = (item - tile * nph) * PHASE;
        const int ty = tile / c.tiles_x, tx = tile - ty * c.tiles_x;
        const int y0 = c.row0 + ty * TC_TILE_H; /* padded row of union row 0 */
        const int x0 = tx * TC_TILE_W;          /* padded column of union column 0 */
        const int np = min(PHASE, npu - P0), h = up16(np);
        const uint32_t lbo_b = 2 * h * 16;
        const uint32_t idesc = instr_desc(2 * h);
        int pi = 0, pj = 0;

        if (m < np) {
            const int pr = s_pair[P0 + m];

            pi = pr >> 8;
            pj = pr & 255;
        }
        prefetch(pf, s, slc, s_uyx, 0, K, y0, x0, t);
        /* SHP bits of window row dy of pixel e % 128 (bit dx), zero for
           pixels outside the output */
        for (int e = t; e < s.wa * TC_TILE_PIX; e += THREADS) {
            const int dy = e >> 7, q = e & 127;
            const int y = y0 + (q >> 3), x = x0 + (q & 7);
            uint32_t f = 0u;

            if (y < c.row0 + c.nrows && y < s.rows && x < s.cols) {
                const int b = dy * s.wr, w = b >> 5, o = b & 31;
                const long long p = (long long)tile * TC_TILE_PIX + q;
                const uint32_t lo = mask[(long long)w * c.npix + p];
                const uint32_t hi = o + s.wr > 32 ? mask[(long long)(w + 1) * c.npix + p] : 0u;

                f = (uint32_t)(((unsigned long long)hi << 32 | lo) >> o) & wr_mask;
            }
            s_rows[e] = f;
        }
        stage_store(pf, stage, n, t);

        for (int kb = 0; kb < nkb; kb++, it++) {
            const int b = it & 1;
            unsigned char *sB = sm + L.ops + b * OP_BYTES, *sA = sB + 3 * TERM_BYTES;

            /* stage holds block kb; fetch block kb + 1 while it is built */
            if (kb + 1 < nkb)
                prefetch(pf, s, slc, s_uyx, kb + 1, K, y0, x0, t);
            if (!buffer_free(bar0, b, parity, pending))
                ok = false;
            if (!__syncthreads_and(ok)) {
                ok = false;
                break;
            }
            /* A: pixel m, candidates u0 .. u0 + 7 -> 16 bytes. The 8
               candidates span at most two union rows (UW >= 8). */
            {
                const int u0 = kb * KB + g * 8;
                uint32_t bits = 0u;

                if (u0 < K) {
                    const int cu = s_uyx[u0], ux = cu & 255, cnt = min(8, UW - ux);
                    int dy = (cu >> 8) - py;

                    if (dy >= 0 && dy < s.wa) {
                        const uint32_t f = s_rows[dy * TC_TILE_PIX + m];
                        const int sh = ux - px;

                        bits = (sh >= 0 ? f >> sh : f << -sh) & ((1u << cnt) - 1u);
                    }
                    dy++;
                    if (cnt < 8 && dy >= 0 && dy < s.wa)
                        bits |= ((s_rows[dy * TC_TILE_PIX + m] << px) & ((1u << (8 - cnt)) - 1u))
                                << cnt;
                }
                const uint2 lo = s_expand[bits & 15u], hi = s_expand[bits >> 4];

                *(uint4 *)(sA + (g * TC_TILE_PIX + m) * 16) = make_uint4(lo.x, lo.y, hi.x, hi.y);
            }
            /* B: entry r = m of the phase, candidates 8g .. 8g + 7; re in row
               r, im in row h + r of each term */
            if (m < h) {
                float re[8], im[8];

                if (m < np) {
                    const float4 *si = (const float4 *)(stage + pi * STAGE_LD + g * 8);
                    const float4 *sj = (const float4 *)(stage + pj * STAGE_LD + g * 8);

#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float4 a = si[k], bb = sj[k];

                        re[2 * k] = fmaf(a.x, bb.x, a.y * bb.y);
                        im[2 * k] = fmaf(a.y, bb.x, -(a.x * bb.y));
                        re[2 * k + 1] = fmaf(a.z, bb.z, a.w * bb.w);
                        im[2 * k + 1] = fmaf(a.w, bb.z, -(a.z * bb.w));
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        re[k] = im[k] = 0.f;
                }
                split_store(re, sB + (g * 2 * h + m) * 16, terms);
                split_store(im, sB + (g * 2 * h + h + m) * 16, terms);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) {
                fence_after();
                const uint64_t adesc = smem_desc(smem_u32(sA), TC_TILE_PIX * 16, 128);

                for (int term = 0; term < terms; term++) {
                    const uint64_t bdesc =
                        smem_desc(smem_u32(sB + term * TERM_BYTES), lbo_b, 128);

                    mma_bf16(tmem, adesc, bdesc, idesc, (kb | term) != 0);
                }
                mma_commit(bar0 + 8 * b);
            }
            pending |= 1u << b;
            /* the B build above was the last reader of stage */
            if (kb + 1 < nkb)
                stage_store(pf, stage, n, t);
        }
        if (!ok)
            break;
        /* every MMA of the phase has completed before TMEM is read */
        for (int bb = 0; bb < STAGES; bb++) {
            const int b = (it + bb) & 1; /* the older block first */

            if (!buffer_free(bar0, b, parity, pending))
                ok = false;
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        fence_after();
        /* epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (pixels), half
           of the phase's 16-entry column groups */
        {
            const int lg = warp & 3;
            const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16);

            /* The warp's 32 pixels x 16 entries go through shared memory
               (the operand buffers, idle until the next item's first
               barrier) so that each store writes two pixels' 16
               consecutive entries: whole 128-byte lines. */
            float2 *stg = (float2 *)(sm + L.ops) + warp * 32 * 17;

            for (int cg = warp >> 2; cg * 16 < np; cg += 2) {
                uint32_t vr[16], vi[16];

                tmem_ld16(lane_addr + cg * 16, vr);
                tmem_ld16(lane_addr + h + cg * 16, vi);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int r = cg * 16 + k, pr = r < np ? s_pair[P0 + r] : 0;

                    stg[lane * 17 + k] =
                        make_float2(__uint_as_float(vr[k]),
                                    (pr >> 8) == (pr & 255) ? 0.f : __uint_as_float(vi[k]));
                }
                __syncwarp();
                const int k = lane & 15, r = cg * 16 + k;

#pragma unroll 4
                for (int q = 0; q < 16; q++) {
                    const int pxl = 2 * q + (lane >> 4);

                    if (r < np)
                        gram[tc_gram_at(npu, (long long)tile * TC_TILE_PIX + lg * 32 + pxl,
                                        P0 + r)] = stg[pxl * 17 + k];
                }
                __syncwarp();
            }
        }
        fence_before();
        /* the next item's first barrier orders these TMEM reads and staging
           loads before its MMAs and operand stores */
        __syncthreads();
    }
    if (!ok) {
        if (t == 0) {
            atomicOr(&g_gram_fault, 1);
            if (!drain_mmas(smem_u32(sm + L.bar + 8 * STAGES + 8)))
                atomicOr(&g_gram_fault, 2);
        }
        __syncthreads();
        /* the items this CTA did not finish: their entries read NaN */
        for (; item < items; item += gridDim.x) {
            const int tile = item / nph, P0 = (item - tile * nph) * PHASE;
            const int np = min(PHASE, npu - P0);

            for (int e = t; e < np * TC_TILE_PIX; e += THREADS)
                gram[tc_gram_at(npu, (long long)tile * TC_TILE_PIX + (e & 127), P0 + (e >> 7))] =
                    make_float2(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000));
        }
    }
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

/* ------------------------------------------------------------------------
 * The transpose: the adjoint's scatter of the Gram gradient onto the
 * candidates (the CUDA-core form is tc_adjoint_scatter_kernel in
 * adjoint.cu). With G_p the Hermitian gradient of pixel p, every candidate
 * u of a tile needs
 *
 *   H_u = sum over the tile's pixels p that took u as an SHP of G_p,
 *   dL/dtheta_u,i += 2 Im(conj(a_u,i) (H_u a_u)_i)
 *
 * and H = A' G is again one GEMM per tile: A'[u][p] = the SHP bit (the
 * forward's A transposed, candidates as M, the 128 pixels as K) and G's
 * columns the real and imaginary parts of G_p,ij for one row i at a time,
 * j = 0 .. J - 1 (J = n rounded up to 16; G_ji = conj(G_ij); the diagonal
 * adds nothing to Im(conj(a_i) G_ii a_i) and is left out). G is split into
 * two truncated BF16 terms (relative error below 2^-16 per value, products
 * with the 0/1 of A' exact). One CTA of 512 threads per tile: thread t owns
 * candidate t (up to 4 blocks of 128, K <= 512), builds its A' row once
 * and keeps its samples in registers; row i's G columns are staged in one
 * of two buffers while the MMAs of row i - 1 run into the other half of
 * TMEM, and the epilogue of row i - 1 forms (H_u a_u)_{i-1} from the
 * accumulator and adds the candidate's dL/dtheta atomically (a candidate
 * lies in the windows of several tiles). Waits are bounded as in the
 * forward kernel; one that runs out sets the same fault flag.
 * ------------------------------------------------------------------------ */
constexpr int ADJ_THREADS = 512;
constexpr int ADJ_MB = 4;                            /* candidate blocks of 128 */
constexpr int ADJ_KCH = TC_TILE_PIX / 8;             /* 16-byte pixel chunks: 16 */
constexpr int ADJ_A_BYTES = ADJ_MB * ADJ_KCH * 128 * 16;   /* 128 KB */
constexpr int ADJ_TERM_BYTES = ADJ_KCH * 64 * 16;    /* 16 chunks x 2J <= 64 rows x 16 B */
constexpr int ADJ_BUF_BYTES = 2 * ADJ_TERM_BYTES;    /* two terms */
constexpr int ADJ_TMEM_COLS = 512;                   /* 2 buffers x 4 blocks x 64 */

struct AdjSmem {
    int a, b, rows, expand, bar, bytes;
};

__host__ __device__ inline AdjSmem adj_smem(int wa)
{
    AdjSmem g;

    g.a = 0;
    g.b = g.a + ADJ_A_BYTES;
    g.rows = g.b + 2 * ADJ_BUF_BYTES;
    g.expand = g.rows + wa * TC_TILE_PIX * 4;
    g.bar = g.expand + 16 * 8;
    g.bytes = g.bar + 32;
    return g;
}

/* 8 FP32 values -> two truncated BF16 terms, 16 bytes each. */
__device__ __forceinline__ void split2_store(const float (&v)[8], unsigned char *dst)
{
    uint32_t hi[4], lo[4];

#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t a = __float_as_uint(v[2 * k]), b = __float_as_uint(v[2 * k + 1]);
        const float ra = v[2 * k] - __uint_as_float(a & 0xffff0000u);
        const float rb = v[2 * k + 1] - __uint_as_float(b & 0xffff0000u);

        hi[k] = __byte_perm(a, b, 0x7632);
        lo[k] = __byte_perm(__float_as_uint(ra), __float_as_uint(rb), 0x7632);
    }
    *(uint4 *)dst = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4 *)(dst + ADJ_TERM_BYTES) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

__global__ void __launch_bounds__(ADJ_THREADS, 1)
tc_gram_adjoint_tc_kernel(TcStrip s, TcChunk c, int halo, const float2 *__restrict__ gbar,
                          const uint32_t *__restrict__ mask, const float2 *__restrict__ slc,
                          float *__restrict__ dtheta)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int n = s.n, J = up16(n), NC = 2 * J;
    const AdjSmem L = adj_smem(s.wa);
    unsigned char *sA = sm + L.a, *sB = sm + L.b;
    uint32_t *s_rows = (uint32_t *)(sm + L.rows);
    uint2 *s_expand = (uint2 *)(sm + L.expand);
    uint32_t *s_taddr = (uint32_t *)(sm + L.bar + 16);
    const uint32_t bar0 = smem_u32(sm + L.bar);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int tile = blockIdx.x;
    const int ty = tile / c.tiles_x, tx = tile - ty * c.tiles_x;
    const int y0 = c.row0 + ty * TC_TILE_H, x0 = tx * TC_TILE_W;
    const int UW = TC_TILE_W + s.wr - 1, K = (TC_TILE_H + s.wa - 1) * UW;
    const int MB = (K + 127) >> 7;
    const uint32_t wr_mask = (1u << s.wr) - 1u;
    const long long pix0 = (long long)tile * TC_TILE_PIX;

    for (int e = t; e < s.wa * TC_TILE_PIX; e += ADJ_THREADS) {
        const int dy = e >> 7, m = e & 127;
        const int y = y0 + (m >> 3), x = x0 + (m & 7);
        uint32_t f = 0u;

        if (y < c.row0 + c.nrows && y < s.rows && x < s.cols) {
            const int b = dy * s.wr, w = b >> 5, o = b & 31;
            const uint32_t lo = mask[(long long)w * c.npix + pix0 + m];
            const uint32_t hi = o + s.wr > 32 ? mask[(long long)(w + 1) * c.npix + pix0 + m] : 0u;

            f = (uint32_t)(((unsigned long long)hi << 32 | lo) >> o) & wr_mask;
        }
        s_rows[e] = f;
    }
    if (t < 16)
        s_expand[t] = make_uint2((t & 1 ? 0x3f80u : 0u) | (t & 2 ? 0x3f800000u : 0u),
                                 (t & 4 ? 0x3f80u : 0u) | (t & 8 ? 0x3f800000u : 0u));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(s_taddr)), "r"(ADJ_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0), "r"(1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0 + 8), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_taddr;

    /* This thread's candidate: its A' row, its samples, its output cell. */
    const int u = t, mb = u >> 7;
    const int uy = u / UW, ux = u - uy * UW;
    const int py = y0 + uy, px = x0 + ux, col = px - halo;
    const bool in_strip = u < K && py < s.padded_rows && px < s.W;
    uint32_t any = 0u;

    if (mb < MB)
        for (int g = 0; g < ADJ_KCH; g++) {
            const int dy = uy - g; /* chunk g = tile row g, pixels 8g .. 8g + 7 */
            uint32_t bits = 0u;

            if (u < K && dy >= 0 && dy < s.wa)
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int dx = ux - k;

                    if (dx >= 0 && dx < s.wr)
                        bits |= ((s_rows[dy * TC_TILE_PIX + g * 8 + k] >> dx) & 1u) << k;
                }
            any |= bits;
            const uint2 lo = s_expand[bits & 15u], hi = s_expand[bits >> 4];

            *(uint4 *)(sA + ((mb * ADJ_KCH + g) * 128 + (u & 127)) * 16) =
                make_uint4(lo.x, lo.y, hi.x, hi.y);
        }
    float2 a[32];

#pragma unroll
    for (int k = 0; k < 32; k++) {
        float2 v = make_float2(0.f, 0.f);

        if (k < n && in_strip && any) {
            v = slc[((long long)py * s.W + px) * n + k];
            if (!isfinite(v.x) || !isfinite(v.y))
                v = make_float2(0.f, 0.f);
        }
        a[k] = v;
    }
    const bool emit = in_strip && any && col >= 0 && col < s.cols;
    const size_t plane = (size_t)s.padded_rows * s.cols;
    float *out = dtheta + (size_t)(emit ? py : 0) * s.cols + (emit ? col : 0);

    /* staging items: J / 8 warps per group of four pixel chunks; a quarter
       warp writes 8 consecutive 16-byte rows (conflict-free) */
    const int jw = J >> 3;
    const int sj = (lane & 7) + 8 * (warp % jw), sg = (lane >> 3) + 4 * (warp / jw);
    const bool stager = sg < ADJ_KCH;
    const uint32_t idesc = instr_desc(NC);
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + mb * 64;
    bool ok = true;

    for (int i = 0; i <= n && ok; i++) {
        const int b = i & 1;

        if (i < n) {
            /* (a) row i of G into buffer b (its last reader, the MMAs of
               row i - 2, completed before the epilogue of row i - 2) */
            if (stager) {
                float re[8], im[8];
                const bool zero = sj == i || sj >= n;

                if (!zero) {
                    const int lo = min(i, sj), hi = max(i, sj);
                    const float sign = sj < i ? -1.f : 1.f;
                    const float4 *src = (const float4 *)(gbar + (long long)tc_pidx(n, lo, hi) *
                                                                    c.npix + pix0 + sg * 8);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float4 v = __ldg(src + k);

                        re[2 * k] = v.x;
                        im[2 * k] = sign * v.y;
                        re[2 * k + 1] = v.z;
                        im[2 * k + 1] = sign * v.w;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        re[k] = im[k] = 0.f;
                }
                unsigned char *dst = sB + b * ADJ_BUF_BYTES + (sg * NC + sj) * 16;

                split2_store(re, dst);
                split2_store(im, dst + J * 16);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            /* (b) the MMAs of row i: M-block m of A' x both terms of G */
            if (t == 0) {
                fence_after();
                for (int m = 0; m < MB; m++)
#pragma unroll
                    for (int ks = 0; ks < ADJ_KCH / 2; ks++) {
                        const uint64_t adesc = smem_desc(
                            smem_u32(sA + (m * ADJ_KCH + 2 * ks) * 128 * 16), 128 * 16, 128);
#pragma unroll
                        for (int term = 0; term < 2; term++) {
                            const uint64_t bdesc = smem_desc(
                                smem_u32(sB + b * ADJ_BUF_BYTES + term * ADJ_TERM_BYTES +
                                         ks * 2 * NC * 16),
                                NC * 16, 128);

                            mma_bf16(tmem + b * 256 + m * 64, adesc, bdesc, idesc,
                                     (ks | term) != 0);
                        }
                    }
                mma_commit(bar0 + 8 * b);
            }
        }
        if (i == 0)
            continue;
        /* (c) epilogue of row r = i - 1 */
        const int r = i - 1, rb = r & 1;

        ok = mbar_wait(bar0 + 8 * rb, (r >> 1) & 1);
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        fence_after();
        if (mb < MB) {
            float2 bsum = make_float2(0.f, 0.f), ar = make_float2(0.f, 0.f);

#pragma unroll
            for (int h = 0; h < 2; h++)
                if (h * 16 < J) {
                    uint32_t vr[16], vi[16];

                    tmem_ld16(lane_addr + rb * 256 + h * 16, vr);
                    tmem_ld16(lane_addr + rb * 256 + J + h * 16, vi);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const float hr = __uint_as_float(vr[k]), hi = __uint_as_float(vi[k]);
                        const float2 aj = a[h * 16 + k];

                        bsum.x = fmaf(hr, aj.x, fmaf(-hi, aj.y, bsum.x));
                        bsum.y = fmaf(hr, aj.y, fmaf(hi, aj.x, bsum.y));
                    }
                }
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k == r)
                    ar = a[k];
            if (emit)
                atomicAdd(out + r * plane, 2.f * (ar.x * bsum.y - ar.y * bsum.x));
        }
        fence_before();
    }
    if (!ok && t == 0) {
        atomicOr(&g_gram_fault, 1);
        if (!drain_mmas(bar0 + 24))
            atomicOr(&g_gram_fault, 2);
    }
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(ADJ_TMEM_COLS) : "memory");
}

} // namespace

bool tc_gram_tensor_supported(int n, int wa, int wr)
{
    int dev = 0, major = 0, minor = 0;

    if (n < 2 || n > TC_MAX_DATES || wa < 1 || wa > MAX_WA || wr < 1 || wr > MAX_WR)
        return false;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return major == 10 && minor == 0;
}

cudaError_t tc_launch_gram_tensor(const TcStrip &s, const TcChunk &c, int split_terms,
                                  const float *slc, const uint32_t *mask, float2 *gram,
                                  cudaStream_t st)
{
    const GramSmem L = gram_smem(s.n, s.wa, s.wr);
    const int bytes = L.bytes < MIN_SMEM ? MIN_SMEM : L.bytes;
    const int items = c.npix / TC_TILE_PIX * ((tc_npu(s.n) + PHASE - 1) / PHASE);
    int dev = 0, sms = 0;
    cudaError_t e;

    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(tc_gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes)) != cudaSuccess)
        return e;
    /* persistent: two CTAs per SM (the TMEM of two accumulators) */
    const int grid = items < 2 * sms ? items : 2 * sms;

    if (grid > 0)
        tc_gram_tc_kernel<<<grid, THREADS, bytes, st>>>(s, c, split_terms < 3 ? 2 : 3,
                                                        (const float2 *)slc, mask, gram);
    return cudaGetLastError();
}

int tc_gram_tensor_fault(void)
{
    int v = 0;

    if (cudaMemcpyFromSymbol(&v, g_gram_fault, sizeof(v)) != cudaSuccess)
        return -1;
    if (v) {
        const int zero = 0;

        cudaMemcpyToSymbol(g_gram_fault, &zero, sizeof(zero));
    }
    return v;
}

bool tc_gram_adjoint_tensor_supported(int n, int wa, int wr)
{
    return n <= 32 && (TC_TILE_H + wa - 1) * (TC_TILE_W + wr - 1) <= ADJ_MB * 128 &&
           tc_gram_tensor_supported(n, wa, wr);
}

cudaError_t tc_launch_adjoint_scatter_tensor(const TcStrip &s, const TcChunk &c, int halo,
                                             const float2 *gbar, const uint32_t *mask,
                                             const float *slc, float *dtheta, cudaStream_t st)
{
    const AdjSmem L = adj_smem(s.wa);
    cudaError_t e;

    if ((e = cudaFuncSetAttribute(tc_gram_adjoint_tc_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, L.bytes)) !=
        cudaSuccess)
        return e;
    tc_gram_adjoint_tc_kernel<<<c.npix / TC_TILE_PIX, ADJ_THREADS, L.bytes, st>>>(
        s, c, halo, gbar, mask, (const float2 *)slc, dtheta);
    return cudaGetLastError();
}
