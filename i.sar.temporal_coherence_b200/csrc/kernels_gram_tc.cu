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
 *   into BF16 terms by truncation: hi = its top 8 significand bits, mid the
 *   next 8, lo the last 8 (hi + mid + lo == the FP32 product, bit for bit).
 *   Each term is one MMA pass into the same FP32 accumulator, so D is an FP32
 *   sum of the exact FP32 products. With two terms the last 8 bits are
 *   dropped: a relative error below 2^-16 per product.
 *
 * Per CTA (256 threads, two CTAs per SM): the packed entries are taken 128 at
 * a time ("phases"); a phase's accumulator is 128 lanes x 2h columns of TMEM
 * (re of entry r in column r, im in column h + r, h = entries rounded up to
 * 16). For each block of 32 candidates the CTA stages their samples in
 * shared memory, builds A and the B terms in the canonical K-major layout
 * without swizzle (8-row x 16-byte core matrices), and one thread issues the
 * MMAs (M = 128, N = 2h, K = 16) and commits them to an mbarrier; the next
 * block's samples load while they run. The epilogue reads the accumulator
 * with tcgen05.ld and writes gram[pidx][p] (float2), the layout the linking
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

constexpr int KB = 32;            /* candidates per K block */
constexpr int KCH = KB / 8;       /* 16-byte K chunks per K block */
constexpr int THREADS = 256;
constexpr int PHASE = 128;        /* packed entries per accumulator phase */
constexpr int TMEM_COLS = 256;    /* 2 x PHASE FP32 columns */
constexpr int STAGE_LD = KB + 2;  /* float2 per date row of the staged samples */
constexpr uint32_t WAIT_LIMIT = 1u << 22;
constexpr int MIN_SMEM = 80 << 10; /* keeps at most two CTAs (512 TMEM columns) per SM */

/* Shared-memory carve-up (byte offsets). */
struct GramSmem {
    int b;       /* 3 terms x KCH chunks x 256 rows x 16 B */
    int a;       /* KCH chunks x 128 rows x 16 B */
    int stage;   /* n x STAGE_LD float2 */
    int mask;    /* mask_words x 128 u32 */
    int pair;    /* npu x u16 */
    int bar;     /* mbarrier (8 B) + TMEM address (4 B) */
    int bytes;
};

constexpr int TERM_BYTES = KCH * 2 * PHASE * 16;

__host__ __device__ inline int up16(int x) { return (x + 15) & ~15; }

__host__ __device__ inline GramSmem gram_smem(int n, int mask_words)
{
    GramSmem g;

    g.b = 0;
    g.a = g.b + 3 * TERM_BYTES;
    g.stage = g.a + KCH * 128 * 16;
    g.mask = g.stage + up16(n * STAGE_LD * 8);
    g.pair = g.mask + up16(mask_words * 128 * 4);
    g.bar = g.pair + up16(tc_npu(n) * 2);
    g.bytes = g.bar + 16;
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

/* Splits 8 FP32 values into truncated BF16 terms and stores each term's 16
   bytes; term t goes to dst + t * TERM_BYTES. */
__device__ __forceinline__ void split_store(const float (&v)[8], unsigned char *dst, int terms)
{
    uint32_t hi[4], mid[4], lo[4];

#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t a = __float_as_uint(v[2 * k]), b = __float_as_uint(v[2 * k + 1]);
        const float ra = v[2 * k] - __uint_as_float(a & 0xffff0000u);
        const float rb = v[2 * k + 1] - __uint_as_float(b & 0xffff0000u);
        const uint32_t ua = __float_as_uint(ra), ub = __float_as_uint(rb);
        const float la = ra - __uint_as_float(ua & 0xffff0000u);
        const float lb = rb - __uint_as_float(ub & 0xffff0000u);

        hi[k] = __byte_perm(a, b, 0x7632);
        mid[k] = __byte_perm(ua, ub, 0x7632);
        lo[k] = __byte_perm(__float_as_uint(la), __float_as_uint(lb), 0x7632);
    }
    *(uint4 *)dst = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *(uint4 *)(dst + TERM_BYTES) = make_uint4(mid[0], mid[1], mid[2], mid[3]);
    if (terms > 2)
        *(uint4 *)(dst + 2 * TERM_BYTES) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

__global__ void __launch_bounds__(THREADS, 2)
tc_gram_tc_kernel(TcStrip s, TcChunk c, int terms, const float2 *__restrict__ slc,
                  const uint32_t *__restrict__ mask, float2 *__restrict__ gram)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int n = s.n, npu = tc_npu(n);
    const GramSmem L = gram_smem(n, s.mask_words);
    unsigned char *sB = sm + L.b, *sA = sm + L.a;
    float2 *stage = (float2 *)(sm + L.stage);
    uint32_t *s_mask = (uint32_t *)(sm + L.mask);
    unsigned short *s_pair = (unsigned short *)(sm + L.pair);
    uint32_t *s_taddr = (uint32_t *)(sm + L.bar + 8);
    const uint32_t bar = smem_u32(sm + L.bar);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int tile = blockIdx.x;
    const int ty = tile / c.tiles_x, tx = tile - ty * c.tiles_x;
    const int y0 = c.row0 + ty * TC_TILE_H; /* padded row of union row 0 */
    const int x0 = tx * TC_TILE_W;          /* padded column of union column 0 */
    const int UW = TC_TILE_W + s.wr - 1, K = (TC_TILE_H + s.wa - 1) * UW;
    const int nkb = (K + KB - 1) / KB;

    /* SHP masks of the tile's pixels; zero for pixels outside the output */
    for (int e = t; e < s.mask_words * TC_TILE_PIX; e += THREADS) {
        const int w = e >> 7, m = e & 127;
        const int y = y0 + (m >> 3), x = x0 + (m & 7);

        s_mask[e] = (y < c.row0 + c.nrows && y < s.rows && x < s.cols)
                        ? mask[(long long)w * c.npix + (long long)tile * TC_TILE_PIX + m]
                        : 0u;
    }
    for (int q = t; q < npu; q += THREADS) {
        int i = 0, r = q;

        while (r >= n - i) {
            r -= n - i;
            i++;
        }
        s_pair[q] = (unsigned short)(i << 8 | (i + r));
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(s_taddr)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_taddr;
    uint32_t parity = 0;
    bool ok = true, pending = false;

    for (int P0 = 0; P0 < npu && ok; P0 += PHASE) {
        const int np = min(PHASE, npu - P0), h = up16(np);
        const uint32_t lbo_b = 2 * h * 16;
        const uint32_t idesc = instr_desc(2 * h);

        for (int kb = 0; kb < nkb; kb++) {
            /* the block's samples, date-major: stage[d * STAGE_LD + kk] */
            for (int e = t; e < KB * n; e += THREADS) {
                const int kk = e / n, d = e - kk * n, u = kb * KB + kk;
                float2 v = make_float2(0.f, 0.f);

                if (u < K) {
                    const int uy = u / UW, py = y0 + uy, px = x0 + (u - uy * UW);

                    if (py < s.padded_rows && px < s.W) {
                        v = __ldg(slc + ((long long)py * s.W + px) * n + d);
                        if (!isfinite(v.x) || !isfinite(v.y))
                            v = make_float2(0.f, 0.f);
                    }
                }
                stage[d * STAGE_LD + kk] = v;
            }
            if (pending) { /* the previous block's MMAs still read A and B */
                ok = mbar_wait(bar, parity);
                if (ok) {
                    parity ^= 1;
                    pending = false;
                }
            }
            if (!__syncthreads_and(ok)) {
                ok = false;
                break;
            }
            /* A: pixel m, candidates 8g .. 8g + 7 of the block -> 16 bytes */
            for (int e = t; e < KCH * TC_TILE_PIX; e += THREADS) {
                const int g = e >> 7, m = e & 127, py = m >> 3, px = m & 7;
                const int u = kb * KB + g * 8;
                int uy = u / UW, ux = u - uy * UW;
                uint32_t wv[4] = {0u, 0u, 0u, 0u};

#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int dy = uy - py, dx = ux - px;

                    if (dy >= 0 && dy < s.wa && dx >= 0 && dx < s.wr) {
                        const int b = dy * s.wr + dx;

                        if ((s_mask[(b >> 5) * TC_TILE_PIX + m] >> (b & 31)) & 1u)
                            wv[k >> 1] |= 0x3f80u << (16 * (k & 1));
                    }
                    if (++ux == UW) {
                        ux = 0;
                        uy++;
                    }
                }
                *(uint4 *)(sA + (g * TC_TILE_PIX + m) * 16) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            }
            /* B: entry r of the phase, candidates 8g .. 8g + 7; re in row r,
               im in row h + r of each term */
            for (int e = t; e < KCH * h; e += THREADS) {
                const int g = e / h, r = e - g * h;
                float re[8], im[8];

                if (r < np) {
                    const int pr = s_pair[P0 + r], i = pr >> 8, j = pr & 255;
                    const float4 *si = (const float4 *)(stage + i * STAGE_LD + g * 8);
                    const float4 *sj = (const float4 *)(stage + j * STAGE_LD + g * 8);

#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float4 a = si[k], b = sj[k];

                        re[2 * k] = fmaf(a.x, b.x, a.y * b.y);
                        im[2 * k] = fmaf(a.y, b.x, -(a.x * b.y));
                        re[2 * k + 1] = fmaf(a.z, b.z, a.w * b.w);
                        im[2 * k + 1] = fmaf(a.w, b.z, -(a.z * b.w));
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        re[k] = im[k] = 0.f;
                }
                split_store(re, sB + (g * 2 * h + r) * 16, terms);
                split_store(im, sB + (g * 2 * h + h + r) * 16, terms);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) {
                fence_after();
#pragma unroll
                for (int ks = 0; ks < KB / 16; ks++) {
                    const uint64_t adesc =
                        smem_desc(smem_u32(sA + ks * 2 * TC_TILE_PIX * 16), TC_TILE_PIX * 16, 128);

                    for (int term = 0; term < terms; term++) {
                        const uint64_t bdesc =
                            smem_desc(smem_u32(sB + term * TERM_BYTES + ks * 2 * lbo_b), lbo_b, 128);

                        mma_bf16(tmem, adesc, bdesc, idesc, (kb | ks | term) != 0);
                    }
                }
                mma_commit(bar);
            }
            pending = true;
        }
        if (!ok)
            break;
        ok = mbar_wait(bar, parity);
        if (ok) {
            parity ^= 1;
            pending = false;
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        fence_after();
        /* epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (pixels), half
           of the phase's 16-entry column groups */
        {
            const int lg = warp & 3, m = lg * 32 + lane;
            const long long p = (long long)tile * TC_TILE_PIX + m;
            const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16);

            for (int cg = warp >> 2; cg * 16 < np; cg += 2) {
                uint32_t vr[16], vi[16];

                tmem_ld16(lane_addr + cg * 16, vr);
                tmem_ld16(lane_addr + h + cg * 16, vi);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int r = cg * 16 + k;

                    if (r < np) {
                        const int q = P0 + r, pr = s_pair[q];

                        gram[(long long)q * c.npix + p] =
                            make_float2(__uint_as_float(vr[k]),
                                        (pr >> 8) == (pr & 255) ? 0.f : __uint_as_float(vi[k]));
                    }
                }
            }
        }
        fence_before();
    }
    if (!ok) {
        if (t == 0)
            atomicOr(&g_gram_fault, 1);
        if (pending)
            mbar_wait(bar, parity);
        for (int e = t; e < npu * TC_TILE_PIX; e += THREADS)
            gram[(long long)(e >> 7) * c.npix + (long long)tile * TC_TILE_PIX + (e & 127)] =
                make_float2(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000));
    }
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

} // namespace

bool tc_gram_tensor_supported(const TcStrip &s)
{
    int dev = 0, major = 0, minor = 0;

    if (s.n < 2 || s.n > TC_MAX_DATES)
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
    const GramSmem L = gram_smem(s.n, s.mask_words);
    const int bytes = L.bytes < MIN_SMEM ? MIN_SMEM : L.bytes;
    cudaError_t e;

    if ((e = cudaFuncSetAttribute(tc_gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes)) != cudaSuccess)
        return e;
    tc_gram_tc_kernel<<<c.npix / TC_TILE_PIX, THREADS, bytes, st>>>(
        s, c, split_terms < 3 ? 2 : 3, (const float2 *)slc, mask, gram);
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
