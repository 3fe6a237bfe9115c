/* Strip preparation and statistically homogeneous pixel (SHP) selection.
 *
 * The SHP tests reproduce the reference kernel's decisions exactly:
 *   KS   (tcoh.cl:34-54)  depends only on comparisons of the sorted float
 *                         amplitudes and the integer KS_MAX;
 *   AD   (tcoh.cl:56-75)  the float rank statistic, accumulated in the same
 *                         order, each term fl(num^2 / den) taken from a
 *                         table of the correctly rounded quotients, and the
 *                         standardization done with round-to-nearest
 *                         intrinsics (no contraction);
 *   tlog (tcoh.cl:77-95)  the float log mean / variance of every pixel,
 *                         computed once per pixel in the kernel's order
 *                         (the reference recomputes them per candidate, with
 *                         identical results), with logs rounded from double
 *                         so that they are the correctly rounded values.
 *
 * Layout of the mask: uint32 [mask_words][npix] per chunk, bit b of word w
 * set when candidate c = 32 w + b (c = dy * WR + dx of the window) is an SHP.
 */
#include "tcoh_internal.h"

#include <math.h>

/* AoS [npad][N] float2 -> SoA [planes][npad] float2, zero planes >= N. */
__global__ void tc_prep_kernel(TcStrip s, const float2 *__restrict__ aos,
                               float2 *__restrict__ soa)
{
    const long long total = (long long)s.planes * s.npad;

    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(i / s.npad);
        const long long p = i - (long long)d * s.npad;

        soa[i] = d < s.n ? aos[p * s.n + d] : make_float2(0.f, 0.f);
    }
}

/* Log mean and variance of every valid pixel's amplitudes, in the float
   order of tcoh.cl:82-90 / 556-564. */
__global__ void tc_logstats_kernel(TcStrip s, const float *__restrict__ amp,
                                   const unsigned char *__restrict__ valid,
                                   float2 *__restrict__ out)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.npad;
         p += (long long)gridDim.x * blockDim.x) {
        const float *a = amp + p * s.n;
        float m = 0.f, v = 0.f;

        if (!valid[p]) {
            out[p] = make_float2(0.f, 0.f);
            continue;
        }
        for (int k = 0; k < s.n; k++)
            m = __fadd_rn(m, (float)log((double)a[k]));
        m = __fdiv_rn(m, (float)s.n);
        for (int k = 0; k < s.n; k++) {
            const float d = __fsub_rn((float)log((double)a[k]), m);

            v = __fadd_rn(v, __fmul_rn(d, d));
        }
        v = __fdiv_rn(v, (float)(s.n - 1));
        out[p] = make_float2(m, v);
    }
}

/* One warp per output pixel; in each round the 32 lanes test 32 window
   candidates against the centre. The centre's sorted amplitudes sit in
   shared memory (every lane reads the same array, so any set of indices is
   conflict-free for N <= 32); each lane's candidate series is transposed
   into a per-warp column buffer b[j][lane], also conflict-free. */
template <int TEST>
__global__ void __launch_bounds__(256)
tc_shp_kernel(TcStrip s, TcChunk c, TcShpConst k, const float *__restrict__ amp,
              const unsigned char *__restrict__ valid, const float2 *__restrict__ logstat,
              uint32_t *__restrict__ mask, int *__restrict__ count, int vec)
{
    extern __shared__ float sm[];
    const int n = s.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int tab_len = TEST == 1 ? (n + 1) * (2 * n - 1) : 0;
    float *tab = sm;
    float *wbuf = sm + tab_len + warp * ((n + 1) + (n + 1) * 32);
    float *a_s = wbuf;          /* n + 1 */
    float *b_s = wbuf + n + 1;  /* (n + 1) x 32 */

    if (TEST == 1) {
        /* fl((2Nm - jN)^2 / (j (2N - j))), j = 1 .. 2N-1, m = 0 .. N. */
        for (int i = threadIdx.x; i < tab_len; i += blockDim.x) {
            const int m = i % (n + 1), j = i / (n + 1) + 1;
            const float num = (float)(2 * n * m - j * n);

            tab[i] = __fdiv_rn(__fmul_rn(num, num), (float)(j * (2 * n - j)));
        }
        __syncthreads();
    }

    for (int p = blockIdx.x * wpb + warp; p < c.npix; p += gridDim.x * wpb) {
        int y, x;

        tc_pixel_yx(c, p, y, x);
        if (y >= c.row0 + c.nrows || y >= s.rows || x >= s.cols)
            continue;
        const long long centre = (long long)(y + s.wa / 2) * s.W + x + s.wr / 2;
        const long long out = (long long)y * s.cols + x;

        if (!valid[centre]) {
            for (int w = lane; w < s.mask_words; w += 32)
                mask[(long long)w * c.npix + p] = 0u;
            if (lane == 0)
                count[out] = -1;
            continue;
        }
        float mean_a = 0.f, var_a = 0.f;

        if (TEST == 2) {
            const float2 st = logstat[centre];

            mean_a = st.x;
            var_a = st.y;
        }
        else {
            for (int j = lane; j < n; j += 32)
                a_s[j] = amp[centre * n + j];
            if (lane == 0)
                a_s[n] = INFINITY;
        }
        __syncwarp();

        int looks = 0;

        for (int w = 0; w < s.mask_words; w++) {
            const int cand = w * 32 + lane;
            bool ok = false;

            if (cand < s.area) {
                const int dy = cand / s.wr, dx = cand - dy * s.wr;
                const long long q = (long long)(y + dy) * s.W + x + dx;

                if (valid[q]) {
                    if (TEST == 2) {
                        /* tcoh.cl:91-94 */
                        const float2 st = logstat[q];
                        const float se = __fsqrt_rn(
                            __fdiv_rn(__fadd_rn(var_a, st.y), (float)n));

                        ok = !(se > 0.f) ||
                             __fdiv_rn(fabsf(__fsub_rn(mean_a, st.x)), se) <= k.tlog_crit;
                    }
                    else {
                        const float *b = amp + q * n;

                        /* the lanes read different pixels: vector loads
                           (vec = 4 or 2 when the series start on 16- or
                           8-byte boundaries, checked on the host) cut the
                           number of scattered requests */
                        if (vec == 4)
                            for (int j = 0; j < n; j += 4) {
                                const float4 v = *(const float4 *)(b + j);

                                b_s[j * 32 + lane] = v.x;
                                b_s[(j + 1) * 32 + lane] = v.y;
                                b_s[(j + 2) * 32 + lane] = v.z;
                                b_s[(j + 3) * 32 + lane] = v.w;
                            }
                        else if (vec == 2)
                            for (int j = 0; j < n; j += 2) {
                                const float2 v = *(const float2 *)(b + j);

                                b_s[j * 32 + lane] = v.x;
                                b_s[(j + 1) * 32 + lane] = v.y;
                            }
                        else
                            for (int j = 0; j < n; j++)
                                b_s[j * 32 + lane] = b[j];
                        b_s[n * 32 + lane] = INFINITY;
                        /* Merge walk, centre first on ties: 2N - 1 steps.
                           Both series end in an INFINITY sentinel, so a
                           side that ran out is never taken without bound
                           checks. The heads of both series stay in
                           registers and each step loads one value, the
                           next one of the side it took (one shared load
                           per step instead of two). */
                        const float *bl = b_s + lane;
                        int ia = 0, ib = 0;
                        float av = a_s[0], bv = bl[0];

                        if (TEST == 0) {
                            int d = 0;

#pragma unroll 4
                            for (int j = 1; j < 2 * n; j++) {
                                const bool ta = av <= bv;

                                ia += ta;
                                ib += !ta;
                                const float v = *(ta ? a_s + ia : bl + ib * 32);

                                av = ta ? v : av;
                                bv = ta ? bv : v;
                                d = max(d, abs(ia - ib));
                            }
                            ok = d <= k.ks_max;
                        }
                        else {
                            float acc = 0.f;
                            const float *tj = tab;

#pragma unroll 4
                            for (int j = 1; j < 2 * n; j++, tj += n + 1) {
                                const bool ta = av <= bv;

                                ia += ta;
                                ib += !ta;
                                const float v = *(ta ? a_s + ia : bl + ib * 32);

                                av = ta ? v : av;
                                bv = ta ? bv : v;
                                acc = __fadd_rn(acc, tj[ia]);
                            }
                            ok = __fdiv_rn(__fsub_rn(__fmul_rn(k.ad_norm, acc), 1.0f),
                                           k.ad_sigma) <= k.ad_crit;
                        }
                    }
                }
            }
            const uint32_t bits = __ballot_sync(0xffffffffu, ok);

            if (lane == 0)
                mask[(long long)w * c.npix + p] = bits;
            looks += __popc(bits);
        }
        if (lane == 0)
            count[out] = looks;
        __syncwarp();
    }
}

cudaError_t tc_launch_prep(const TcStrip &s, const float *slc_aos, float2 *soa,
                           cudaStream_t st)
{
    const long long total = (long long)s.planes * s.npad;
    const int threads = 256;
    const long long blocks = (total + threads - 1) / threads;

    tc_prep_kernel<<<(unsigned)(blocks < 148 * 64 ? blocks : 148 * 64), threads, 0, st>>>(
        s, (const float2 *)slc_aos, soa);
    return cudaGetLastError();
}

cudaError_t tc_launch_logstats(const TcStrip &s, const float *amp,
                               const unsigned char *valid, float2 *logstat,
                               cudaStream_t st)
{
    const int threads = 256;
    const long long blocks = (s.npad + threads - 1) / threads;

    tc_logstats_kernel<<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), threads, 0, st>>>(
        s, amp, valid, logstat);
    return cudaGetLastError();
}

cudaError_t tc_launch_shp(const TcStrip &s, const TcChunk &c, const TcShpConst &k,
                          const float *amp, const unsigned char *valid,
                          const float2 *logstat, uint32_t *mask, int *count, int sms,
                          cudaStream_t st)
{
    const int threads = 256, wpb = threads / 32;
    const int tab = k.test == 1 ? (s.n + 1) * (2 * s.n - 1) : 0;
    const size_t smem = sizeof(float) * (tab + wpb * ((s.n + 1) + (s.n + 1) * 32));
    const int want = (c.npix + wpb - 1) / wpb;
    const int blocks = want < sms * 8 ? want : sms * 8;
    const uintptr_t base = (uintptr_t)amp;
    const int vec = (s.n % 4 == 0 && base % 16 == 0) ? 4 : (s.n % 2 == 0 && base % 8 == 0) ? 2 : 1;
    cudaError_t e;

    switch (k.test) {
    case 0:
        e = cudaFuncSetAttribute(tc_shp_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            tc_shp_kernel<0><<<blocks, threads, smem, st>>>(s, c, k, amp, valid, logstat, mask,
                                                            count, vec);
        break;
    case 1:
        e = cudaFuncSetAttribute(tc_shp_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            tc_shp_kernel<1><<<blocks, threads, smem, st>>>(s, c, k, amp, valid, logstat, mask,
                                                            count, vec);
        break;
    default:
        e = cudaFuncSetAttribute(tc_shp_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            tc_shp_kernel<2><<<blocks, threads, smem, st>>>(s, c, k, amp, valid, logstat, mask,
                                                            count, vec);
        break;
    }
    if (e != cudaSuccess)
        return e;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* SHP selection over a block of chunks, each pair of pixels tested    */
/* once.                                                               */
/* ------------------------------------------------------------------ */

/* Candidate c = dy * WR + dx of pixel p is pixel q = p + (dy - WA/2, dx -
   WR/2), and p is candidate area - 1 - c of q (odd windows). The three
   tests are symmetric in the two series: tlog exactly (a sum and a
   difference of the pair's log statistics); KS and AD whenever the two
   series share no value, since their merged order is then the same
   whichever series goes first on ties, KS's largest |ia - ib| does not
   depend on the order of the two, and AD's term fl((2N m - jN)^2 / (j (2N
   - j))) is the same for the centre's count m and the candidate's j - m
   (the numerators differ only in sign). So the warp of p tests its
   candidates from itself on, and those before it whose pixel lies
   outside the block (whose own warp does not test them); a pair found
   homogeneous sets q's bit for p too, by an atomic OR, after a second,
   reversed walk if the series share a value. */

/* Word w of the mask of output pixel (y, x) of the block. */
__device__ __forceinline__ long long blk_mask_at(const TcStrip &s, const TcShpBlock &b, int y,
                                                 int x, int w)
{
    const int j = (y - b.row0) / b.crows;
    const int r0 = b.row0 + j * b.crows;
    const int nr = min(b.crows, s.rows - r0);
    const int yl = y - r0;
    const long long npix =
        (long long)b.tiles_x * ((nr + TC_TILE_H - 1) / TC_TILE_H) * TC_TILE_PIX;
    const int pl = ((yl / TC_TILE_H) * b.tiles_x + x / TC_TILE_W) * TC_TILE_PIX +
                   (yl % TC_TILE_H) * TC_TILE_W + x % TC_TILE_W;

    return j * b.chunk_words + w * npix + pl;
}

/* KS (TEST 0) or AD (TEST 1) of the centre series a_s against the lane's
   candidate column bl (stride 32), both ending in an INFINITY sentinel:
   the merge walk of tc_shp_kernel. REV: the candidate is the centre (it
   goes first on ties, and AD counts its values). tie: the two series met
   with equal heads. */
template <int TEST, bool REV>
__device__ __forceinline__ bool shp_walk(const float *a_s, const float *bl, int n,
                                         const float *tab, const TcShpConst &k, bool &tie)
{
    int ia = 0, ib = 0;
    float av = a_s[0], bv = bl[0];
    bool eq = false;

    if (TEST == 0) {
        int d = 0;

#pragma unroll 4
        for (int j = 1; j < 2 * n; j++) {
            const bool ta = REV ? av < bv : av <= bv;

            eq |= av == bv;
            ia += ta;
            ib += !ta;
            const float v = *(ta ? a_s + ia : bl + ib * 32);

            av = ta ? v : av;
            bv = ta ? bv : v;
            d = max(d, abs(ia - ib));
        }
        tie = eq;
        return d <= k.ks_max;
    }
    float acc = 0.f;
    const float *tj = tab;

#pragma unroll 4
    for (int j = 1; j < 2 * n; j++, tj += n + 1) {
        const bool ta = REV ? av < bv : av <= bv;

        eq |= av == bv;
        ia += ta;
        ib += !ta;
        const float v = *(ta ? a_s + ia : bl + ib * 32);

        av = ta ? v : av;
        bv = ta ? bv : v;
        acc = __fadd_rn(acc, tj[REV ? ib : ia]);
    }
    tie = eq;
    return __fdiv_rn(__fsub_rn(__fmul_rn(k.ad_norm, acc), 1.0f), k.ad_sigma) <= k.ad_crit;
}

/* One warp per output pixel of the block; the candidates it tests are
   compacted into a per-warp list and taken 32 at a time, one per lane. */
template <int TEST>
__global__ void __launch_bounds__(256)
tc_shp_pair_kernel(TcStrip s, TcShpBlock b, TcShpConst k, const float *__restrict__ amp,
                   const unsigned char *__restrict__ valid, const float2 *__restrict__ logstat,
                   uint32_t *__restrict__ mask, int vec)
{
    extern __shared__ float sm[];
    const int n = s.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int tab_len = TEST == 1 ? (n + 1) * (2 * n - 1) : 0;
    const int per_warp = (n + 1) + (n + 1) * 32 + (s.area + 1) / 2;
    float *tab = sm;
    float *a_s = sm + tab_len + warp * per_warp; /* n + 1 */
    float *b_s = a_s + n + 1;                     /* (n + 1) x 32 */
    unsigned short *list = (unsigned short *)(b_s + (n + 1) * 32);
    const int cc = (s.wa / 2) * s.wr + s.wr / 2; /* the centre's own index */
    const long long npx = (long long)b.nrows * s.cols;

    if (TEST == 1) {
        for (int i = threadIdx.x; i < tab_len; i += blockDim.x) {
            const int m = i % (n + 1), j = i / (n + 1) + 1;
            const float num = (float)(2 * n * m - j * n);

            tab[i] = __fdiv_rn(__fmul_rn(num, num), (float)(j * (2 * n - j)));
        }
        __syncthreads();
    }
    for (long long pix = blockIdx.x * (long long)wpb + warp; pix < npx;
         pix += (long long)gridDim.x * wpb) {
        const int y = b.row0 + (int)(pix / s.cols), x = (int)(pix % s.cols);
        const long long centre = (long long)(y + s.wa / 2) * s.W + x + s.wr / 2;

        if (!valid[centre])
            continue;
        float mean_a = 0.f, var_a = 0.f;

        if (TEST == 2) {
            const float2 st = logstat[centre];

            mean_a = st.x;
            var_a = st.y;
        }
        else {
            for (int j = lane; j < n; j += 32)
                a_s[j] = amp[centre * n + j];
            if (lane == 0)
                a_s[n] = INFINITY;
        }
        int cnt = 0;

        for (int w = 0; w < s.mask_words; w++) {
            const int c = w * 32 + lane;
            bool need = false;

            if (c < s.area) {
                const int dy = c / s.wr, dx = c - dy * s.wr;

                if (valid[(long long)(y + dy) * s.W + x + dx]) {
                    const int yq = y + dy - s.wa / 2, xq = x + dx - s.wr / 2;

                    need = c >= cc ||
                           !(yq >= b.row0 && yq < b.row0 + b.nrows && xq >= 0 && xq < s.cols);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, need);

            if (need)
                list[cnt + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)c;
            cnt += __popc(bal);
        }
        __syncwarp();
        uint32_t own = 0u; /* lane w: word w of this pixel's bits */

        for (int r0 = 0; r0 < cnt; r0 += 32) {
            const int e = r0 + lane;
            const bool act = e < cnt;
            const int c = act ? list[e] : 0;
            const int dy = c / s.wr, dx = c - dy * s.wr;
            const long long q = (long long)(y + dy) * s.W + x + dx;
            bool ok = false, tie = false;

            if (act) {
                if (TEST == 2) {
                    /* tcoh.cl:91-94 */
                    const float2 st = logstat[q];
                    const float se = __fsqrt_rn(__fdiv_rn(__fadd_rn(var_a, st.y), (float)n));

                    ok = !(se > 0.f) ||
                         __fdiv_rn(fabsf(__fsub_rn(mean_a, st.x)), se) <= k.tlog_crit;
                }
                else {
                    const float *bq = amp + q * n;

                    if (vec == 4)
                        for (int j = 0; j < n; j += 4) {
                            const float4 v = *(const float4 *)(bq + j);

                            b_s[j * 32 + lane] = v.x;
                            b_s[(j + 1) * 32 + lane] = v.y;
                            b_s[(j + 2) * 32 + lane] = v.z;
                            b_s[(j + 3) * 32 + lane] = v.w;
                        }
                    else if (vec == 2)
                        for (int j = 0; j < n; j += 2) {
                            const float2 v = *(const float2 *)(bq + j);

                            b_s[j * 32 + lane] = v.x;
                            b_s[(j + 1) * 32 + lane] = v.y;
                        }
                    else
                        for (int j = 0; j < n; j++)
                            b_s[j * 32 + lane] = bq[j];
                    b_s[n * 32 + lane] = INFINITY;
                    ok = shp_walk<TEST == 2 ? 0 : TEST, false>(a_s, b_s + lane, n, tab, k, tie);
                }
            }
            /* this pixel's bits, gathered into lane w for word w */
            const int wlo = list[r0] >> 5, whi = list[min(r0 + 31, cnt - 1)] >> 5;

            for (int w = wlo; w <= whi; w++) {
                const unsigned v =
                    __reduce_or_sync(0xffffffffu, ok && (c >> 5) == w ? 1u << (c & 31) : 0u);

                if (lane == w)
                    own |= v;
            }
            /* q's bit for this pixel, when q is an output pixel of the
               block that does not test the pair itself */
            if (act && c > cc) {
                const int yq = y + dy - s.wa / 2, xq = x + dx - s.wr / 2;

                if (yq < b.row0 + b.nrows && xq >= 0 && xq < s.cols) {
                    bool okr = ok;

                    if (TEST != 2 && tie) {
                        bool t2;

                        okr = shp_walk<TEST == 2 ? 0 : TEST, true>(a_s, b_s + lane, n, tab, k, t2);
                    }
                    if (okr) {
                        const int cr = s.area - 1 - c;

                        atomicOr(&mask[blk_mask_at(s, b, yq, xq, cr >> 5)], 1u << (cr & 31));
                    }
                }
            }
            __syncwarp();
        }
        if (lane < s.mask_words && own)
            atomicOr(&mask[blk_mask_at(s, b, y, x, lane)], own);
        __syncwarp();
    }
}

/* SHP counts of the block's output pixels from their masks; -1 for an
   invalid centre. */
__global__ void tc_shp_count_kernel(TcStrip s, TcShpBlock b, const unsigned char *__restrict__ valid,
                                    const uint32_t *__restrict__ mask, int *__restrict__ count)
{
    const long long npx = (long long)b.nrows * s.cols;

    for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < npx;
         pix += (long long)gridDim.x * blockDim.x) {
        const int y = b.row0 + (int)(pix / s.cols), x = (int)(pix % s.cols);
        int looks = -1;

        if (valid[(long long)(y + s.wa / 2) * s.W + x + s.wr / 2]) {
            looks = 0;
            for (int w = 0; w < s.mask_words; w++)
                looks += __popc(mask[blk_mask_at(s, b, y, x, w)]);
        }
        count[(long long)y * s.cols + x] = looks;
    }
}

cudaError_t tc_launch_shp_block(const TcStrip &s, const TcShpBlock &b, const TcShpConst &k,
                                const float *amp, const unsigned char *valid,
                                const float2 *logstat, uint32_t *mask, int *count, int sms,
                                cudaStream_t st)
{
    const int threads = 256, wpb = threads / 32;
    const int tab = k.test == 1 ? (s.n + 1) * (2 * s.n - 1) : 0;
    const int per_warp = (s.n + 1) + (s.n + 1) * 32 + (s.area + 1) / 2;
    const size_t smem = sizeof(float) * (tab + wpb * per_warp);
    const long long npx = (long long)b.nrows * s.cols;
    const long long want = (npx + wpb - 1) / wpb;
    const int blocks = (int)(want < sms * 8 ? want : sms * 8);
    const uintptr_t base = (uintptr_t)amp;
    const int vec = (s.n % 4 == 0 && base % 16 == 0) ? 4 : (s.n % 2 == 0 && base % 8 == 0) ? 2 : 1;
    cudaError_t e;

    if (npx <= 0)
        return cudaSuccess;
    switch (k.test) {
    case 0:
        e = cudaFuncSetAttribute(tc_shp_pair_kernel<0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            tc_shp_pair_kernel<0><<<blocks, threads, smem, st>>>(s, b, k, amp, valid, logstat,
                                                                 mask, vec);
        break;
    case 1:
        e = cudaFuncSetAttribute(tc_shp_pair_kernel<1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            tc_shp_pair_kernel<1><<<blocks, threads, smem, st>>>(s, b, k, amp, valid, logstat,
                                                                 mask, vec);
        break;
    default:
        e = cudaFuncSetAttribute(tc_shp_pair_kernel<2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            tc_shp_pair_kernel<2><<<blocks, threads, smem, st>>>(s, b, k, amp, valid, logstat,
                                                                 mask, vec);
        break;
    }
    if (e != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
        return e;
    const long long cb = (npx + 255) / 256;

    tc_shp_count_kernel<<<(unsigned)(cb < sms * 16 ? cb : sms * 16), 256, 0, st>>>(s, b, valid,
                                                                                  mask, count);
    return cudaGetLastError();
}
