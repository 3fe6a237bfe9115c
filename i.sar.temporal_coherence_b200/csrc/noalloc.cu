/* The allocation-free entry point, tc_run_device_static.
 *
 * For callers that must not allocate device memory while they run: hosts
 * that manage every device buffer themselves (a fixed memory pool, a GPU
 * shared under a strict budget), code running where cudaMalloc is not
 * allowed or would synchronize (inside a callback, between the launches of
 * a latency-bound loop), or wrappers that cannot own a context object.
 * tc_run_device needs a context from tc_open, which allocates its buffers;
 * this entry point needs none: the caller passes the strip and the outputs
 * (device memory it owns), and every intermediate buffer of the path lives
 * in tc_static_scratch below, a file-scope device array of 64 MiB.
 *
 * That array is held by every GPU that loads this library until the
 * process exits. All calls share it and it keeps the last call's contents;
 * every scratch element is written before it is read within a call, so
 * nothing has to start at zero. Calls that overlap on the GPU (from several
 * host threads, or on streams that do not serialize them) race on it.
 *
 * The strip is processed as a sequence of sub-strips of 16 k output rows,
 * each small enough for the array; a strip whose 16-row sub-strip does not
 * fit (very wide strips with many dates) is rejected with TC_ERR_ARG and a
 * message giving the limit. The coherence matrices use the plain FP32
 * arithmetic (TC_GRAM_FP32); results are those of tc_run_device with that
 * option.
 *
 * Every call looks up the array's device address with cudaGetSymbolAddress
 * on the current device, so that the address stays right when the device's
 * context is destroyed and created again (cudaDeviceReset reloads the
 * library's device code, and the array may move). The first call on a
 * device also loads that device code; make it before any stream capture.
 */
#include "../../include/tcoh_b200.h"
#include "tcoh_internal.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define TC_API extern "C" __attribute__((visibility("default")))

#define TC_STATIC_SCRATCH_BYTES ((size_t)64 << 20)
static __device__ __align__(256) unsigned char tc_static_scratch[TC_STATIC_SCRATCH_BYTES];

/* Device address of tc_static_scratch on the current device. In host code
   the symbol's name is only a host-side stand-in, never a device address. */
static int static_scratch(unsigned char **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, tc_static_scratch);

    if (e != cudaSuccess)
        return tc_error(TC_ERR_CUDA, "cudaGetSymbolAddress of the static scratch: %s",
                        cudaGetErrorString(e));
    *out = (unsigned char *)p;
    return TC_OK;
}

/* The date pairs of the packed upper triangle and of the first npairs pair
   planes (none when npairs is 0: the planes' slot then holds one entry). */
__global__ void tc_static_tables_kernel(int n, int npairs, int pairs_all,
                                        unsigned short *upper, unsigned short *planes)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    int q = 0;

    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++)
            upper[q++] = (unsigned short)(i << 8 | j);
    q = 0;
    for (int i = 0; i < n - 1 && q < npairs; i++)
        for (int j = i + 1; j < (pairs_all ? n : i + 2) && q < npairs; j++)
            planes[q++] = (unsigned short)(i << 8 | j);
}

static size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

/* Scratch bytes for a sub-strip of mr output rows (mr a multiple of 16). */
static size_t substrip_bytes(const struct settings *s, int padded_cols, int cols, int mr,
                             int planes)
{
    const size_t P = (size_t)mr + s->win_az - 1, W = padded_cols;
    const size_t words = (s->win_az * s->win_rg + 31) / 32;
    const size_t npix = (size_t)(mr / TC_TILE_H) * ((cols + TC_TILE_W - 1) / TC_TILE_W) * TC_TILE_PIX;
    size_t b = up256(sizeof(float2) * planes * P * W);

    if (s->test == SHP_TLOG)
        b += up256(sizeof(float2) * P * W);
    b += up256(sizeof(uint32_t) * words * npix);
    b += up256(sizeof(float2) * (size_t)tc_npu(s->ndates) * npix);
    if (s->npairs)
        b += up256(sizeof(float) * (size_t)s->npairs * mr * cols);
    if (s->emi || s->bias) /* the exact tier's queue, one sub-strip's pixels */
        b += up256(tc_exact_queue_bytes((int)words, (long long)npix));
    return b;
}

TC_API int tc_run_device_static(const struct settings *s, int padded_cols, const float *slc,
                                const float *amp, const unsigned char *valid, int padded_rows,
                                int rows, int cols, float *coh, int *count, float *pairs,
                                float *phases, unsigned char *status, void *stream)
{
    int rc;

    if ((rc = tc_check_settings(s, padded_cols)) != TC_OK)
        return rc;
    if (!slc || !amp || !valid || !coh || !count || (s->npairs && !pairs))
        return tc_error(TC_ERR_ARG, "missing strip or output buffer");
    if (rows < 1 || cols < 1 || cols + s->win_rg - 1 != padded_cols ||
        padded_rows != rows + s->win_az - 1)
        return tc_error(TC_ERR_ARG, "strip of %d x %d (padded %d x %d) does not match the "
                        "window %d x %d", rows, cols, padded_rows, padded_cols, s->win_az,
                        s->win_rg);
    const int n = s->ndates;
    const int block = tc_gram_block_for(n);
    const int planes = (n + block - 1) / block * block;
    const size_t fixed = up256(sizeof(unsigned short) * tc_npu(n)) +
                         up256(sizeof(unsigned short) * (s->npairs ? s->npairs : 1));
    int dev = 0, sms = 0;
    cudaError_t e;

    if ((e = cudaGetDevice(&dev)) != cudaSuccess)
        return tc_error(TC_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return tc_error(TC_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
    const size_t link = s->emi ? up256(tc_link_scratch_bytes(n, sms)) : 256;
    const size_t avail = TC_STATIC_SCRATCH_BYTES > fixed + link
                             ? TC_STATIC_SCRATCH_BYTES - fixed - link : 0;
    const int max_mr = (rows + TC_TILE_H - 1) / TC_TILE_H * TC_TILE_H;
    int mr = 0;

    for (int m = TC_TILE_H; m <= max_mr; m += TC_TILE_H) {
        if (substrip_bytes(s, padded_cols, cols, m, planes) > avail)
            break;
        mr = m;
    }
    if (mr == 0)
        return tc_error(TC_ERR_ARG,
                        "tc_run_device_static holds %zu MiB of scratch: %d columns with %d "
                        "dates need %zu bytes for 16 rows; use tc_run_device",
                        TC_STATIC_SCRATCH_BYTES >> 20, cols, n,
                        substrip_bytes(s, padded_cols, cols, TC_TILE_H, planes) + fixed + link);

    unsigned char *base;

    if ((rc = static_scratch(&base)) != TC_OK)
        return rc;
    unsigned short *upper = (unsigned short *)base;
    unsigned short *ptab = (unsigned short *)(base + up256(sizeof(unsigned short) * tc_npu(n)));
    double *lscr = (double *)(base + fixed);
    unsigned char *sub = base + fixed + link;
    cudaStream_t st = (cudaStream_t)stream;

    tc_static_tables_kernel<<<1, 32, 0, st>>>(n, s->npairs, s->pairs_all, upper, ptab);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return tc_error(TC_ERR_CUDA, "table kernel: %s", cudaGetErrorString(e));

    TcShpConst shp;

    shp.test = (int)s->test;
    shp.ks_max = s->ks_max;
    shp.ad_norm = tc_float_literal(s->ad_norm);
    shp.ad_sigma = tc_float_literal(s->ad_sigma);
    shp.ad_crit = tc_float_literal(s->ad_crit);
    shp.tlog_crit = tc_float_literal(s->tlog_crit);
    TcLinkConst lk;

    lk.emi = s->emi;
    lk.bias = s->bias;
    lk.min_looks = s->min_looks;
    lk.npairs = s->npairs;
    lk.pairs_all = s->pairs_all;
    const size_t W = padded_cols;

    for (int r0 = 0; r0 < rows; r0 += mr) {
        const int m = rows - r0 < mr ? rows - r0 : mr;
        TcStrip ss;

        ss.n = n;
        ss.wa = s->win_az;
        ss.wr = s->win_rg;
        ss.area = ss.wa * ss.wr;
        ss.mask_words = (ss.area + 31) / 32;
        ss.W = padded_cols;
        ss.padded_rows = m + ss.wa - 1;
        ss.rows = m;
        ss.cols = cols;
        ss.npad = (long long)ss.padded_rows * padded_cols;
        ss.planes = planes;
        TcChunk c;

        c.row0 = 0;
        c.nrows = m;
        c.tiles_x = (cols + TC_TILE_W - 1) / TC_TILE_W;
        c.tiles_y = (m + TC_TILE_H - 1) / TC_TILE_H;
        c.npix = c.tiles_x * c.tiles_y * TC_TILE_PIX;

        /* carve this sub-strip's buffers */
        unsigned char *q = sub;
        float2 *soa = (float2 *)q;

        q += up256(sizeof(float2) * planes * (size_t)ss.npad);
        float2 *logstat = nullptr;

        if (s->test == SHP_TLOG) {
            logstat = (float2 *)q;
            q += up256(sizeof(float2) * (size_t)ss.npad);
        }
        uint32_t *mask = (uint32_t *)q;

        q += up256(sizeof(uint32_t) * (size_t)ss.mask_words * c.npix);
        float2 *gram = (float2 *)q;

        q += up256(sizeof(float2) * (size_t)tc_npu(n) * c.npix);
        float *spairs = nullptr;

        if (s->npairs) {
            spairs = (float *)q;
            q += up256(sizeof(float) * (size_t)s->npairs * m * cols);
        }
        TcExactQueue eq = {};

        if (tc_link_queues(n, lk)) {
            eq.buf = (int *)q;
            eq.stride = 1 + ss.mask_words;
            eq.capacity = c.npix;
            if ((e = cudaMemsetAsync(eq.buf, 0, sizeof(int) * TC_QUEUE_HEAD, st)) != cudaSuccess)
                return tc_error(TC_ERR_CUDA, "exact-tier queue: %s", cudaGetErrorString(e));
        }

        const float *s_slc = slc + (size_t)r0 * W * n * 2;
        const float *s_amp = amp + (size_t)r0 * W * n;
        const unsigned char *s_valid = valid + (size_t)r0 * W;
        float *s_coh = coh + (size_t)r0 * cols;
        int *s_count = count + (size_t)r0 * cols;

        if ((e = tc_launch_prep(ss, s_slc, soa, st)) != cudaSuccess ||
            (s->test == SHP_TLOG &&
             (e = tc_launch_logstats(ss, s_amp, s_valid, logstat, st)) != cudaSuccess) ||
            (e = tc_launch_shp(ss, c, shp, s_amp, s_valid, logstat, mask, s_count, sms, st)) !=
                cudaSuccess ||
            (tc_link_needs_gram(n, s->emi) &&
             (e = tc_launch_gram_fp32(ss, c, block, soa, mask, gram, st)) != cudaSuccess) ||
            (e = tc_launch_link(ss, c, lk, gram, s_slc, mask, s_count, &eq, upper, ptab, lscr,
                                s_coh, spairs,
                                phases ? phases + (size_t)r0 * cols * n : nullptr,
                                status ? status + (size_t)r0 * cols : nullptr, sms, st)) !=
                cudaSuccess ||
            (eq.buf &&
             (e = tc_flush_exact(ss, lk, &eq, s_slc, s_count, upper, ptab, lscr, s_coh, spairs,
                                 phases ? phases + (size_t)r0 * cols * n : nullptr,
                                 status ? status + (size_t)r0 * cols : nullptr, sms, st)) !=
                 cudaSuccess))
            return tc_error(TC_ERR_CUDA, "sub-strip at row %d: %s", r0, cudaGetErrorString(e));
        if (s->npairs &&
            (e = cudaMemcpy2DAsync(pairs + (size_t)r0 * cols, sizeof(float) * (size_t)rows * cols,
                                   spairs, sizeof(float) * (size_t)m * cols,
                                   sizeof(float) * (size_t)m * cols, s->npairs,
                                   cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return tc_error(TC_ERR_CUDA, "pair planes at row %d: %s", r0, cudaGetErrorString(e));
    }
    return TC_OK;
}
