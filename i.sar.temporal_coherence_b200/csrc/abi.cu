/* C-ABI of the B200 backend: the ocl_* drop-in for ocl.c and the tc_*
 * extensions (include/tcoh_b200.h).
 *
 * A context owns one CUDA stream and device buffers that grow on demand, as
 * ocl.c's ensure_buffer does (ocl.c:265-277). A run processes the padded
 * strip in chunks of output rows (a whole number of 16-row tile rows, all
 * columns), each chunk being three launches on the context's stream:
 * SHP selection -> masked coherence matrices -> phase linking. Chunks
 * bound the intermediate matrices to a few hundred MB and keep every launch
 * far below any watchdog limit, the role of ocl.c's 0.5 s chunks
 * (ocl.c:22-23, 329-363).
 */
#include "../../include/tcoh_b200.h"
#include "tcoh_internal.h"

#include <dlfcn.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#define TC_API extern "C" __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Errors.                                                             */
/* ------------------------------------------------------------------ */

static thread_local char g_error[512];
static void (*g_fatal)(const char *) = nullptr;

static int set_error(int code, const char *fmt, ...)
{
    va_list ap;

    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return set_error(e_ == cudaErrorMemoryAllocation ? TC_ERR_MEMORY         \
                                                              : TC_ERR_CUDA,         \
                             "CUDA error %d (%s) in %s", (int)e_,                    \
                             cudaGetErrorString(e_), #call);                         \
    } while (0)

typedef void (*grass_fatal_fn)(const char *, ...);

/* ocl.c:44-48 reports through G_fatal_error, which never returns. */
static void fatal(const char *what)
{
    char msg[700];

    snprintf(msg, sizeof(msg), "%s: %s", what, g_error);
    if (g_fatal) {
        g_fatal(msg);
    }
    else {
        grass_fatal_fn gf = (grass_fatal_fn)dlsym(RTLD_DEFAULT, "G_fatal_error");

        if (gf)
            gf("%s", msg);
        fprintf(stderr, "ERROR: %s\n", msg);
    }
    exit(EXIT_FAILURE);
}

static void message(const char *fmt, ...)
{
    char msg[512];
    va_list ap;
    grass_fatal_fn gm = (grass_fatal_fn)dlsym(RTLD_DEFAULT, "G_message");

    va_start(ap, fmt);
    vsnprintf(msg, sizeof(msg), fmt, ap);
    va_end(ap);
    if (gm)
        gm("%s", msg);
    else if (getenv("TCOH_VERBOSE"))
        fprintf(stderr, "%s\n", msg);
}

TC_API const char *tc_last_error(void) { return g_error; }

/* For the other translation units of the library. */
int tc_error(int code, const char *fmt, ...)
{
    va_list ap;

    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return code;
}

TC_API void tc_set_fatal_handler(void (*handler)(const char *message)) { g_fatal = handler; }

/* ------------------------------------------------------------------ */
/* SHP constants (stats.c:61-95) and their float literals.             */
/* ------------------------------------------------------------------ */

static const double ad_alpha_tab[7] = {0.25, 0.10, 0.05, 0.025, 0.01, 0.005, 0.001};
static const double ad_crit_tab[7] = {0.325, 1.226, 1.961, 2.718, 3.752, 4.592, 6.546};

/* Standard deviation of the two-sample A2 under the null (Scholz and
   Stephens 1987, eq. 4), samples of sizes na and nb. */
static double ad_sigma_of(int na, int nb)
{
    const int k = 2, total = na + nb;
    const double big_h = 1.0 / na + 1.0 / nb;
    double h = 0.0, g = 0.0;

    if (total <= 3)
        return 1.0;
    for (int j = 1; j < total; j++)
        h += 1.0 / j;
    for (int i = 1; i <= total - 2; i++)
        for (int j = i + 1; j <= total - 1; j++)
            g += 1.0 / ((double)(total - i) * j);
    const double a = (4 * g - 6) * (k - 1) + (10 - 6 * g) * big_h;
    const double b = (2 * g - 4) * k * k + 8 * h * k + (2 * g - 14 * h - 4) * big_h - 8 * h +
                     4 * g - 6;
    const double c = (6 * h + 2 * g - 2) * k * k + (4 * h - 4 * g + 6) * k +
                     (2 * h - 6) * big_h + 4 * h;
    const double d = (2 * h + 6) * k * k - 4 * h * k;
    const double var = (a * pow(total, 3) + b * (double)total * total + c * total + d) /
                       ((total - 1.0) * (total - 2.0) * (total - 3.0));

    return var > 0 ? sqrt(var) : 1.0;
}

/* Two-sided standard normal quantile by bisection on erfc. */
static double normal_quantile(double alpha)
{
    double lo = 0.0, hi = 40.0;

    for (int i = 0; i < 200; i++) {
        const double mid = 0.5 * (lo + hi);

        if (erfc(mid / sqrt(2.0)) > alpha)
            lo = mid;
        else
            hi = mid;
    }
    return 0.5 * (lo + hi);
}

TC_API int tc_shp_constants(struct settings *s)
{
    const int n = s->ndates;

    if (!s || n < 2 || !(s->alpha > 0 && s->alpha < 1))
        return set_error(TC_ERR_ARG, "invalid dates or alpha");
    s->ks_max = (int)floor(sqrt(-0.5 * log(s->alpha / 2.0)) * sqrt(2.0 / n) * n);
    s->ad_norm = 1.0 / (2.0 * n) * (2.0 / n);
    s->ad_sigma = ad_sigma_of(n, n);
    s->ad_crit = 0.0;
    if (s->test == SHP_AD) {
        int i;

        if (s->alpha > ad_alpha_tab[0] || s->alpha < ad_alpha_tab[6])
            return set_error(TC_ERR_ARG,
                             "Anderson-Darling test: alpha must be between %g and %g",
                             ad_alpha_tab[6], ad_alpha_tab[0]);
        for (i = 0; i < 6; i++)
            if (s->alpha >= ad_alpha_tab[i + 1])
                break;
        if (i == 6)
            i = 5;
        const double f = (log(s->alpha) - log(ad_alpha_tab[i])) /
                         (log(ad_alpha_tab[i + 1]) - log(ad_alpha_tab[i]));

        s->ad_crit = ad_crit_tab[i] + f * (ad_crit_tab[i + 1] - ad_crit_tab[i]);
    }
    s->tlog_crit = normal_quantile(s->alpha);
    return TC_OK;
}

/* The float value of a constant written as "%.9ef" into the OpenCL build
   options (ocl.c:222-229). */
static float float_literal(double v)
{
    char buf[64];

    snprintf(buf, sizeof(buf), "%.9e", v);
    return strtof(buf, nullptr);
}

/* ------------------------------------------------------------------ */
/* Context.                                                            */
/* ------------------------------------------------------------------ */

struct DevBuf {
    void *p = nullptr;
    size_t size = 0;
};

static cudaError_t ensure(DevBuf &b, size_t size)
{
    if (b.p && b.size >= size)
        return cudaSuccess;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.size = 0;
    cudaError_t e = cudaMalloc(&b.p, size ? size : 16);

    if (e == cudaSuccess)
        b.size = size;
    return e;
}

enum { ST_PREP, ST_SHP, ST_GRAM, ST_LINK, ST_COPY, ST_ADJOINT, ST_EXACT, ST_COUNT };

/* tc_run_ex copies a strip in this many row blocks on a second stream, and
   each chunk waits only for the blocks holding its rows. */
#define TC_COPY_BLOCKS 32

struct ocl {
    int device;
    int sms;
    int n, wa, wr, test, emi, bias, min_looks, npairs, pairs_all;
    TcShpConst shp;
    int padded_cols;
    tc_options opt;
    int gram_block;
    cudaStream_t stream;
    cudaStream_t copy_stream; /* host -> device copies of tc_run_ex, by row blocks */
    cudaEvent_t block_done[TC_COPY_BLOCKS];
    cudaStream_t out_stream;  /* device -> host copies of the outputs, by chunks */
    std::vector<cudaEvent_t> chunk_done;
    DevBuf slc, amp, valid, coh, count, pairs, phases, status;
    DevBuf soa, logstat, mask, gram, upper_tab, pair_tab, link_scratch, exact_list;
    DevBuf raw_re, raw_im, raw_elev, geo_grid, adj_dh, adj_psi, adj_gbar, adj_dtheta, adj_gdh;
    bool has_geo;
    TcGeo geo;
    bool timing;
    float stage_ms[ST_COUNT];
    int stage_launches[ST_COUNT];
    /* Host-side fault injection for tests of the error paths: with the
       environment variable TCOH_FAIL_AT_CHUNK=k when the context opens,
       every run fails before launching its chunk k (0-based), as a CUDA
       error would, without touching the GPU: tc_run_* return TC_ERR_CUDA
       and ocl_run calls the fatal handler (ocl.c:44-48). -1: off. */
    int fail_chunk;
};

static int check_settings(const struct settings *s, int padded_cols)
{
    if (!s)
        return set_error(TC_ERR_ARG, "no settings");
    if (s->ndates < 2 || s->ndates > TC_MAX_DATES)
        return set_error(TC_ERR_ARG, "%d dates: 2 to %d are supported", s->ndates,
                         TC_MAX_DATES);
    if (s->win_az < 1 || s->win_rg < 1 || !(s->win_az & 1) || !(s->win_rg & 1))
        return set_error(TC_ERR_ARG, "Window sizes must be odd, got %d,%d", s->win_az,
                         s->win_rg);
    if (s->win_az * s->win_rg > 32 * TC_MAX_MASK_WORDS)
        return set_error(TC_ERR_ARG, "window of %d candidates: at most %d are supported",
                         s->win_az * s->win_rg, 32 * TC_MAX_MASK_WORDS);
    if ((int)s->test < 0 || (int)s->test > 2)
        return set_error(TC_ERR_ARG, "unknown SHP test %d", (int)s->test);
    if (s->npairs != 0 &&
        s->npairs != (s->pairs_all ? s->ndates * (s->ndates - 1) / 2 : s->ndates - 1))
        return set_error(TC_ERR_ARG, "%d pair planes for %d dates (%s pairs)", s->npairs,
                         s->ndates, s->pairs_all ? "all" : "consecutive");
    if (padded_cols < s->win_rg)
        return set_error(TC_ERR_ARG, "padded strip of %d columns for a window of %d",
                         padded_cols, s->win_rg);
    return TC_OK;
}

int tc_check_settings(const struct settings *s, int padded_cols)
{
    return check_settings(s, padded_cols);
}

float tc_float_literal(double v) { return float_literal(v); }

TC_API int tc_device_count(void)
{
    int c = 0;

    if (cudaGetDeviceCount(&c) != cudaSuccess)
        return 0;
    return c;
}

TC_API void ocl_list_devices(void)
{
    const int c = tc_device_count();

    fprintf(stdout, "platform|device|type|name|version|compute_units|global_memory_mb\n");
    for (int d = 0; d < c; d++) {
        cudaDeviceProp p;

        if (cudaGetDeviceProperties(&p, d) != cudaSuccess)
            continue;
        fprintf(stdout, "0|%d|GPU|%s|CUDA sm_%d%d|%d|%lu\n", d, p.name, p.major, p.minor,
                p.multiProcessorCount, (unsigned long)(p.totalGlobalMem / (1024 * 1024)));
    }
    fflush(stdout);
}

static void free_bufs(struct ocl *o)
{
    DevBuf *b[] = {&o->slc, &o->amp, &o->valid, &o->coh, &o->count, &o->pairs,
                   &o->phases, &o->status, &o->soa, &o->logstat, &o->mask, &o->gram,
                   &o->upper_tab, &o->pair_tab, &o->link_scratch, &o->exact_list,
                   &o->raw_re, &o->raw_im,
                   &o->raw_elev, &o->geo_grid, &o->adj_dh, &o->adj_psi, &o->adj_gbar,
                   &o->adj_dtheta, &o->adj_gdh};

    for (size_t i = 0; i < sizeof(b) / sizeof(b[0]); i++)
        if (b[i]->p) {
            cudaFree(b[i]->p);
            b[i]->p = nullptr;
            b[i]->size = 0;
        }
}

TC_API int tc_open(int device, const struct settings *s, int padded_cols,
                   const struct tc_options *opt, struct ocl **out, size_t *max_alloc)
{
    int rc, count = 0;

    if (!out)
        return set_error(TC_ERR_ARG, "no output handle");
    *out = nullptr;
    if ((rc = check_settings(s, padded_cols)) != TC_OK)
        return rc;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return set_error(TC_ERR_DEVICE, "No CUDA device found");
    if (device < 0)
        device = 0;
    if (device >= count)
        return set_error(TC_ERR_DEVICE, "CUDA device %d not found (%d devices, see -l)",
                         device, count);
    cudaDeviceProp prop;

    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(TC_ERR_DEVICE,
                         "CUDA device %d (%s, sm_%d%d) is not an sm_100 GPU; this build "
                         "targets sm_100a only",
                         device, prop.name, prop.major, prop.minor);
    CK(cudaSetDevice(device));

    struct ocl *o = new ocl();

    o->device = device;
    o->sms = prop.multiProcessorCount;
    o->n = s->ndates;
    o->wa = s->win_az;
    o->wr = s->win_rg;
    o->test = (int)s->test;
    o->emi = s->emi;
    o->bias = s->bias;
    o->min_looks = s->min_looks;
    o->npairs = s->npairs;
    o->pairs_all = s->pairs_all;
    o->padded_cols = padded_cols;
    o->shp.test = (int)s->test;
    o->shp.ks_max = s->ks_max;
    o->shp.ad_norm = float_literal(s->ad_norm);
    o->shp.ad_sigma = float_literal(s->ad_sigma);
    o->shp.ad_crit = float_literal(s->ad_crit);
    o->shp.tlog_crit = float_literal(s->tlog_crit);
    o->opt.gram = tc_gram_tensor_supported(o->n, o->wa, o->wr) ? TC_GRAM_TENSOR : TC_GRAM_FP32;
    o->opt.split_terms = 3;
    o->opt.chunk_pixels = 0;
    if (opt) {
        const int dflt = o->opt.gram;

        o->opt = *opt;
        if (o->opt.gram < 0)
            o->opt.gram = dflt;
    }
    if (o->opt.split_terms != 2 && o->opt.split_terms != 3)
        o->opt.split_terms = 3;
    if (o->opt.gram != TC_GRAM_FP32 && o->opt.gram != TC_GRAM_TENSOR) {
        delete o;
        return set_error(TC_ERR_ARG, "unknown Gram arithmetic %d", opt->gram);
    }
    if (o->opt.gram == TC_GRAM_TENSOR && !tc_gram_tensor_supported(o->n, o->wa, o->wr)) {
        delete o;
        return set_error(TC_ERR_ARG, "tensor-core Gram not available for %d dates and a %d x %d "
                         "window", s->ndates, s->win_az, s->win_rg);
    }
    o->gram_block = tc_gram_block_for(o->n);
    o->timing = false;
    o->has_geo = false;
    {
        const char *env = getenv("TCOH_FAIL_AT_CHUNK");

        o->fail_chunk = env && *env ? atoi(env) : -1;
    }
    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));

    cudaError_t e = cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking);

    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&o->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&o->out_stream, cudaStreamNonBlocking);
    for (int b = 0; b < TC_COPY_BLOCKS && e == cudaSuccess; b++)
        e = cudaEventCreateWithFlags(&o->block_done[b], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete o;
        return set_error(TC_ERR_CUDA, "stream / event creation: %s", cudaGetErrorString(e));
    }
    /* Date pairs of the packed upper triangle and of the pair planes. */
    {
        const int n = o->n, npu = tc_npu(n);
        unsigned short *up = (unsigned short *)malloc(sizeof(unsigned short) * npu);
        unsigned short *pt = (unsigned short *)malloc(sizeof(unsigned short) * (n * n + 1));
        int q = 0;

        for (int i = 0; i < n; i++)
            for (int j = i; j < n; j++)
                up[q++] = (unsigned short)(i << 8 | j);
        q = 0;
        for (int i = 0; i < n - 1; i++)
            for (int j = i + 1; j < (o->pairs_all ? n : i + 2); j++)
                pt[q++] = (unsigned short)(i << 8 | j);
        e = ensure(o->upper_tab, sizeof(unsigned short) * npu);
        if (e == cudaSuccess)
            e = ensure(o->pair_tab, sizeof(unsigned short) * (q ? q : 1));
        if (e == cudaSuccess)
            e = cudaMemcpy(o->upper_tab.p, up, sizeof(unsigned short) * npu,
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess && q)
            e = cudaMemcpy(o->pair_tab.p, pt, sizeof(unsigned short) * q,
                           cudaMemcpyHostToDevice);
        free(up);
        free(pt);
        if (e != cudaSuccess) {
            free_bufs(o);
            for (int b = 0; b < TC_COPY_BLOCKS; b++)
                cudaEventDestroy(o->block_done[b]);
            cudaStreamDestroy(o->out_stream);
            cudaStreamDestroy(o->copy_stream);
            cudaStreamDestroy(o->stream);
            delete o;
            return set_error(TC_ERR_CUDA, "table upload: %s", cudaGetErrorString(e));
        }
    }
    if (max_alloc) {
        size_t fr = 0, tot = 0;

        cudaMemGetInfo(&fr, &tot);
        /* The strip (slc + amp, 12 N bytes per pixel), the outputs and the
           internal chunk buffers must fit together. */
        *max_alloc = fr / 3;
    }
    message("CUDA device: %s (NVIDIA CUDA, %d SMs)", prop.name, o->sms);
    *out = o;
    return TC_OK;
}

TC_API int tc_close(struct ocl *o)
{
    if (!o)
        return TC_OK;
    cudaSetDevice(o->device);
    cudaStreamSynchronize(o->stream);
    cudaStreamSynchronize(o->copy_stream);
    cudaStreamSynchronize(o->out_stream);
    free_bufs(o);
    for (int b = 0; b < TC_COPY_BLOCKS; b++)
        cudaEventDestroy(o->block_done[b]);
    for (cudaEvent_t ev : o->chunk_done)
        cudaEventDestroy(ev);
    cudaStreamDestroy(o->out_stream);
    cudaStreamDestroy(o->copy_stream);
    cudaStreamDestroy(o->stream);
    delete o;
    return TC_OK;
}

TC_API int tc_get_options(const struct ocl *o, struct tc_options *opt)
{
    if (!o || !opt)
        return set_error(TC_ERR_ARG, "no context or options");
    *opt = o->opt;
    return TC_OK;
}

TC_API int tc_set_timing(struct ocl *o, int on)
{
    if (!o)
        return set_error(TC_ERR_ARG, "no context");
    o->timing = on != 0;
    return TC_OK;
}

TC_API int tc_stage_stats(const struct ocl *o, float *ms, int *launches, int n)
{
    if (!o)
        return 0;
    if (n > ST_COUNT)
        n = ST_COUNT;
    for (int i = 0; i < n; i++) {
        if (ms)
            ms[i] = o->stage_ms[i];
        if (launches)
            launches[i] = o->stage_launches[i];
    }
    return n;
}

/* ------------------------------------------------------------------ */
/* Runs.                                                               */
/* ------------------------------------------------------------------ */

/* Event pairs around launches when timing is on. */
struct Timer {
    struct ocl *o;
    cudaStream_t st;
    cudaEvent_t ev[2 * 1024];
    int stage[1024];
    int used = 0;

    Timer(struct ocl *o_, cudaStream_t s) : o(o_), st(s) {}
    int begin(int stg)
    {
        if (!o->timing || used >= 1024)
            return -1;
        const int i = used++;

        cudaEventCreate(&ev[2 * i]);
        cudaEventCreate(&ev[2 * i + 1]);
        stage[i] = stg;
        cudaEventRecord(ev[2 * i], st);
        return i;
    }
    void end(int i)
    {
        if (i >= 0)
            cudaEventRecord(ev[2 * i + 1], st);
    }
    /* After a synchronize: sum per stage. */
    void collect()
    {
        for (int i = 0; i < used; i++) {
            float ms = 0.f;

            cudaEventSynchronize(ev[2 * i + 1]);
            cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
            o->stage_ms[stage[i]] += ms;
            if (stage[i] != ST_COPY)
                o->stage_launches[stage[i]]++;
            cudaEventDestroy(ev[2 * i]);
            cudaEventDestroy(ev[2 * i + 1]);
        }
        used = 0;
    }
};

static int chunk_rows_for(const struct ocl *o, int rows, int cols)
{
    const int tiles_x = (cols + TC_TILE_W - 1) / TC_TILE_W;
    const long long per_tile_row = (long long)tiles_x * TC_TILE_PIX;
    long long target = o->opt.chunk_pixels;

    if (target <= 0) {
        /* About 256 MB of coherence matrices per chunk. */
        target = (256ll << 20) / ((long long)tc_npu(o->n) * 8);
    }
    long long trows = target / per_tile_row;

    if (trows < 1)
        trows = 1;
    long long r = trows * TC_TILE_H;

    if (r > rows)
        r = (rows + TC_TILE_H - 1) / TC_TILE_H * TC_TILE_H;
    return (int)r;
}

/* The computation on device buffers (asynchronous on st). */
/* The adjoint's per-run state: the Gram-gradient buffer and dL/dtheta. */
struct AdjRun {
    float2 *gbar;
    float *dtheta;
};

/* Padded rows still arriving by blocks: block b (rows b * block_rows ..)
   is complete once block_done[b] has fired. */
struct RowsReady {
    int block_rows, nblocks;
    const cudaEvent_t *done;
};

static int run_device(struct ocl *o, const float *slc, const float *amp,
                      const unsigned char *valid, int padded_rows, int rows, int cols,
                      float *coh, int *count, float *pairs, float *phases,
                      unsigned char *status, cudaStream_t st, Timer &tm,
                      const AdjRun *adj = nullptr, const RowsReady *ready = nullptr,
                      bool mark_chunks = false)
{
    if (rows < 1 || cols < 1)
        return set_error(TC_ERR_ARG, "empty strip (%d x %d)", rows, cols);
    if (cols + o->wr - 1 != o->padded_cols)
        return set_error(TC_ERR_ARG, "%d columns do not match the padded width %d", cols,
                         o->padded_cols);
    if (padded_rows != rows + o->wa - 1)
        return set_error(TC_ERR_ARG, "%d padded rows for %d rows and a %d-line window",
                         padded_rows, rows, o->wa);
    if (o->npairs && !pairs)
        return set_error(TC_ERR_ARG, "no pair buffer for %d pair planes", o->npairs);
    if (o->opt.gram == TC_GRAM_TENSOR && !tc_gram_tensor_supported(o->n, o->wa, o->wr))
        return set_error(TC_ERR_ARG, "tensor-core Gram not available for %d dates and a %d x %d "
                         "window", o->n, o->wa, o->wr);

    TcStrip s;

    s.n = o->n;
    s.wa = o->wa;
    s.wr = o->wr;
    s.area = o->wa * o->wr;
    s.mask_words = (s.area + 31) / 32;
    s.W = o->padded_cols;
    s.padded_rows = padded_rows;
    s.rows = rows;
    s.cols = cols;
    s.npad = (long long)padded_rows * o->padded_cols;
    s.planes = (o->n + o->gram_block - 1) / o->gram_block * o->gram_block;

    const int crows = chunk_rows_for(o, rows, cols);
    const int tiles_x = (cols + TC_TILE_W - 1) / TC_TILE_W;
    const long long max_npix = (long long)(crows / TC_TILE_H) * tiles_x * TC_TILE_PIX;

    /* SHP masks are selected for blocks of up to 16 chunks at once (each
       pair of the block's pixels tested once): about 64 MB of masks */
    const long long chunk_words = (long long)s.mask_words * max_npix;
    long long shp_chunks = (64ll << 20) / (4 * chunk_words);

    if (shp_chunks > 16)
        shp_chunks = 16;
    if (shp_chunks < 1)
        shp_chunks = 1;
    CK(ensure(o->mask, sizeof(uint32_t) * chunk_words * shp_chunks));
    CK(ensure(o->gram, sizeof(float2) * tc_npu(o->n) * max_npix));
    CK(ensure(o->link_scratch, tc_link_scratch_bytes(o->n, o->sms)));
    TcLinkConst lk;

    lk.emi = o->emi;
    lk.bias = o->bias;
    lk.min_looks = o->min_looks;
    lk.npairs = o->npairs;
    lk.pairs_all = o->pairs_all;
    /* the exact tier's queue: about 32 MB, at least one chunk, at most 16
       chunks (a flush is one launch over the queued pixels of its chunks) */
    TcExactQueue q = {};

    if (!adj && tc_link_queues(o->n, lk)) {
        const long long entry = 4ll * (1 + s.mask_words);
        long long cap = (32ll << 20) / entry;

        if (cap > 16 * max_npix)
            cap = 16 * max_npix;
        if (cap < max_npix)
            cap = max_npix;
        CK(ensure(o->exact_list, tc_exact_queue_bytes(s.mask_words, cap)));
        q.buf = (int *)o->exact_list.p;
        q.stride = 1 + s.mask_words;
        q.capacity = cap;
        CK(cudaMemsetAsync(q.buf, 0, sizeof(int) * TC_QUEUE_HEAD, st));
    }
    if (o->opt.gram == TC_GRAM_FP32)
        CK(ensure(o->soa, sizeof(float2) * s.planes * s.npad));
    if (o->test == SHP_TLOG)
        CK(ensure(o->logstat, sizeof(float2) * s.npad));

    int t;

    /* the date-plane transpose and the log statistics read the whole strip */
    if (ready && (o->opt.gram == TC_GRAM_FP32 || o->test == SHP_TLOG))
        CK(cudaStreamWaitEvent(st, ready->done[ready->nblocks - 1], 0));
    if (o->opt.gram == TC_GRAM_FP32) {
        t = tm.begin(ST_PREP);
        CK(tc_launch_prep(s, slc, (float2 *)o->soa.p, st));
        tm.end(t);
    }
    if (o->test == SHP_TLOG) {
        t = tm.begin(ST_PREP);
        CK(tc_launch_logstats(s, amp, valid, (float2 *)o->logstat.p, st));
        tm.end(t);
    }
    if (mark_chunks) {
        const size_t nchunks = (size_t)((rows + crows - 1) / crows);

        while (o->chunk_done.size() < nchunks) {
            cudaEvent_t ev;

            CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            o->chunk_done.push_back(ev);
        }
    }
    /* chunks whose outputs the queued exact-tier pixels may still change:
       their completion events follow the flush */
    int unflushed = 0;
    auto flush = [&](int upto) -> int {
        if (q.buf) {
            const int tf = q.pending > 0 ? tm.begin(ST_EXACT) : -1;

            CK(tc_flush_exact(s, lk, &q, slc, count, (const unsigned short *)o->upper_tab.p,
                              (const unsigned short *)o->pair_tab.p,
                              (double *)o->link_scratch.p, coh, pairs, phases, status, o->sms,
                              st));
            tm.end(tf);
        }
        if (mark_chunks)
            for (; unflushed < upto; unflushed++)
                CK(cudaEventRecord(o->chunk_done[unflushed], st));
        unflushed = upto;
        return TC_OK;
    };

    for (int row0 = 0, chunk = 0; row0 < rows; row0 += crows, chunk++) {
        TcChunk c;

        if (chunk == o->fail_chunk)
            return set_error(TC_ERR_CUDA, "injected failure before chunk %d "
                             "(TCOH_FAIL_AT_CHUNK)", chunk);

        c.row0 = row0;
        c.nrows = rows - row0 < crows ? rows - row0 : crows;
        c.tiles_x = tiles_x;
        c.tiles_y = (c.nrows + TC_TILE_H - 1) / TC_TILE_H;
        c.npix = c.tiles_x * c.tiles_y * TC_TILE_PIX;
        if (ready) {
            const int last = row0 + c.nrows + o->wa - 2; /* last padded row read */
            int b = last / ready->block_rows;

            if (b >= ready->nblocks)
                b = ready->nblocks - 1;
            CK(cudaStreamWaitEvent(st, ready->done[b], 0));
        }

        if (chunk % shp_chunks == 0) {
            TcShpBlock b;

            b.row0 = row0;
            b.nrows = rows - row0 < shp_chunks * crows ? rows - row0 : (int)(shp_chunks * crows);
            b.crows = crows;
            b.tiles_x = tiles_x;
            b.chunk_words = chunk_words;
            if (ready) {
                const int last = row0 + b.nrows + o->wa - 2;
                int rb = last / ready->block_rows;

                if (rb >= ready->nblocks)
                    rb = ready->nblocks - 1;
                CK(cudaStreamWaitEvent(st, ready->done[rb], 0));
            }
            t = tm.begin(ST_SHP);
            CK(cudaMemsetAsync(o->mask.p, 0,
                               sizeof(uint32_t) * chunk_words *
                                   ((b.nrows + crows - 1) / crows), st));
            CK(tc_launch_shp_block(s, b, o->shp, amp, valid, (const float2 *)o->logstat.p,
                                   (uint32_t *)o->mask.p, count, o->sms, st));
            tm.end(t);
        }
        /* this chunk's masks in the block's region */
        const uint32_t *cmask = (const uint32_t *)o->mask.p + (chunk % shp_chunks) * chunk_words;

        if (adj || tc_link_needs_gram(o->n, o->emi)) {
            t = tm.begin(ST_GRAM);
            if (o->opt.gram == TC_GRAM_FP32)
                CK(tc_launch_gram_fp32(s, c, o->gram_block, (const float2 *)o->soa.p,
                                       cmask, (float2 *)o->gram.p, st));
            else
                CK(tc_launch_gram_tensor(s, c, o->opt.split_terms, slc,
                                         cmask, (float2 *)o->gram.p, st));
            tm.end(t);
        }
        if (q.buf && q.pending + c.npix > q.capacity) {
            const int rc = flush(chunk);

            if (rc != TC_OK)
                return rc;
        }
        t = tm.begin(ST_LINK);
        if (!adj)
            CK(tc_launch_link(s, c, lk, (const float2 *)o->gram.p, slc,
                              cmask, count, &q,
                              (const unsigned short *)o->upper_tab.p,
                              (const unsigned short *)o->pair_tab.p,
                              (double *)o->link_scratch.p, coh, pairs, phases, status, o->sms,
                              st));
        else {
            CK(tc_launch_link_adjoint(s, c, lk, (const float2 *)o->gram.p, count,
                                      (const unsigned short *)o->upper_tab.p,
                                      (const unsigned short *)o->pair_tab.p,
                                      (double *)o->link_scratch.p, coh, pairs, adj->gbar,
                                      o->sms, st));
            tm.end(t);
            t = tm.begin(ST_ADJOINT);
            if (o->opt.gram == TC_GRAM_TENSOR && tc_gram_adjoint_tensor_supported(o->n, o->wa, o->wr))
                CK(tc_launch_adjoint_scatter_tensor(s, c, o->wr / 2, adj->gbar,
                                                    cmask, slc, adj->dtheta,
                                                    st));
            else
                CK(tc_launch_adjoint_scatter(s, c, o->wr / 2, adj->gbar,
                                             cmask, slc, adj->dtheta, st));
        }
        tm.end(t);
        if (!q.buf) {
            const int rc = flush(chunk + 1);

            if (rc != TC_OK)
                return rc;
        }
    }
    return flush((rows + crows - 1) / crows);
}

TC_API int tc_run_device(struct ocl *o, const float *slc, const float *amp,
                         const unsigned char *valid, int padded_rows, int rows, int cols,
                         float *coh, int *count, float *pairs, float *phases,
                         unsigned char *status, void *stream)
{
    if (!o)
        return set_error(TC_ERR_ARG, "no context");
    CK(cudaSetDevice(o->device));
    cudaStream_t st = (cudaStream_t)stream;
    Timer tm(o, st);

    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));
    int rc = run_device(o, slc, amp, valid, padded_rows, rows, cols, coh, count, pairs,
                        phases, status, st, tm);

    if (o->timing) {
        cudaStreamSynchronize(st);
        tm.collect();
    }
    return rc;
}

/* Device output buffers of the context for a strip of nout pixels. */
static int ensure_outputs(struct ocl *o, size_t nout, bool phases, bool status)
{
    CK(ensure(o->coh, nout * sizeof(float)));
    CK(ensure(o->count, nout * sizeof(int)));
    if (o->npairs)
        CK(ensure(o->pairs, o->npairs * nout * sizeof(float)));
    if (phases)
        CK(ensure(o->phases, nout * o->n * sizeof(float)));
    if (status)
        CK(ensure(o->status, nout));
    return TC_OK;
}

/* The outputs of a run on the context's buffers back to the host, chunk
   by chunk on the output stream as each chunk's kernels complete: all the
   strip's kernels are queued first, so the GPU keeps computing even where
   the host buffers are pageable and a copy holds the calling thread. */
static int stream_outputs(struct ocl *o, int rows, int cols, float *coh, int *count,
                          float *pairs, float *phases, unsigned char *status)
{
    const int crows = chunk_rows_for(o, rows, cols);
    const size_t plane = (size_t)rows * cols;
    cudaStream_t os = o->out_stream;

    for (int row0 = 0; row0 < rows; row0 += crows) {
        const int nr = rows - row0 < crows ? rows - row0 : crows;
        const size_t at = (size_t)row0 * cols, np_ = (size_t)nr * cols;

        CK(cudaStreamWaitEvent(os, o->chunk_done[row0 / crows], 0));
        CK(cudaMemcpyAsync(coh + at, (float *)o->coh.p + at, np_ * sizeof(float),
                           cudaMemcpyDeviceToHost, os));
        CK(cudaMemcpyAsync(count + at, (int *)o->count.p + at, np_ * sizeof(int),
                           cudaMemcpyDeviceToHost, os));
        if (o->npairs && pairs)
            CK(cudaMemcpy2DAsync(pairs + at, plane * sizeof(float), (float *)o->pairs.p + at,
                                 plane * sizeof(float), np_ * sizeof(float), o->npairs,
                                 cudaMemcpyDeviceToHost, os));
        if (phases)
            CK(cudaMemcpyAsync(phases + at * o->n, (float *)o->phases.p + at * o->n,
                               np_ * o->n * sizeof(float), cudaMemcpyDeviceToHost, os));
        if (status)
            CK(cudaMemcpyAsync(status + at, (unsigned char *)o->status.p + at, np_,
                               cudaMemcpyDeviceToHost, os));
    }
    return TC_OK;
}

static int finish_run(struct ocl *o, Timer &tm)
{
    CK(cudaStreamSynchronize(o->stream));
    CK(cudaStreamSynchronize(o->out_stream));
    tm.collect();
    if (o->opt.gram == TC_GRAM_TENSOR && tc_gram_tensor_fault() > 0)
        return set_error(TC_ERR_DEVICE, "tensor-core Gram: a wait for MMA completion ran out; "
                         "the tiles concerned are NULL");
    return TC_OK;
}

static int run_context_buffers(struct ocl *o, int padded_rows, int rows, int cols, float *coh,
                               int *count, float *pairs, float *phases, unsigned char *status,
                               Timer &tm, const RowsReady *ready = nullptr)
{
    int rc = run_device(o, (const float *)o->slc.p, (const float *)o->amp.p,
                        (const unsigned char *)o->valid.p, padded_rows, rows, cols,
                        (float *)o->coh.p, (int *)o->count.p,
                        o->npairs ? (float *)o->pairs.p : nullptr,
                        phases ? (float *)o->phases.p : nullptr,
                        status ? (unsigned char *)o->status.p : nullptr, o->stream, tm, nullptr,
                        ready, true);

    if (rc == TC_OK)
        rc = stream_outputs(o, rows, cols, coh, count, pairs, phases, status);
    if (rc != TC_OK) {
        cudaStreamSynchronize(o->copy_stream);
        cudaStreamSynchronize(o->out_stream);
        cudaStreamSynchronize(o->stream);
        tm.collect();
        return rc;
    }
    return finish_run(o, tm);
}

TC_API int tc_run_ex(struct ocl *o, const float *slc, const float *amp,
                     const unsigned char *valid, int padded_rows, int rows, int cols,
                     float *coh, int *count, float *pairs, float *phases,
                     unsigned char *status)
{
    if (!o)
        return set_error(TC_ERR_ARG, "no context");
    if (!slc || !amp || !valid || !coh || !count)
        return set_error(TC_ERR_ARG, "missing strip or output buffer");
    if (rows < 1 || cols < 1 || padded_rows != rows + o->wa - 1 ||
        cols + o->wr - 1 != o->padded_cols)
        return set_error(TC_ERR_ARG, "strip of %d x %d (padded %d x %d) does not match "
                         "the window %d x %d",
                         rows, cols, padded_rows, o->padded_cols, o->wa, o->wr);
    CK(cudaSetDevice(o->device));
    const size_t npad = (size_t)padded_rows * o->padded_cols;
    const size_t n = o->n;
    cudaStream_t st = o->stream;
    Timer tm(o, st);

    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));
    CK(ensure(o->slc, npad * n * 2 * sizeof(float)));
    CK(ensure(o->amp, npad * n * sizeof(float)));
    CK(ensure(o->valid, npad));
    int rc = ensure_outputs(o, (size_t)rows * cols, phases != nullptr, status != nullptr);

    if (rc != TC_OK)
        return rc;
    /* the strip goes over in row blocks on the copy stream; each chunk
       waits for the blocks that hold its rows */
    const size_t W = o->padded_cols;
    const int block_rows = (padded_rows + TC_COPY_BLOCKS - 1) / TC_COPY_BLOCKS;
    RowsReady ready;

    ready.block_rows = block_rows;
    ready.nblocks = (padded_rows + block_rows - 1) / block_rows;
    ready.done = o->block_done;
    /* work already queued on the context's stream may still read the strip
       buffers (a wait captures the event as recorded at the call) */
    CK(cudaEventRecord(o->block_done[0], st));
    CK(cudaStreamWaitEvent(o->copy_stream, o->block_done[0], 0));
    for (int b = 0; b < ready.nblocks; b++) {
        const size_t r0 = (size_t)b * block_rows;
        const size_t nr = (size_t)(b + 1 < ready.nblocks ? block_rows : padded_rows - r0);
        const size_t px = r0 * W, np_ = nr * W;

        CK(cudaMemcpyAsync((float *)o->slc.p + px * n * 2, slc + px * n * 2,
                           np_ * n * 2 * sizeof(float), cudaMemcpyHostToDevice, o->copy_stream));
        CK(cudaMemcpyAsync((float *)o->amp.p + px * n, amp + px * n, np_ * n * sizeof(float),
                           cudaMemcpyHostToDevice, o->copy_stream));
        CK(cudaMemcpyAsync((unsigned char *)o->valid.p + px, valid + px, np_,
                           cudaMemcpyHostToDevice, o->copy_stream));
        CK(cudaEventRecord(o->block_done[b], o->copy_stream));
    }
    return run_context_buffers(o, padded_rows, rows, cols, coh, count, pairs, phases, status,
                               tm, &ready);
}

/* ------------------------------------------------------------------ */
/* Geometry and raw strips.                                            */
/* ------------------------------------------------------------------ */

TC_API int tc_geometry_grid_shape(const struct tc_geometry *g, int *grid_rows, int *grid_cols,
                                  int *nheights, double *heights)
{
    TcGeo d;
    int rc;

    if (!g)
        return set_error(TC_ERR_ARG, "no geometry");
    if ((rc = tc_geometry_shape(*g, d)) != TC_OK)
        return rc;
    if (grid_rows)
        *grid_rows = d.grid_rows;
    if (grid_cols)
        *grid_cols = d.grid_cols;
    if (nheights)
        *nheights = d.nheights;
    if (heights)
        for (int i = 0; i < 3; i++)
            heights[i] = d.heights[i];
    return TC_OK;
}

TC_API int tc_geometry_init(const struct tc_geometry *g, const struct tc_orbit *orbits,
                            double *grid)
{
    TcGeo d;
    int rc;
    cudaStream_t st;

    if (!g || !orbits || !grid)
        return set_error(TC_ERR_ARG, "no geometry, orbits or grid");
    if ((rc = tc_geometry_shape(*g, d)) != TC_OK)
        return rc;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    rc = tc_geometry_grid(d, orbits, grid, st);
    cudaStreamDestroy(st);
    return rc;
}

TC_API int tc_set_geometry(struct ocl *o, const struct tc_geometry *g, const double *grid)
{
    if (!o)
        return set_error(TC_ERR_ARG, "no context");
    if (!g || !grid) {
        o->has_geo = false;
        return TC_OK;
    }
    TcGeo d;
    int rc;

    if ((rc = tc_geometry_shape(*g, d)) != TC_OK)
        return rc;
    if (d.ndates != o->n)
        return set_error(TC_ERR_ARG, "geometry of %d dates for a context of %d", d.ndates, o->n);
    const size_t nodes = (size_t)d.grid_rows * d.grid_cols * d.ndates;
    const size_t bytes = nodes * d.nheights * sizeof(double);
    DevBuf raw;

    /* the grid as given, then its coefficient form (TcGridCell) */
    CK(cudaSetDevice(o->device));
    CK(ensure(o->geo_grid, nodes * 3 * sizeof(double)));
    CK(ensure(raw, bytes));
    cudaError_t e = cudaMemcpyAsync(raw.p, grid, bytes, cudaMemcpyHostToDevice, o->stream);

    if (e == cudaSuccess)
        e = tc_launch_geometry_coef(d, (const double *)raw.p, (double *)o->geo_grid.p, o->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(o->stream);
    cudaFree(raw.p);
    CK(e);
    o->geo = d;
    o->has_geo = true;
    return TC_OK;
}

static int check_raw(struct ocl *o, const float *re, const float *im, int region_rows,
                     int padded_rows, int rows, int cols, const float *coh, const int *count)
{
    if (!o)
        return set_error(TC_ERR_ARG, "no context");
    if (!re || !im || !coh || !count)
        return set_error(TC_ERR_ARG, "missing raw rows or output buffer");
    if (rows < 1 || cols < 1 || region_rows < 1 || padded_rows != rows + o->wa - 1 ||
        cols + o->wr - 1 != o->padded_cols)
        return set_error(TC_ERR_ARG, "raw strip of %d x %d (padded %d rows, %d columns) does "
                         "not match the window %d x %d", rows, cols, padded_rows,
                         o->padded_cols, o->wa, o->wr);
    if (o->has_geo && (cols > (o->geo.grid_cols - 1) * 16 ||
                       region_rows > (o->geo.grid_rows - 1) * 16))
        return set_error(TC_ERR_ARG, "region of %d rows x %d columns beyond the geometry grid",
                         region_rows, cols);
    return TC_OK;
}

static int prepare_raw(struct ocl *o, const float *re, const float *im, const double *elev,
                       int row0, int region_rows, int padded_rows, int cols, cudaStream_t st,
                       Timer &tm, const double *dh = nullptr, const float *psi = nullptr)
{
    const size_t npad = (size_t)padded_rows * o->padded_cols;
    const size_t n = o->n;

    CK(ensure(o->slc, npad * n * 2 * sizeof(float)));
    CK(ensure(o->amp, npad * n * sizeof(float)));
    CK(ensure(o->valid, npad));
    const int t = tm.begin(ST_PREP);

    CK(tc_launch_prep_raw(o->n, re, im, elev, row0, region_rows, padded_rows, cols, o->wr / 2,
                          0, padded_rows, o->has_geo ? &o->geo : nullptr,
                          (const double *)o->geo_grid.p, dh, psi,
                          (float *)o->slc.p, (float *)o->amp.p, (unsigned char *)o->valid.p,
                          st));
    tm.end(t);
    return TC_OK;
}

TC_API int tc_run_raw(struct ocl *o, const float *re, const float *im, const double *elevation,
                      int row0, int region_rows, int padded_rows, int rows, int cols,
                      float *coh, int *count, float *pairs, float *phases,
                      unsigned char *status)
{
    int rc;

    if ((rc = check_raw(o, re, im, region_rows, padded_rows, rows, cols, coh, count)) != TC_OK)
        return rc;
    CK(cudaSetDevice(o->device));
    const size_t plane = (size_t)padded_rows * cols;
    const size_t n = o->n;
    const size_t npad = (size_t)padded_rows * o->padded_cols;
    cudaStream_t st = o->stream, cs = o->copy_stream;
    Timer tm(o, st);

    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));
    CK(ensure(o->raw_re, n * plane * sizeof(float)));
    CK(ensure(o->raw_im, n * plane * sizeof(float)));
    if (elevation)
        CK(ensure(o->raw_elev, plane * sizeof(double)));
    CK(ensure(o->slc, npad * n * 2 * sizeof(float)));
    CK(ensure(o->amp, npad * n * sizeof(float)));
    CK(ensure(o->valid, npad));
    if ((rc = ensure_outputs(o, (size_t)rows * cols, phases != nullptr, status != nullptr)) !=
        TC_OK)
        return rc;
    /* The raw rows go over in row blocks on the copy stream (one strided
       copy per block for all the date planes), each block prepared there
       as soon as its rows have arrived, and each chunk of the path waits
       only for the blocks that hold its rows: the copies and the
       preparation overlap the path (and are not timed as stages here). */
    const int block_rows = (padded_rows + TC_COPY_BLOCKS - 1) / TC_COPY_BLOCKS;
    RowsReady ready;

    ready.block_rows = block_rows;
    ready.nblocks = (padded_rows + block_rows - 1) / block_rows;
    ready.done = o->block_done;
    /* work already queued on the context's stream may still read the
       buffers */
    CK(cudaEventRecord(o->block_done[0], st));
    CK(cudaStreamWaitEvent(cs, o->block_done[0], 0));
    for (int b = 0; b < ready.nblocks; b++) {
        const int r0 = b * block_rows;
        const int nr = b + 1 < ready.nblocks ? block_rows : padded_rows - r0;
        const size_t at = (size_t)r0 * cols, bytes = (size_t)nr * cols * sizeof(float);

        CK(cudaMemcpy2DAsync((float *)o->raw_re.p + at, plane * sizeof(float), re + at,
                             plane * sizeof(float), bytes, n, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpy2DAsync((float *)o->raw_im.p + at, plane * sizeof(float), im + at,
                             plane * sizeof(float), bytes, n, cudaMemcpyHostToDevice, cs));
        if (elevation)
            CK(cudaMemcpyAsync((double *)o->raw_elev.p + at, elevation + at,
                               (size_t)nr * cols * sizeof(double), cudaMemcpyHostToDevice, cs));
        CK(tc_launch_prep_raw(o->n, (const float *)o->raw_re.p, (const float *)o->raw_im.p,
                              elevation ? (const double *)o->raw_elev.p : nullptr, row0,
                              region_rows, padded_rows, cols, o->wr / 2, r0, r0 + nr,
                              o->has_geo ? &o->geo : nullptr, (const double *)o->geo_grid.p,
                              nullptr, nullptr, (float *)o->slc.p, (float *)o->amp.p,
                              (unsigned char *)o->valid.p, cs));
        CK(cudaEventRecord(o->block_done[b], cs));
    }
    return run_context_buffers(o, padded_rows, rows, cols, coh, count, pairs, phases, status, tm,
                               &ready);
}

TC_API int tc_run_raw_device(struct ocl *o, const float *re, const float *im,
                             const double *elevation, int row0, int region_rows, int padded_rows,
                             int rows, int cols, float *coh, int *count, float *pairs,
                             float *phases, unsigned char *status, void *stream)
{
    int rc;

    if ((rc = check_raw(o, re, im, region_rows, padded_rows, rows, cols, coh, count)) != TC_OK)
        return rc;
    CK(cudaSetDevice(o->device));
    cudaStream_t st = (cudaStream_t)stream;
    Timer tm(o, st);

    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));
    if ((rc = prepare_raw(o, re, im, elevation, row0, region_rows, padded_rows, cols, st, tm)) !=
        TC_OK)
        return rc;
    rc = run_device(o, (const float *)o->slc.p, (const float *)o->amp.p,
                    (const unsigned char *)o->valid.p, padded_rows, rows, cols, coh, count,
                    pairs, phases, status, st, tm);
    if (o->timing) {
        cudaStreamSynchronize(st);
        tm.collect();
    }
    return rc;
}

TC_API int tc_adjoint_raw(struct ocl *o, const float *re, const float *im,
                          const double *elevation, const double *dh, const float *psi, int row0,
                          int region_rows, int padded_rows, int rows, int cols, float *coh,
                          int *count, float *grad_dh, float *grad_psi)
{
    int rc;

    if ((rc = check_raw(o, re, im, region_rows, padded_rows, rows, cols, coh, count)) != TC_OK)
        return rc;
    if (o->n > 32)
        return set_error(TC_ERR_ARG, "the adjoint takes stacks of up to 32 dates, not %d", o->n);
    if (!grad_psi)
        return set_error(TC_ERR_ARG, "no gradient buffer");
    CK(cudaSetDevice(o->device));
    const size_t plane = (size_t)padded_rows * cols;
    const size_t n = o->n;
    cudaStream_t st = o->stream;
    Timer tm(o, st);

    memset(o->stage_ms, 0, sizeof(o->stage_ms));
    memset(o->stage_launches, 0, sizeof(o->stage_launches));
    CK(ensure(o->raw_re, n * plane * sizeof(float)));
    CK(ensure(o->raw_im, n * plane * sizeof(float)));
    if (elevation)
        CK(ensure(o->raw_elev, plane * sizeof(double)));
    if (dh)
        CK(ensure(o->adj_dh, plane * sizeof(double)));
    if (psi)
        CK(ensure(o->adj_psi, n * plane * sizeof(float)));
    CK(ensure(o->adj_dtheta, n * plane * sizeof(float)));
    CK(ensure(o->adj_gdh, plane * sizeof(float)));
    if ((rc = ensure_outputs(o, (size_t)rows * cols, false, false)) != TC_OK)
        return rc;
    int t = tm.begin(ST_COPY);

    CK(cudaMemcpyAsync(o->raw_re.p, re, n * plane * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(o->raw_im.p, im, n * plane * sizeof(float), cudaMemcpyHostToDevice, st));
    if (elevation)
        CK(cudaMemcpyAsync(o->raw_elev.p, elevation, plane * sizeof(double),
                           cudaMemcpyHostToDevice, st));
    if (dh)
        CK(cudaMemcpyAsync(o->adj_dh.p, dh, plane * sizeof(double), cudaMemcpyHostToDevice, st));
    if (psi)
        CK(cudaMemcpyAsync(o->adj_psi.p, psi, n * plane * sizeof(float), cudaMemcpyHostToDevice,
                           st));
    CK(cudaMemsetAsync(o->adj_dtheta.p, 0, n * plane * sizeof(float), st));
    tm.end(t);
    const double *d_elev = elevation ? (const double *)o->raw_elev.p : nullptr;
    const double *d_dh = dh ? (const double *)o->adj_dh.p : nullptr;

    if ((rc = prepare_raw(o, (const float *)o->raw_re.p, (const float *)o->raw_im.p, d_elev, row0,
                          region_rows, padded_rows, cols, st, tm, d_dh,
                          psi ? (const float *)o->adj_psi.p : nullptr)) != TC_OK)
        return rc;
    /* the Gram gradient has the Gram's size */
    const int crows = chunk_rows_for(o, rows, cols);
    const size_t max_npix = (size_t)(crows / TC_TILE_H) * ((cols + TC_TILE_W - 1) / TC_TILE_W) *
                            TC_TILE_PIX;

    CK(ensure(o->adj_gbar, sizeof(float2) * tc_npu(o->n) * max_npix));
    AdjRun adj = {(float2 *)o->adj_gbar.p, (float *)o->adj_dtheta.p};

    rc = run_device(o, (const float *)o->slc.p, (const float *)o->amp.p,
                    (const unsigned char *)o->valid.p, padded_rows, rows, cols, (float *)o->coh.p,
                    (int *)o->count.p, o->npairs ? (float *)o->pairs.p : nullptr, nullptr, nullptr,
                    st, tm, &adj);
    if (rc != TC_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    CK(tc_launch_adjoint_height(o->n, padded_rows, cols, row0, region_rows, d_elev, d_dh,
                                o->has_geo ? &o->geo : nullptr, (const double *)o->geo_grid.p,
                                (const float *)o->adj_dtheta.p, (float *)o->adj_gdh.p, st));
    t = tm.begin(ST_COPY);
    CK(cudaMemcpyAsync(coh, o->coh.p, (size_t)rows * cols * sizeof(float), cudaMemcpyDeviceToHost,
                       st));
    CK(cudaMemcpyAsync(count, o->count.p, (size_t)rows * cols * sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(grad_psi, o->adj_dtheta.p, n * plane * sizeof(float),
                       cudaMemcpyDeviceToHost, st));
    if (grad_dh)
        CK(cudaMemcpyAsync(grad_dh, o->adj_gdh.p, plane * sizeof(float), cudaMemcpyDeviceToHost,
                           st));
    tm.end(t);
    CK(cudaStreamSynchronize(st));
    tm.collect();
    if (o->opt.gram == TC_GRAM_TENSOR && tc_gram_tensor_fault() > 0)
        return set_error(TC_ERR_DEVICE, "tensor-core Gram: a wait for MMA completion ran out; "
                         "the tiles concerned are NULL");
    return TC_OK;
}

/* ------------------------------------------------------------------ */
/* ocl_* drop-in.                                                      */
/* ------------------------------------------------------------------ */

TC_API struct ocl *ocl_open(int platform, int device, const struct settings *s,
                            int padded_cols, size_t *max_alloc)
{
    struct ocl *o = nullptr;
    tc_options opt;
    const char *env;

    if (platform < 0 && device >= 0) {
        set_error(TC_ERR_ARG, "Option device requires option platform");
        fatal("CUDA backend");
    }
    if (platform > 0) {
        set_error(TC_ERR_DEVICE, "platform %d not found (1 platform, see -l)", platform);
        fatal("CUDA backend");
    }
    opt.gram = (s && tc_gram_tensor_supported(s->ndates, s->win_az, s->win_rg)) ? TC_GRAM_TENSOR
                                                                     : TC_GRAM_FP32;
    opt.split_terms = 3;
    opt.chunk_pixels = 0;
    if ((env = getenv("TCOH_GRAM")) && !strcmp(env, "fp32"))
        opt.gram = TC_GRAM_FP32;
    if ((env = getenv("TCOH_SPLIT_TERMS")))
        opt.split_terms = atoi(env);
    if ((env = getenv("TCOH_CHUNK_PIXELS")))
        opt.chunk_pixels = atoi(env);
    if (tc_open(device, s, padded_cols, &opt, &o, max_alloc) != TC_OK)
        fatal("CUDA backend");
    return o;
}

TC_API void ocl_run(struct ocl *o, const float *slc, const float *amp,
                    const unsigned char *valid, int padded_rows, int rows, int cols,
                    float *coh, int *count, float *pairs)
{
    if (tc_run_ex(o, slc, amp, valid, padded_rows, rows, cols, coh, count, pairs, nullptr,
                  nullptr) != TC_OK)
        fatal("CUDA backend");
}

TC_API void ocl_close(struct ocl *o)
{
    tc_close(o);
}
