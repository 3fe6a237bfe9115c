/* Internal definitions shared by the kernels and the C-ABI layer. */
#ifndef TCOH_INTERNAL_H
#define TCOH_INTERNAL_H

#include <cuda_runtime.h>

#include "../../include/tcoh_b200.h"
#include <stdint.h>

#define TC_MAX_DATES 64
#define TC_MAX_MASK_WORDS 32 /* SHP windows of up to 1024 candidates */

/* Output pixels are processed in tiles of 16 rows x 8 columns (128 pixels,
   the M extent of one tensor-core accumulator tile). Within a chunk, pixel
   p belongs to tile p / 128, row (p % 128) / 8, column p % 8 of the tile;
   tiles run row-major over the chunk. */
#define TC_TILE_H 16
#define TC_TILE_W 8
#define TC_TILE_PIX (TC_TILE_H * TC_TILE_W)

/* Per-strip constants. */
struct TcStrip {
    int n;           /* dates */
    int wa, wr;      /* window lines, samples */
    int area;        /* wa * wr candidates */
    int mask_words;  /* ceil(area / 32) */
    int W;           /* padded columns */
    int padded_rows;
    int rows, cols;  /* output size */
    long long npad;  /* padded pixels */
    int planes;      /* SoA date planes (n rounded up to the Gram block) */
};

/* One chunk: output rows row0 .. row0 + nrows - 1, all columns. */
struct TcChunk {
    int row0, nrows;
    int tiles_x, tiles_y;
    int npix; /* tiles_x * tiles_y * 128 */
};

/* Decision constants of the SHP tests, as the float values the reference
   kernel is built with (ocl.c:222-229). */
struct TcShpConst {
    int test, ks_max;
    float ad_norm, ad_sigma, ad_crit, tlog_crit;
};

struct TcLinkConst {
    int emi, bias, min_looks;
    int npairs, pairs_all;
};

__host__ __device__ inline int tc_npu(int n) { return n * (n + 1) / 2; }

/* The bias correction zeroes an entry when L m2 <= 1 (tcoh.cl:626-632), a
   jump of gamma by up to 2 / (n (n - 1)). Where the float rounding of the
   sums could decide it otherwise than double sums, |L m2 - 1| within this
   fraction of L m2 (the float error there is about 2e-6 of it), the float
   kernels send the pixel to the exact tier, which decides in double. */
#define TC_BIAS_BAND 3.0e-5f

/* The coherence sums of a chunk are float2 [npix][npu], pixel-major: the
   lanes that load one pixel's matrix read contiguous bytes. */
__host__ __device__ inline long long tc_gram_at(int npu, long long p, int q)
{
    return p * npu + q;
}

/* Packed upper-triangle index of (i, j), i <= j. */
__host__ __device__ inline int tc_pidx(int n, int i, int j)
{
    return i * (2 * n - i + 1) / 2 + (j - i);
}

__host__ __device__ inline void tc_pixel_yx(const TcChunk &c, int p, int &y, int &x)
{
    const int t = p >> 7, w = p & 127;
    const int ty = t / c.tiles_x, tx = t - ty * c.tiles_x;

    y = c.row0 + ty * TC_TILE_H + (w >> 3);
    x = tx * TC_TILE_W + (w & 7);
}

/* The pixels handed to the exact tier, queued across the chunks of a strip
   so that one launch of the exact kernel takes many chunks' pixels: buf[0]
   counts the entries, buf[1] the entries that the exact kernel's CTAs have
   taken beyond their first (each CTA takes its next pixel from it, so that
   pixels of unequal cost spread evenly); entry e (buf + TC_QUEUE_HEAD + e *
   stride, stride = 1 + mask_words) holds the pixel's output index y * cols + x and its SHP-mask
   words, copied from the chunk's mask (which the next chunk overwrites).
   The float link kernels append to it; the host flushes it
   (tc_flush_exact) before a chunk could overflow it and at the end of the
   strip, and counts in `pending` an upper bound on the entries queued. */
constexpr int TC_QUEUE_HEAD = 2; /* ints before the first entry, zeroed per flush */

struct TcExactQueue {
    int *buf;
    int stride;
    long long capacity; /* entries */
    long long pending;
};

#ifdef __CUDACC__
/* Appends pixel p of a chunk (output index out) with its mask words. */
__device__ __forceinline__ void tc_exact_push(int *q, int stride, long long out,
                                              const uint32_t *mask, long long npix, int p)
{
    int *e = q + TC_QUEUE_HEAD + (long long)atomicAdd(q, 1) * stride;

    e[0] = (int)out;
    for (int w = 1; w < stride; w++)
        e[w] = (int)mask[(long long)(w - 1) * npix + p];
}
#endif

/* Geometry (geometry.cu): the device copy of struct tc_geometry with the
   grid shape, and the orbits of all dates concatenated. */
struct TcGeo {
    int ndates, ref, grid_rows, grid_cols, nheights;
    double heights[3];
    double first_line_time, azimuth_time_interval, slant_range_time, range_sampling_rate;
    double wavelength, line0, sample0, h0;
};

struct TcOrbitSet {
    const int *count, *offset;
    const double *t, *pos, *vel;
};

/* The phase grid on the device, in coefficient form: for every node and
   date, phase(h) = c0 + u (c1 + u c2) with u = h - (the middle height level)
   is the quadratic through the node's phases at the three height levels
   (c1 = c2 = 0 with one level), double [grid_rows][grid_cols][ndates][3].
   Interpolation between nodes is bilinear in line and sample, every 16 of
   each; with linear interpolation commuting with the polynomial, this is
   the reference's bilinear-then-quadratic interpolation (geometry.c:256-291)
   evaluated in another order. */
#define TC_GEO_STEP 16

struct TcGridCell {
    const double *q00, *q01, *q10, *q11;
    double w00, w01, w10, w11, u;
    bool quad;

    /* phase of date k, and its height derivative when dh is not null */
    __device__ __forceinline__ double phase(int k, double *dh) const
    {
        const double *a = q00 + 3 * k, *b = q01 + 3 * k, *c = q10 + 3 * k, *d = q11 + 3 * k;
        const double c0 = w00 * a[0] + w01 * b[0] + w10 * c[0] + w11 * d[0];

        if (!quad) {
            if (dh)
                *dh = 0.0;
            return c0;
        }
        const double c1 = w00 * a[1] + w01 * b[1] + w10 * c[1] + w11 * d[1];
        const double c2 = w00 * a[2] + w01 * b[2] + w10 * c[2] + w11 * d[2];

        if (dh)
            *dh = c1 + 2.0 * u * c2;
        return c0 + u * (c1 + u * c2);
    }
};

/* Region cell (row, col) at height h (the grid covers it: row, col >= 0). */
__host__ __device__ inline TcGridCell tc_grid_cell(const TcGeo &g, const double *coef, int row,
                                                   int col, double h)
{
    TcGridCell c;
    const int gr = row / TC_GEO_STEP, gc = col / TC_GEO_STEP, n = g.ndates;
    const double fr = (double)(row - gr * TC_GEO_STEP) / TC_GEO_STEP;
    const double fc = (double)(col - gc * TC_GEO_STEP) / TC_GEO_STEP;
    const size_t node = (size_t)3 * n;

    c.q00 = coef + ((size_t)gr * g.grid_cols + gc) * node;
    c.q01 = c.q00 + node;
    c.q10 = c.q00 + (size_t)g.grid_cols * node;
    c.q11 = c.q10 + node;
    c.w00 = (1.0 - fr) * (1.0 - fc);
    c.w01 = (1.0 - fr) * fc;
    c.w10 = fr * (1.0 - fc);
    c.w11 = fr * fc;
    c.quad = g.nheights == 3;
    c.u = c.quad ? h - g.heights[1] : 0.0;
    return c;
}

int tc_geometry_shape(const struct tc_geometry &in, TcGeo &g);
int tc_geometry_grid(const TcGeo &g, const struct tc_orbit *orbits, double *grid_host,
                     cudaStream_t st);
/* The coefficient form of a phase grid (device, as tc_geometry_grid writes
   it: double [grid_rows][grid_cols][nheights][ndates]) into coef. */
cudaError_t tc_launch_geometry_coef(const TcGeo &g, const double *grid, double *coef,
                                    cudaStream_t st);
/* Strip preparation from raw planes for padded rows prow0 .. prow1 - 1. */
cudaError_t tc_launch_prep_raw(int n, const float *re, const float *im, const double *elev,
                               int row0, int region_rows, int padded_rows, int cols, int halo,
                               int prow0, int prow1, const TcGeo *g, const double *grid,
                               const double *dh, const float *psi, float *slc, float *amp,
                               unsigned char *valid, cudaStream_t st);
/* Adjoint (adjoint.cu): dL/dtheta += the chunk's contribution (dtheta
   [n][padded_rows][cols], zeroed by the caller); dL/ddh from dL/dtheta. */
cudaError_t tc_launch_adjoint_scatter(const TcStrip &s, const TcChunk &c, int halo,
                                      const float2 *gbar, const uint32_t *mask,
                                      const float *slc, float *dtheta, cudaStream_t st);
cudaError_t tc_launch_adjoint_height(int n, int padded_rows, int cols, int row0, int region_rows,
                                     const double *elev, const double *dh, const TcGeo *g,
                                     const double *grid, const float *dtheta, float *gdh,
                                     cudaStream_t st);

/* Helpers of abi.cu shared with the other translation units. */
int tc_error(int code, const char *fmt, ...);
int tc_check_settings(const struct settings *s, int padded_cols);
float tc_float_literal(double v);

/* Kernel launchers (kernels_*.cu); all asynchronous on `st`. */
cudaError_t tc_launch_prep(const TcStrip &s, const float *slc_aos, float2 *soa,
                           cudaStream_t st);
cudaError_t tc_launch_logstats(const TcStrip &s, const float *amp,
                               const unsigned char *valid, float2 *logstat,
                               cudaStream_t st);
cudaError_t tc_launch_shp(const TcStrip &s, const TcChunk &c, const TcShpConst &k,
                          const float *amp, const unsigned char *valid,
                          const float2 *logstat, uint32_t *mask, int *count,
                          int sms, cudaStream_t st);

/* A block of consecutive chunks whose SHP masks are selected together
   (tc_launch_shp_block): output rows row0 .. row0 + nrows - 1, chunks of
   crows rows (a multiple of TC_TILE_H) whose masks lie chunk_words u32
   apart, chunk j's in the layout of a chunk (word w of its pixel p at
   w * npix_j + p). */
struct TcShpBlock {
    int row0, nrows, crows, tiles_x;
    long long chunk_words;
};

/* SHP masks and counts of a block of chunks with every unordered pair of
   output pixels of the block tested once (the tests are symmetric when
   the two series share no value; pairs with a tie are tested both ways).
   The block's mask region must be zero on entry (the kernels OR bits in). */
cudaError_t tc_launch_shp_block(const TcStrip &s, const TcShpBlock &b, const TcShpConst &k,
                                const float *amp, const unsigned char *valid,
                                const float2 *logstat, uint32_t *mask, int *count, int sms,
                                cudaStream_t st);
cudaError_t tc_launch_gram_fp32(const TcStrip &s, const TcChunk &c, int block,
                                const float2 *soa, const uint32_t *mask,
                                float2 *gram, cudaStream_t st);
cudaError_t tc_launch_gram_tensor(const TcStrip &s, const TcChunk &c, int split_terms,
                                  const float *slc_aos, const uint32_t *mask,
                                  float2 *gram, cudaStream_t st);
/* Tensor-core Gram for n dates and a wa x wr window on the current device. */
bool tc_gram_tensor_supported(int n, int wa, int wr);
/* Non-zero if a tensor-core Gram wait ran out since the last call (and
   clears it): bit 1 a working wait, bit 2 also the teardown's drain of the
   issued MMAs; 0 if none, -1 if the flag cannot be read. Synchronous. */
int tc_gram_tensor_fault(void);
/* The adjoint's scatter as the transposed tensor-core Gram (n <= 32, at most
   512 candidates in a tile's union window); faults set the flag above. */
bool tc_gram_adjoint_tensor_supported(int n, int wa, int wr);
cudaError_t tc_launch_adjoint_scatter_tensor(const TcStrip &s, const TcChunk &c, int halo,
                                             const float2 *gbar, const uint32_t *mask,
                                             const float *slc, float *dtheta, cudaStream_t st);
int tc_gram_block_for(int n);
/* The link stage: phase linking and gamma of every pixel of a chunk from its
   coherence sums (gram), or, for EMI, from the samples (slc, AoS) and SHP
   masks in double precision where float sums are not accurate enough:
   every pixel above 32 dates (the Gram stage is then skipped, see
   tc_link_needs_gram), the flagged ones otherwise: those of EMI and of the
   bias correction go to the queue q (tc_link_queues), which must have
   room for the chunk's npix entries; the caller flushes it. */
cudaError_t tc_launch_link(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                           const float2 *gram, const float *slc, const uint32_t *mask,
                           const int *count, TcExactQueue *q,
                           const unsigned short *upper_tab, const unsigned short *pair_tab,
                           double *scratch, float *coh, float *pairs, float *phases,
                           unsigned char *status, int sms, cudaStream_t st);
/* Whether tc_launch_link queues pixels for the exact tier. */
bool tc_link_queues(int n, const TcLinkConst &k);
/* Device bytes of a queue of `capacity` entries. */
size_t tc_exact_queue_bytes(int mask_words, long long capacity);
/* Runs the exact tier on the queued pixels (strip-level outputs) and
   empties the queue; nothing to do when it is empty. */
cudaError_t tc_flush_exact(const TcStrip &s, const TcLinkConst &k, TcExactQueue *q,
                           const float *slc, const int *count, const unsigned short *upper_tab,
                           const unsigned short *pair_tab, double *scratch, float *coh,
                           float *pairs, float *phases, unsigned char *status, int sms,
                           cudaStream_t st);
bool tc_link_needs_gram(int n, int emi);
size_t tc_link_scratch_bytes(int n, int sms);
/* queue, when not null: its buffer (TcExactQueue::buf) and stride. */
cudaError_t tc_launch_link_half(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                const float2 *gram, const uint32_t *mask, const int *count,
                                const unsigned short *upper_tab, const unsigned short *pair_tab,
                                double *scratch, float *coh, float *pairs, float *phases,
                                unsigned char *status, int *queue, int qstride, int sms,
                                cudaStream_t st);
size_t tc_link_half_scratch_bytes(int n, int sms);
/* The link stage with the adjoint (n <= 32): gamma into coh, and into gbar
   (layout of gram) the gradient of gamma with respect to each pixel's
   coherence sums, zero for the pixels not estimated. */
cudaError_t tc_launch_link_adjoint(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                   const float2 *gram, const int *count,
                                   const unsigned short *upper_tab,
                                   const unsigned short *pair_tab, double *scratch, float *coh,
                                   float *pairs, float2 *gbar, int sms, cudaStream_t st);

#endif
