/* B200 (sm_100a) backend of the GRASS module i.sar.temporal_coherence.
 *
 * A drop-in replacement for the module's OpenCL backend ocl.c: the four
 * ocl_* entry points below have the exact prototypes of local_proto.h:104-112
 * and the behaviour of ocl.c (synchronous ocl_run over one padded strip,
 * fatal errors through G_fatal_error), so that main.c links against
 * libtcoh_b200.so instead of ocl.c unchanged. The tc_* entry points extend
 * it: return codes instead of fatal errors, device-resident strips, per-date
 * phase output, the choice of Gram arithmetic, stage timings and the
 * flat-earth / topographic geometry on the GPU.
 *
 * Strip layouts (row-major over the padded strip, main.c:28-34, 52-127):
 *   slc   float [padded_rows][padded_cols][N][2]  re, im, phase removed
 *   amp   float [padded_rows][padded_cols][N]     amplitudes, ascending
 *   valid uchar [padded_rows][padded_cols]        every date non-null, != 0
 * with padded_rows = rows + WA - 1 and padded_cols = cols + WR - 1. Outputs:
 *   coh   float [rows][cols]          temporal coherence, NaN = NULL
 *   count int   [rows][cols]          SHP count, -1 = NULL
 *   pairs float [npairs][rows][cols]  |T_ij|, NaN = NULL
 *   phases float [rows][cols][N]      phase-linked phases (radians, relative
 *                                      to the reference date), NaN = NULL
 */
#ifndef TCOH_B200_H
#define TCOH_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef I_SAR_TEMPORAL_COHERENCE_LOCAL_PROTO_H
/* Same layout as local_proto.h:12 and 34-49, which main.c passes in. */
enum shp_test { SHP_KS = 0, SHP_AD = 1, SHP_TLOG = 2 };

struct settings {
    int ndates;
    int win_az, win_rg;
    enum shp_test test;
    double alpha;
    int emi;
    int bias;
    int min_looks;
    int ks_max;
    double ad_norm, ad_sigma, ad_crit;
    double tlog_crit;
    int npairs;    /* pair coherence maps to write, 0 for none */
    int pairs_all; /* all pairs i < j instead of consecutive ones */
    const char *phase_reference; /* none, ellipsoid or elevation */
    const char *orbit;           /* orbit source, NULL without phase */
};
#endif

/* ------------------------------------------------------------------ */
/* Drop-in for ocl.c (local_proto.h:104-112).                          */
/* ------------------------------------------------------------------ */

struct ocl;

/* Replaces ocl.c:105-136: prints platform|device|type|name|version|
   compute_units|global_memory_mb, one line per CUDA device. */
void ocl_list_devices(void);

/* Replaces ocl.c:191-254. platform -1 or 0 (the CUDA platform), device -1
   for the first GPU. *max_alloc receives the largest strip buffer the
   backend accepts, which main.c:731-742 uses to size the strips. */
struct ocl *ocl_open(int platform, int device, const struct settings *s,
                     int padded_cols, size_t *max_alloc);

/* Replaces ocl.c:279-375: copies one padded strip to the GPU, computes
   every output pixel and copies the outputs back before returning. pairs
   may be NULL when s->npairs is 0. */
void ocl_run(struct ocl *o, const float *slc, const float *amp,
             const unsigned char *valid, int padded_rows, int rows, int cols,
             float *coh, int *count, float *pairs);

/* Replaces ocl.c:377-391. */
void ocl_close(struct ocl *o);

/* ------------------------------------------------------------------ */
/* Extensions.                                                         */
/* ------------------------------------------------------------------ */

/* Return codes of the tc_* functions. */
#define TC_OK           0
#define TC_ERR_ARG      1 /* invalid argument or shape */
#define TC_ERR_CUDA     2 /* CUDA runtime error, see tc_last_error() */
#define TC_ERR_MEMORY   3 /* device allocation failed */
#define TC_ERR_DEVICE   4 /* no such device, or not an sm_100 GPU */

/* Arithmetic of the masked coherence-matrix accumulation. */
#define TC_GRAM_TENSOR 0 /* tcgen05 tensor cores, split BF16 terms, FP32 sums */
#define TC_GRAM_FP32   1 /* plain FP32 FMA on the CUDA cores */

struct tc_options {
    int gram;         /* TC_GRAM_TENSOR or TC_GRAM_FP32; -1 for the default
                         (the tensor cores where available) */
    int split_terms;  /* BF16 terms per FP32 product for TC_GRAM_TENSOR:
                         2 (16 significant bits) or 3 (24, FP32-exact) */
    int chunk_pixels; /* output pixels per internal launch, 0 = automatic */
};

/* Status bits per pixel (tc_run_ex). */
#define TC_STATUS_EMI_PINV   1 /* EMI: |T| (numerically) singular or nearly,
                                  inverted by its eigen-pseudo-inverse */
#define TC_STATUS_UNLINKED   2 /* bias correction unlinked the dates */
#define TC_STATUS_ITER_CAP   4 /* an iterative solver reached its cap */
#define TC_STATUS_FP64       8 /* recomputed from double-precision
                                  coherence sums: EMI, every pixel above 32
                                  dates, and up to 32 dates the pixels whose
                                  float result the conditioning of |T| and
                                  of M's eigengap may have moved by more
                                  than ~1e-5; with the bias correction, the
                                  pixels with an entry at the threshold of
                                  the correction */
#define TC_STATUS_EMI_PIVOTED 16 /* EMI: |T| inverted by elimination with
                                    pivoting (the symmetric sweep met a
                                    pivot below 1e-5) */

/* Message of the last failed tc_* call of this thread. */
const char *tc_last_error(void);

/* Handler the ocl_* entry points call on a fatal error (ocl.c:44-48). By
   default G_fatal_error when the host program provides it, else the
   message is printed to stderr and the process exits with failure. The
   handler must not return. */
void tc_set_fatal_handler(void (*handler)(const char *message));

/* The SHP test constants of stats.c:61-95 (ks_max, ad_norm, ad_sigma,
   ad_crit, tlog_crit) for s->ndates, s->test and s->alpha, for hosts that
   do not link stats.c. TC_ERR_ARG when alpha is outside the AD table. */
int tc_shp_constants(struct settings *s);

/* Number of CUDA devices. */
int tc_device_count(void);

/* Open a context on CUDA device `device` (-1: the first one) for strips of
   padded_cols columns. opt may be NULL for the defaults. */
int tc_open(int device, const struct settings *s, int padded_cols,
            const struct tc_options *opt, struct ocl **out,
            size_t *max_alloc);

/* ocl_run with a return code and optional extra outputs: phases
   float [rows][cols][N] and status unsigned char [rows][cols] (either may
   be NULL). Host buffers. Returns TC_ERR_DEVICE if a bounded wait of the
   tensor-core Gram ran out during this or an earlier tc_run_device call;
   the tiles concerned come out NULL. */
int tc_run_ex(struct ocl *o, const float *slc, const float *amp,
              const unsigned char *valid, int padded_rows, int rows, int cols,
              float *coh, int *count, float *pairs, float *phases,
              unsigned char *status);

/* The same on device buffers, asynchronously on `stream` (a cudaStream_t;
   NULL is CUDA's default stream). Every pointer is a device address. */
int tc_run_device(struct ocl *o, const float *slc, const float *amp,
                  const unsigned char *valid, int padded_rows, int rows,
                  int cols, float *coh, int *count, float *pairs,
                  float *phases, unsigned char *status, void *stream);

/* The options a context runs with, defaults resolved (the Gram
   arithmetic chosen for gram = -1, the split terms in force). */
int tc_get_options(const struct ocl *o, struct tc_options *opt);

/* Flat-earth and topographic phase removal and strip preparation on the
   device (geometry.c, orbit.c, main.c:52-127). */

/* Orbit of one date (orbit.c:52-57): n >= 8 state vectors, times in
   seconds (increasing), Earth-fixed positions and velocities [n][3] in m
   and m/s. */
struct tc_orbit {
    int n;
    const double *t;
    const double *pos;
    const double *vel;
};

/* Acquisition geometry (geometry.c:161-216): the raster timing of the
   reference date's image and the region in it. */
struct tc_geometry {
    int ndates, ref;              /* dates; the reference date */
    double first_line_time;       /* s, time of image line 0 */
    double azimuth_time_interval; /* s per line */
    double slant_range_time;      /* s, two-way time of image sample 0 */
    double range_sampling_rate;   /* Hz */
    double wavelength;            /* m */
    double line0, sample0;        /* image line and sample of region cell (0, 0) */
    int rows, cols;               /* region size */
    double hmin, hmax;            /* height range of the elevation map; h0, h0 without */
    double h0;                    /* height used without an elevation map */
};

/* Shape of the phase grid: nodes every 16 lines and samples, one height
   level when hmax - hmin < 1 m, else three (hmin, mid, hmax), written to
   heights[3]. The grid is double [grid_rows][grid_cols][nheights][ndates]. */
int tc_geometry_grid_shape(const struct tc_geometry *g, int *grid_rows, int *grid_cols,
                           int *nheights, double *heights);

/* The phase grid, computed in double precision on the current device
   (geometry_init, geometry.c:161-254): for every node and height level the
   ground point of the reference date is located on the WGS84 ellipsoid and
   every date's phase 4 pi / lambda (R_k - R_ref) at its zero-Doppler time is
   written to grid (host). orbits[ndates]. TC_ERR_ARG when a point cannot be
   located or falls outside an orbit, as the reference's fatal errors. */
int tc_geometry_init(const struct tc_geometry *g, const struct tc_orbit *orbits,
                     double *grid);

/* Attaches a phase grid (host, as tc_geometry_init writes it) to the
   context for tc_run_raw; grid NULL detaches it. */
int tc_set_geometry(struct ocl *o, const struct tc_geometry *g, const double *grid);

/* tc_run_ex from raw rows: re, im float [ndates][padded_rows][cols] (host)
   are the I/Q samples of region rows row0 .. row0 + padded_rows - 1 (rows
   outside 0 .. region_rows - 1 are ignored; NaN marks NULL), elevation
   double [padded_rows][cols] or NULL. The strip preparation of
   main.c:52-127 runs on the device: validity, sorted amplitudes, and, with
   a geometry attached, the rotation of date k by exp(i phase_k) interpolated
   at each cell's height (the elevation, else h0). */
int tc_run_raw(struct ocl *o, const float *re, const float *im, const double *elevation,
               int row0, int region_rows, int padded_rows, int rows, int cols, float *coh,
               int *count, float *pairs, float *phases, unsigned char *status);

/* The same on device buffers, asynchronously on `stream`. */
int tc_run_raw_device(struct ocl *o, const float *re, const float *im,
                      const double *elevation, int row0, int region_rows, int padded_rows,
                      int rows, int cols, float *coh, int *count, float *pairs,
                      float *phases, unsigned char *status, void *stream);

/* Adjoint of the temporal coherence (no counterpart in the reference,
   whose module only evaluates it). The objective is L = the sum of gamma
   over the strip's estimated pixels, as a function of the phase removed
   from every sample, theta_k = phi_k(h + dh) + psi_k: the attached
   geometry's phase (tc_set_geometry; none: phi = 0) at the cell's height
   (elevation, else h0) plus a height error dh, and a per-date phase screen
   psi. Arguments as tc_run_raw, plus dh double [padded_rows][cols] and psi
   float [ndates][padded_rows][cols] (either NULL for zero). Outputs: coh
   and count of the forward, grad_psi float [ndates][padded_rows][cols] =
   dL/dpsi = dL/dtheta, and grad_dh float [padded_rows][cols] = dL/ddh (NULL
   to skip; zero without three height levels). Stacks of up to 32 dates;
   the SHP selection depends on the amplitudes only and is held fixed. */
int tc_adjoint_raw(struct ocl *o, const float *re, const float *im, const double *elevation,
                   const double *dh, const float *psi, int row0, int region_rows,
                   int padded_rows, int rows, int cols, float *coh, int *count,
                   float *grad_dh, float *grad_psi);

/* Stage timing. With timing on, every launch of the following runs is
   bracketed by CUDA events on its stream, and tc_stage_stats gives, per
   stage, the device milliseconds summed over the last run and the number
   of kernel launches: [0] strip preparation, [1] SHP selection,
   [2] coherence matrices, [3] phase linking and coherence (with the
   adjoint: and its backward pass), [4] host<->device copies (ms only),
   [5] the adjoint's scatter onto the samples, [6] the exact tier's
   launches over the pixels the float kernels queued for it (up to 16
   chunks' pixels per launch; the exact tier of every pixel, EMI above 32
   dates, counts in [3]). Returns the number of stages written (at most
   n). */
int tc_set_timing(struct ocl *o, int on);
int tc_stage_stats(const struct ocl *o, float *ms, int *launches, int n);

/* Close the context and free its device memory. */
int tc_close(struct ocl *o);

/* Measured FP32 FMA throughput of device `device` in TFLOP/s (two flops per
   FMA), the roofline denominator of the kernels on the CUDA cores. */
int tc_fp32_peak(int device, double *tflops);

/* The same in double precision: the denominator of the kernels that
   compute in FP64 (the EMI exact tier, the geometry grid, the raw strip
   preparation). */
int tc_fp64_peak(int device, double *tflops);

/* tc_run_device for callers that must not allocate device memory: no
   context, no cudaMalloc, on the current device and `stream` (NULL: CUDA's
   default stream); every pointer is a device address the caller owns. The
   path's intermediate buffers live in one static device array of 64 MiB,
   which every GPU that loads the library holds until exit; a strip whose
   16-row sub-strip needs more (very wide strips with many dates) gets
   TC_ERR_ARG and a message with the limit. All calls share that array:
   calls that overlap on the GPU race. Every call looks up the array's
   address (cudaGetSymbolAddress), so it stays right after a device reset;
   the first call on a device also loads the library's device code there
   and should come before any stream capture. The coherence matrices use
   plain FP32 (TC_GRAM_FP32).
   No counterpart in the reference, whose ocl_open always allocates. */
int tc_run_device_static(const struct settings *s, int padded_cols,
                         const float *slc, const float *amp,
                         const unsigned char *valid, int padded_rows,
                         int rows, int cols, float *coh, int *count,
                         float *pairs, float *phases, unsigned char *status,
                         void *stream);

#ifdef __cplusplus
}
#endif

#endif
