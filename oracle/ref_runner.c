/* Host loop around the reference kernel compiled as C (see ref_shim.h).
 *
 * TEST INFRASTRUCTURE ONLY: the reference's own per-pixel code, run over a
 * padded strip with one OpenMP thread per row block, in place of ocl.c's
 * NDRange launch (ocl.c:329-363). The kernel constants are given here as
 * the float values that ocl.c:222-229 writes into the OpenCL build options;
 * a specialised build (TCOH_REF_SPECIALISED) has them compiled in and
 * rejects (-2) a strip or options that are not its configuration.
 */
#include <stddef.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    float x, y;
} float2;

int ref_N, ref_WA, ref_WR, ref_W, ref_SHP_TEST, ref_EMI, ref_BIAS,
    ref_MIN_LOOKS, ref_KS_MAX, ref_PAIRS_ALL;
float ref_AD_NORM, ref_AD_SIGMA, ref_AD_CRIT, ref_TLOG_CRIT;
__thread int ref_gid[2];

void temporal_coherence(const float2 *slc, const float *amp,
                        const unsigned char *valid, float *coh, int *count,
                        float *pair_coh, const int rows, const int cols);

int ref_run(int n, int wa, int wr, int test, int emi, int bias, int min_looks,
            int ks_max, float ad_norm, float ad_sigma, float ad_crit,
            float tlog_crit, int pairs_all, const float *slc,
            const float *amp, const unsigned char *valid, int padded_rows,
            int padded_cols, int rows, int cols, float *coh, int *count,
            float *pairs, int nthreads)
{
    if (padded_rows != rows + wa - 1 || padded_cols != cols + wr - 1)
        return -1;
#ifdef TCOH_REF_SPECIALISED
    /* built for one configuration: the strip and the options must be it */
    if (n != N || wa != WA || wr != WR || padded_cols != W || test != SHP_TEST ||
        emi != EMI || bias != BIAS || min_looks != MIN_LOOKS || ks_max != KS_MAX ||
        ad_norm != AD_NORM || ad_sigma != AD_SIGMA || ad_crit != AD_CRIT ||
        tlog_crit != TLOG_CRIT || pairs_all != PAIRS_ALL)
        return -2;
#endif
    ref_N = n;
    ref_WA = wa;
    ref_WR = wr;
    ref_W = padded_cols;
    ref_SHP_TEST = test;
    ref_EMI = emi;
    ref_BIAS = bias;
    ref_MIN_LOOKS = min_looks;
    ref_KS_MAX = ks_max;
    ref_AD_NORM = ad_norm;
    ref_AD_SIGMA = ad_sigma;
    ref_AD_CRIT = ad_crit;
    ref_TLOG_CRIT = tlog_crit;
    ref_PAIRS_ALL = pairs_all;
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int y = 0; y < rows; y++)
        for (int x = 0; x < cols; x++) {
            ref_gid[0] = x;
            ref_gid[1] = y;
            temporal_coherence((const float2 *)slc, amp, valid, coh, count,
                               pairs, rows, cols);
        }
    (void)nthreads;
    return 0;
}

int ref_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
