/* CPU oracle of the phase-linking temporal coherence path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA path is
 * compared with; nothing in the product links or calls it. It is called only
 * from tests/, from __graft_entry__.smoke() and from bench.py's CPU baseline.
 *
 * It restates, in plain double-precision C, the per-pixel algorithm of the
 * reference's FP64 oracle tests/reference.py (a loop transcription of SNAP's
 * phase linking), on the same padded strip buffers that the module hands to
 * its device backend (main.c:52-127 read_strip, ocl.c:279 ocl_run):
 *
 *   slc   float [padded_rows][padded_cols][N][2]  (re, im), phase-rotated
 *   amp   float [padded_rows][padded_cols][N]     amplitudes sorted ascending
 *   valid uchar [padded_rows][padded_cols]
 *
 * The output pixel (y, x) has its window at padded rows y..y+WA-1 and
 * columns x..x+WR-1 (tcoh.cl:547, 572-576); halo cells outside the region are
 * invalid, which cuts the windows at the region edges exactly as
 * reference.py:242-243 does.
 *
 * Two arithmetics are offered for the SHP decisions:
 *   shp_fp32 = 0  reference.py:27-80 in double precision (the FP64 oracle);
 *   shp_fp32 = 1  the reference kernel's single-precision statistics
 *                 (tcoh.cl:34-95, 555-565), evaluated in IEEE float with no
 *                 contraction, so that the decisions are those of the kernel.
 * Everything after the SHP selection is double precision and follows
 * reference.py:124-197: coherence matrix, bias correction, connectivity,
 * EVD / EMI (eigen-pseudo-inverse with absolute floor 1e-9) through a cyclic
 * complex Jacobi eigensolver run to convergence (reference.py calls LAPACK's
 * zheevd through np.linalg.eigh), phases relative to the median date and the
 * Pepe-Lanari goodness of fit.
 *
 * Parity of this restatement is pinned against golden vectors produced by
 * importing tests/reference.py itself (tests/golden/make_golden.py) and
 * against the reference kernel compiled as C (oracle/Makefile, oracle/_ref).
 */

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_DATES 64

typedef struct {
    int ndates;
    int win_az, win_rg;
    int test; /* 0 KS, 1 AD, 2 t-test on logs */
    double alpha;
    int emi;
    int bias;
    int min_looks; /* max(min_shp, N), main.c:585-587 */
    int npairs;    /* pair planes to write, 0 for none */
    int pairs_all; /* all pairs i < j, else consecutive (i, i + 1) */
    int shp_fp32;  /* SHP statistics in the kernel's float arithmetic */
} orc_settings;

/* ------------------------------------------------------------------ */
/* Test constants.                                                     */
/* ------------------------------------------------------------------ */

/* Standard deviation of the two-sample A2 under the null, samples of size n
   (reference.py:87-116; Scholz and Stephens 1987, eq. 4). */
static double orc_ad_sigma(int n)
{
    const int k = 2, total = 2 * n;
    const double big_h = 2.0 / n;
    double h = 0.0, g = 0.0, a, b, c, d, var;

    for (int j = 1; j < total; j++)
        h += 1.0 / j;
    for (int i = 1; i < total - 1; i++)
        for (int j = i + 1; j < total; j++)
            g += 1.0 / ((double)(total - i) * j);
    a = (4 * g - 6) * (k - 1) + (10 - 6 * g) * big_h;
    b = (2 * g - 4) * k * k + 8 * h * k + (2 * g - 14 * h - 4) * big_h -
        8 * h + 4 * g - 6;
    c = (6 * h + 2 * g - 2) * k * k + (4 * h - 4 * g + 6) * k +
        (2 * h - 6) * big_h + 4 * h;
    d = (2 * h + 6) * k * k - 4 * h * k;
    var = (a * pow(total, 3) + b * (double)total * total + c * total + d) /
          ((total - 1.0) * (total - 2.0) * (total - 3.0));
    return var > 0 ? sqrt(var) : 1.0;
}

static const double orc_ad_alpha[7] = {0.25, 0.10, 0.05, 0.025,
                                       0.01, 0.005, 0.001};
static const double orc_ad_table[7] = {0.325, 1.226, 1.961, 2.718,
                                       3.752, 4.592, 6.546};

/* T_1 critical value, linear in log(alpha) between the table levels and
   clamped outside, as np.interp in reference.py:119-121. */
double orc_ad_critical(double alpha)
{
    const double x = log(alpha);

    if (x <= log(orc_ad_alpha[6]))
        return orc_ad_table[6];
    if (x >= log(orc_ad_alpha[0]))
        return orc_ad_table[0];
    for (int i = 6; i > 0; i--) {
        const double x0 = log(orc_ad_alpha[i]), x1 = log(orc_ad_alpha[i - 1]);

        if (x <= x1)
            return orc_ad_table[i] + (x - x0) * (orc_ad_table[i - 1] -
                                                 orc_ad_table[i]) /
                                         (x1 - x0);
    }
    return orc_ad_table[0];
}

/* Two-sided standard normal quantile: P(|Z| > z) = alpha, by bisection on
   erfc (stats.c:45-59 computes it this way; reference.py:71 uses
   NormalDist().inv_cdf(1 - alpha / 2), equal to double rounding). */
double orc_normal_quantile(double alpha)
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

/* The float constants of the reference kernel: stats.c:61-95 in double,
   then written by ocl.c:222-229 with "%.9e" into float literals. */
typedef struct {
    int ks_max;
    float ad_norm, ad_sigma, ad_crit, tlog_crit;
} orc_kernel_constants;

static float orc_float_literal(double v)
{
    char buf[64];

    snprintf(buf, sizeof(buf), "%.9e", v);
    return strtof(buf, NULL);
}

void orc_kernel_constants_for(const orc_settings *s, orc_kernel_constants *k)
{
    const int n = s->ndates;
    double ad_crit = 0.0;

    k->ks_max =
        (int)floor(sqrt(-0.5 * log(s->alpha / 2.0)) * sqrt(2.0 / n) * n);
    k->ad_norm = orc_float_literal(1.0 / (2.0 * n) * (2.0 / n));
    k->ad_sigma = orc_float_literal(orc_ad_sigma(n));
    if (s->test == 1) {
        /* stats.c:194-205: linear in log(alpha), table levels decreasing. */
        int i;

        for (i = 0; i < 6; i++)
            if (s->alpha >= orc_ad_alpha[i + 1])
                break;
        if (i == 6)
            i = 5;
        {
            const double f = (log(s->alpha) - log(orc_ad_alpha[i])) /
                             (log(orc_ad_alpha[i + 1]) - log(orc_ad_alpha[i]));

            ad_crit = orc_ad_table[i] + f * (orc_ad_table[i + 1] -
                                             orc_ad_table[i]);
        }
    }
    k->ad_crit = orc_float_literal(ad_crit);
    k->tlog_crit = orc_float_literal(orc_normal_quantile(s->alpha));
}

/* ------------------------------------------------------------------ */
/* SHP tests.                                                          */
/* ------------------------------------------------------------------ */

/* reference.py:27-49: merge walk with the centre first on ties, CDF steps
   accumulated in double, compared with c(alpha) sqrt(2 / n). */
static int orc_ks64(const float *a, const float *b, int n, double critical)
{
    int ia = 0, ib = 0;
    double fa = 0.0, fb = 0.0, d = 0.0;

    while (ia < n && ib < n) {
        if (a[ia] <= b[ib]) {
            fa += 1.0 / n;
            ia++;
        }
        else {
            fb += 1.0 / n;
            ib++;
        }
        d = fmax(d, fabs(fa - fb));
    }
    while (ia < n) {
        fa += 1.0 / n;
        ia++;
        d = fmax(d, fabs(fa - fb));
    }
    while (ib < n) {
        fb += 1.0 / n;
        ib++;
        d = fmax(d, fabs(fa - fb));
    }
    return d <= critical;
}

/* reference.py:52-66: Scholz-Stephens eq. 6 rank statistic, standardized,
   in double. */
static double orc_ad64(const float *a, const float *b, int n, double sigma)
{
    const int total = 2 * n;
    const double norm = 1.0 / total * (2.0 / n);
    int ia = 0, ib = 0, m = 0;
    double s = 0.0;

    for (int j = 1; j < total; j++) {
        long num;

        if (ia < n && (ib >= n || a[ia] <= b[ib])) {
            m++;
            ia++;
        }
        else
            ib++;
        num = (long)total * m - (long)j * n;
        s += (double)(num * num) / (double)((long)j * (total - j));
    }
    return (norm * s - 1.0) / sigma;
}

/* reference.py:69-80: Welch t of the log amplitudes in double. */
static int orc_tlog64(const float *a, const float *b, int n, double critical)
{
    double mc = 0.0, mx = 0.0, vc = 0.0, vx = 0.0, se;

    for (int k = 0; k < n; k++) {
        mc += log((double)a[k]);
        mx += log((double)b[k]);
    }
    mc /= n;
    mx /= n;
    for (int k = 0; k < n; k++) {
        const double dc = log((double)a[k]) - mc, dx = log((double)b[k]) - mx;

        vc += dc * dc;
        vx += dx * dx;
    }
    vc /= n - 1;
    vx /= n - 1;
    se = sqrt(vc / n + vx / n);
    if (!(se > 0))
        return 1;
    return fabs(mc - mx) / se <= critical;
}

/* The kernel's integer KS (tcoh.cl:34-54). */
static int orc_ks32(const float *a, const float *b, int n, int ks_max)
{
    int ia = 0, ib = 0, d = 0;

    while (ia < n && ib < n) {
        int diff;

        if (a[ia] <= b[ib])
            ia++;
        else
            ib++;
        diff = abs(ia - ib);
        if (diff > d)
            d = diff;
    }
    return d <= ks_max;
}

/* The kernel's float AD (tcoh.cl:56-75); volatile keeps every operation
   rounded to float in source order. */
static int orc_ad32(const float *a, const float *b, int n,
                    const orc_kernel_constants *k)
{
    int ia = 0, ib = 0, m = 0;
    volatile float s = 0.0f;

    for (int j = 1; j < 2 * n; j++) {
        volatile float num, q;

        if (ia < n && (ib >= n || a[ia] <= b[ib])) {
            m++;
            ia++;
        }
        else
            ib++;
        num = (float)(2 * n * m - j * n);
        q = num * num;
        q = q / (float)(j * (2 * n - j));
        s = s + q;
    }
    {
        volatile float t = k->ad_norm * s;

        t = t - 1.0f;
        t = t / k->ad_sigma;
        return t <= k->ad_crit;
    }
}

/* The kernel's float log statistics of one sorted series (tcoh.cl:82-90,
   555-565). */
static void orc_logstats32(const float *a, int n, float *mean, float *var)
{
    volatile float m = 0.0f, v = 0.0f;

    for (int k = 0; k < n; k++)
        m = m + logf(a[k]);
    m = m / (float)n;
    for (int k = 0; k < n; k++) {
        volatile float d = logf(a[k]) - m;

        d = d * d;
        v = v + d;
    }
    v = v / (float)(n - 1);
    *mean = m;
    *var = v;
}

/* tcoh.cl:91-94 */
static int orc_tlog32(float mean_a, float var_a, float mean_b, float var_b,
                      int n, float crit)
{
    volatile float se = var_a + var_b, t;

    se = se / (float)n;
    se = sqrtf(se);
    if (!(se > 0.0f))
        return 1;
    t = fabsf(mean_a - mean_b);
    t = t / se;
    return t <= crit;
}

/* ------------------------------------------------------------------ */
/* Complex Hermitian eigensolver (double).                             */
/* ------------------------------------------------------------------ */

/* Cyclic Jacobi on the Hermitian n x n matrix (ar + i ai, full storage,
   row-major): on return the diagonal of ar holds the eigenvalues and the
   columns of (vr + i vi) the eigenvectors. Each step first gives a_pq a zero
   phase with a diagonal unitary on index q, then annihilates it with a real
   plane rotation. Sweeps run until the off-diagonal mass is below 1e-30 of
   the total, so the result is accurate to double rounding. */
static void orc_jacobi(int n, double *ar, double *ai, double *vr, double *vi)
{
    for (int p = 0; p < n * n; p++) {
        vr[p] = 0.0;
        vi[p] = 0.0;
    }
    for (int p = 0; p < n; p++)
        vr[p * n + p] = 1.0;

    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, total = 0.0;

        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++) {
                const double m2 = ar[p * n + q] * ar[p * n + q] +
                                  ai[p * n + q] * ai[p * n + q];

                total += m2;
                if (p != q)
                    off += m2;
            }
        if (off <= 1e-30 * total || off == 0.0)
            break;

        for (int p = 0; p < n - 1; p++) {
            for (int q = p + 1; q < n; q++) {
                const double xr = ar[p * n + q], xi = ai[p * n + q];
                const double r = hypot(xr, xi);
                double er, ei, tau, t, c, s;

                if (r == 0.0)
                    continue;
                /* D = diag(1, .., e^{-i theta} at q, ..): A <- D^H A D makes
                   a_pq = r real; V <- V D. */
                er = xr / r;
                ei = -xi / r; /* e^{-i theta} */
                for (int k = 0; k < n; k++) {
                    double re = ar[k * n + q], im = ai[k * n + q];

                    /* column q times e^{-i theta} */
                    ar[k * n + q] = re * er - im * ei;
                    ai[k * n + q] = re * ei + im * er;
                    re = vr[k * n + q];
                    im = vi[k * n + q];
                    vr[k * n + q] = re * er - im * ei;
                    vi[k * n + q] = re * ei + im * er;
                }
                for (int k = 0; k < n; k++) {
                    const double re = ar[q * n + k], im = ai[q * n + k];

                    /* row q times e^{+i theta} */
                    ar[q * n + k] = re * er + im * ei;
                    ai[q * n + k] = im * er - re * ei;
                }
                ar[p * n + q] = r;
                ai[p * n + q] = 0.0;
                ar[q * n + p] = r;
                ai[q * n + p] = 0.0;
                ai[q * n + q] = 0.0;

                /* Real rotation annihilating the real a_pq = r. */
                tau = (ar[q * n + q] - ar[p * n + p]) / (2.0 * r);
                t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                c = 1.0 / sqrt(1.0 + t * t);
                s = t * c;
                for (int k = 0; k < n; k++) {
                    if (k != p && k != q) {
                        const double kpr = ar[k * n + p], kpi = ai[k * n + p];
                        const double kqr = ar[k * n + q], kqi = ai[k * n + q];

                        ar[k * n + p] = c * kpr - s * kqr;
                        ai[k * n + p] = c * kpi - s * kqi;
                        ar[k * n + q] = s * kpr + c * kqr;
                        ai[k * n + q] = s * kpi + c * kqi;
                        ar[p * n + k] = ar[k * n + p];
                        ai[p * n + k] = -ai[k * n + p];
                        ar[q * n + k] = ar[k * n + q];
                        ai[q * n + k] = -ai[k * n + q];
                    }
                    {
                        const double kpr = vr[k * n + p], kpi = vi[k * n + p];
                        const double kqr = vr[k * n + q], kqi = vi[k * n + q];

                        vr[k * n + p] = c * kpr - s * kqr;
                        vi[k * n + p] = c * kpi - s * kqi;
                        vr[k * n + q] = s * kpr + c * kqr;
                        vi[k * n + q] = s * kpi + c * kqi;
                    }
                }
                ar[p * n + p] -= t * r;
                ar[q * n + q] += t * r;
                ar[p * n + q] = ar[q * n + p] = 0.0;
                ai[p * n + q] = ai[q * n + p] = 0.0;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Per-pixel pipeline.                                                 */
/* ------------------------------------------------------------------ */

typedef struct {
    double *cr, *ci;       /* covariance, then coherence T */
    double *ar, *ai;       /* eigensolver input */
    double *vr, *vi;       /* eigenvectors */
    double *g, *gi;        /* |T| and its pseudo-inverse */
} orc_work;

static void orc_work_alloc(orc_work *w, int n)
{
    const size_t nn = (size_t)n * n;

    w->cr = calloc(nn, sizeof(double));
    w->ci = calloc(nn, sizeof(double));
    w->ar = calloc(nn, sizeof(double));
    w->ai = calloc(nn, sizeof(double));
    w->vr = calloc(nn, sizeof(double));
    w->vi = calloc(nn, sizeof(double));
    w->g = calloc(nn, sizeof(double));
    w->gi = calloc(nn, sizeof(double));
}

static void orc_work_free(orc_work *w)
{
    free(w->cr);
    free(w->ci);
    free(w->ar);
    free(w->ai);
    free(w->vr);
    free(w->vi);
    free(w->g);
    free(w->gi);
}

/* reference.py:187-197 */
static int orc_connected(int n, const double *tr, const double *ti)
{
    int seen[ORC_MAX_DATES] = {0}, todo[ORC_MAX_DATES], top = 0, reached = 1;

    seen[0] = 1;
    todo[top++] = 0;
    while (top > 0) {
        const int i = todo[--top];

        for (int j = 0; j < n; j++)
            if (!seen[j] && (tr[i * n + j] != 0.0 || ti[i * n + j] != 0.0)) {
                seen[j] = 1;
                reached++;
                todo[top++] = j;
            }
    }
    return reached == n;
}

/* Phase-linked phases of T (reference.py:145-169), relative to the median
   date, or to the strongest component when that one is below 1e-3 of the
   largest; components below that floor get phase 0. */
static void orc_phases(int n, int emi, orc_work *w, double *phi)
{
    double ur[ORC_MAX_DATES], ui[ORC_MAX_DATES];
    int col = 0;

    if (!emi) {
        memcpy(w->ar, w->cr, sizeof(double) * n * n);
        memcpy(w->ai, w->ci, sizeof(double) * n * n);
        orc_jacobi(n, w->ar, w->ai, w->vr, w->vi);
        for (int k = 1; k < n; k++)
            if (w->ar[k * n + k] >= w->ar[col * n + col])
                col = k;
    }
    else {
        /* |T|^+ with eigenvalues |w| < 1e-9 dropped (reference.py:151-156). */
        for (int p = 0; p < n * n; p++) {
            w->ar[p] = hypot(w->cr[p], w->ci[p]);
            w->ai[p] = 0.0;
            w->gi[p] = 0.0;
        }
        orc_jacobi(n, w->ar, w->ai, w->vr, w->vi);
        for (int k = 0; k < n; k++) {
            const double lam = w->ar[k * n + k];

            if (fabs(lam) >= 1e-9)
                for (int i = 0; i < n; i++)
                    for (int j = 0; j < n; j++)
                        w->gi[i * n + j] += w->vr[i * n + k] * w->vr[j * n + k] / lam;
        }
        /* M = |T|^+ o T, smallest eigenvector. */
        for (int p = 0; p < n * n; p++) {
            w->ar[p] = w->gi[p] * w->cr[p];
            w->ai[p] = w->gi[p] * w->ci[p];
        }
        orc_jacobi(n, w->ar, w->ai, w->vr, w->vi);
        for (int k = 1; k < n; k++)
            if (w->ar[k * n + k] < w->ar[col * n + col])
                col = k;
    }
    for (int k = 0; k < n; k++) {
        ur[k] = w->vr[k * n + col];
        ui[k] = w->vi[k * n + col];
    }
    {
        double top = 0.0, floor_, datum;
        int ref = n / 2;

        for (int k = 0; k < n; k++)
            top = fmax(top, hypot(ur[k], ui[k]));
        floor_ = 1e-3 * top;
        if (hypot(ur[ref], ui[ref]) <= floor_) {
            ref = 0;
            for (int k = 1; k < n; k++)
                if (hypot(ur[k], ui[k]) > hypot(ur[ref], ui[ref]))
                    ref = k;
        }
        datum = atan2(ui[ref], ur[ref]);
        for (int k = 0; k < n; k++)
            phi[k] = hypot(ur[k], ui[k]) > floor_ ? atan2(ui[k], ur[k]) - datum
                                                  : 0.0;
    }
}

/* reference.py:172-184 */
static double orc_goodness(int n, const double *tr, const double *ti,
                           const double *phi)
{
    double re = 0.0, im = 0.0;

    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            const double res = atan2(ti[i * n + j] + 0.0, tr[i * n + j] + 0.0) -
                               (phi[i] - phi[j]);

            re += cos(res);
            im += sin(res);
        }
    return hypot(re, im) / (0.5 * n * (n - 1));
}

typedef struct {
    orc_settings s;
    orc_kernel_constants k;
    double ks_crit, ad_sigma, ad_crit, tlog_crit;
} orc_ctx;

static void orc_pixel(const orc_ctx *c, const float *slc, const float *amp,
                      const unsigned char *valid, int W, int y, int x,
                      size_t out, size_t plane, double *coh, int *count,
                      double *pairs, double *phases, unsigned *mask,
                      int mask_words, orc_work *w)
{
    const int n = c->s.ndates, wa = c->s.win_az, wr = c->s.win_rg;
    const size_t centre = (size_t)(y + wa / 2) * W + x + wr / 2;
    const float *a = amp + centre * n;
    float mean_a = 0.0f, var_a = 0.0f;
    int looks = 0;

    if (mask)
        memset(mask + out * mask_words, 0, sizeof(unsigned) * mask_words);
    if (phases)
        for (int k = 0; k < n; k++)
            phases[out * n + k] = NAN;
    if (pairs)
        for (int p = 0; p < c->s.npairs; p++)
            pairs[p * plane + out] = NAN;
    coh[out] = NAN;
    if (!valid[centre]) {
        count[out] = -1;
        return;
    }
    if (c->s.test == 2 && c->s.shp_fp32)
        orc_logstats32(a, n, &mean_a, &var_a);

    memset(w->cr, 0, sizeof(double) * n * n);
    memset(w->ci, 0, sizeof(double) * n * n);
    for (int dy = 0; dy < wa; dy++)
        for (int dx = 0; dx < wr; dx++) {
            const size_t cand = (size_t)(y + dy) * W + x + dx;
            const float *b = amp + cand * n;
            const float *s = slc + cand * n * 2;
            int ok;

            if (!valid[cand])
                continue;
            if (c->s.shp_fp32) {
                if (c->s.test == 0)
                    ok = orc_ks32(a, b, n, c->k.ks_max);
                else if (c->s.test == 1)
                    ok = orc_ad32(a, b, n, &c->k);
                else {
                    float mean_b, var_b;

                    orc_logstats32(b, n, &mean_b, &var_b);
                    ok = orc_tlog32(mean_a, var_a, mean_b, var_b, n,
                                    c->k.tlog_crit);
                }
            }
            else {
                if (c->s.test == 0)
                    ok = orc_ks64(a, b, n, c->ks_crit);
                else if (c->s.test == 1)
                    ok = orc_ad64(a, b, n, c->ad_sigma) <= c->ad_crit;
                else
                    ok = orc_tlog64(a, b, n, c->tlog_crit);
            }
            if (!ok)
                continue;
            if (mask) {
                const int bit = dy * wr + dx;

                mask[out * mask_words + bit / 32] |= 1u << (bit % 32);
            }
            looks++;
            /* cov += s s^H (reference.py:255-256) */
            for (int i = 0; i < n; i++) {
                const double sir = s[2 * i], sii = s[2 * i + 1];

                for (int j = 0; j < n; j++) {
                    const double sjr = s[2 * j], sji = s[2 * j + 1];

                    w->cr[i * n + j] += sir * sjr + sii * sji;
                    w->ci[i * n + j] += sii * sjr - sir * sji;
                }
            }
        }
    count[out] = looks;
    if (looks < c->s.min_looks)
        return;

    /* Coherence matrix (reference.py:124-142). */
    {
        double diag[ORC_MAX_DATES];

        for (int i = 0; i < n; i++)
            diag[i] = sqrt(w->cr[i * n + i] / looks);
        for (int i = 0; i < n; i++) {
            for (int j = i + 1; j < n; j++) {
                const double dij = diag[i] * diag[j];
                double vr = 0.0, vi = 0.0;

                if (dij > 0) {
                    vr = w->cr[i * n + j] / looks / dij;
                    vi = w->ci[i * n + j] / looks / dij;
                    if (c->s.bias && looks > 1) {
                        const double m2 = vr * vr + vi * vi;
                        const double m2c = (looks * m2 - 1.0) / (looks - 1.0);
                        const double f = (m2 > 0 && m2c > 0) ? sqrt(m2c / m2) : 0.0;

                        vr *= f;
                        vi *= f;
                    }
                }
                w->cr[i * n + j] = vr;
                w->ci[i * n + j] = vi;
                w->cr[j * n + i] = vr;
                w->ci[j * n + i] = -vi;
            }
            w->cr[i * n + i] = 1.0;
            w->ci[i * n + i] = 0.0;
        }
    }
    if (pairs) {
        int p = 0;

        for (int i = 0; i < n - 1; i++)
            for (int j = i + 1; j < (c->s.pairs_all ? n : i + 2); j++, p++)
                pairs[p * plane + out] = hypot(w->cr[i * n + j], w->ci[i * n + j]);
    }
    if (c->s.bias && !orc_connected(n, w->cr, w->ci))
        return;
    {
        double phi[ORC_MAX_DATES];

        orc_phases(n, c->s.emi, w, phi);
        coh[out] = orc_goodness(n, w->cr, w->ci, phi);
        if (phases)
            for (int k = 0; k < n; k++)
                phases[out * n + k] = phi[k];
    }
}

/* Oracle over one padded strip. Outputs are row-major [rows][cols]; pairs
   has npairs planes; phases [rows][cols][N] (radians, relative to the
   reference date); mask [rows][cols][mask_words] SHP bits (bit dy*WR+dx).
   Any of pairs, phases, mask may be NULL. Returns 0, or -1 on bad
   arguments. */
int orc_strip(const orc_settings *s, const float *slc, const float *amp,
              const unsigned char *valid, int padded_rows, int padded_cols,
              int rows, int cols, double *coh, int *count, double *pairs,
              double *phases, unsigned *mask, int nthreads)
{
    orc_ctx c;
    const size_t plane = (size_t)rows * cols;
    const int mask_words = (s->win_az * s->win_rg + 31) / 32;

    if (s->ndates < 2 || s->ndates > ORC_MAX_DATES || s->win_az < 1 ||
        s->win_rg < 1 || !(s->win_az & 1) || !(s->win_rg & 1) ||
        padded_rows != rows + s->win_az - 1 ||
        padded_cols != cols + s->win_rg - 1)
        return -1;
    c.s = *s;
    orc_kernel_constants_for(s, &c.k);
    c.ks_crit = sqrt(-0.5 * log(s->alpha / 2.0)) * sqrt(2.0 / s->ndates);
    c.ad_sigma = orc_ad_sigma(s->ndates);
    c.ad_crit = orc_ad_critical(s->alpha);
    c.tlog_crit = orc_normal_quantile(s->alpha);

#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        orc_work w;

        orc_work_alloc(&w, s->ndates);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int y = 0; y < rows; y++)
            for (int x = 0; x < cols; x++)
                orc_pixel(&c, slc, amp, valid, padded_cols, y, x,
                          (size_t)y * cols + x, plane, coh, count, pairs,
                          phases, mask, mask_words, &w);
        orc_work_free(&w);
    }
    (void)nthreads;
    return 0;
}

/* The statistics themselves, for the known-answer tests of the oracle
   (reference.py's test_reference_statistics_match_scipy). */
double orc_ad_statistic(const float *a, const float *b, int n)
{
    return orc_ad64(a, b, n, orc_ad_sigma(n));
}

int orc_ks_accept(const float *a, const float *b, int n, double alpha)
{
    return orc_ks64(a, b, n, sqrt(-0.5 * log(alpha / 2.0)) * sqrt(2.0 / n));
}

double orc_ad_sigma_of(int n)
{
    return orc_ad_sigma(n);
}

/* Eigen-decomposition entry point for unit tests of the solver. */
void orc_hermitian_eigen(int n, double *ar, double *ai, double *vr, double *vi)
{
    orc_jacobi(n, ar, ai, vr, vi);
}
