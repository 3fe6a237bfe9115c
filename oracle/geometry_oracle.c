/* CPU oracle of the geometry and strip-preparation stages.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA strip
 * preparation is compared with; nothing in the product links or calls it.
 * It is called only from tests/ (through oracle/oracle.py).
 *
 * It restates in double-precision C:
 *   - the 8-point Lagrange orbit interpolation (orbit.c:324-346);
 *   - the zero-Doppler time of a ground point, Newton from the closest state
 *     vector (geometry.c:33-71);
 *   - the range-Doppler geolocation on the WGS84 ellipsoid raised by h,
 *     Newton with Cramer's rule (geometry.c:73-157);
 *   - the coarse phase grid, every 16 lines and samples, at one or three
 *     heights (geometry.c:161-254);
 *   - its bilinear-in-position, quadratic-in-height interpolation
 *     (geometry.c:256-291);
 *   - the strip preparation of main.c:52-127: validity (NULL or zero I/Q,
 *     NULL height), amplitudes sorted ascending before the rotation, and the
 *     rotation of date k by exp(i phase_k) in double precision.
 * Where the reference stops the program (G_fatal_error) these functions
 * return a negative code instead.
 *
 * Compiled without floating-point contraction (oracle/Makefile), as the
 * reference is on x86-64.
 */

#include <math.h>
#include <stddef.h>
#include <string.h>

#define GEO_C       299792458.0
#define GEO_A       6378137.0
#define GEO_B       6356752.314245
#define GEO_STEP    16
#define GEO_LAGR    8

/* One date's orbit: n state vectors. */
typedef struct {
    int n;
    const double *t;   /* n */
    const double *pos; /* n x 3 */
    const double *vel; /* n x 3 */
} orc_orbit;

/* Geometry of the reference date and the region. */
typedef struct {
    int ndates, ref;
    double first_line_time, azimuth_time_interval, slant_range_time;
    double range_sampling_rate, wavelength;
    double line0, sample0;
    int rows, cols;
    double hmin, hmax, h0;
} orc_geometry;

static double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* orbit.c:324-346 */
void orc_orbit_state(const orc_orbit *o, double t, double *pos, double *vel)
{
    int first = 0;

    while (first + GEO_LAGR < o->n && o->t[first + GEO_LAGR / 2] < t)
        first++;
    for (int k = 0; k < 3; k++)
        pos[k] = vel[k] = 0.0;
    for (int i = first; i < first + GEO_LAGR; i++) {
        double w = 1.0;

        for (int j = first; j < first + GEO_LAGR; j++)
            if (j != i)
                w *= (t - o->t[j]) / (o->t[i] - o->t[j]);
        for (int k = 0; k < 3; k++) {
            pos[k] += w * o->pos[3 * i + k];
            vel[k] += w * o->vel[3 * i + k];
        }
    }
}

/* geometry.c:33-71; -1 when the time falls outside the orbit. */
int orc_zero_doppler(const orc_orbit *o, const double *p, double *tz)
{
    double t = o->t[0], best = -1.0;

    for (int i = 0; i < o->n; i++) {
        double d[3], dist;

        for (int k = 0; k < 3; k++)
            d[k] = p[k] - o->pos[3 * i + k];
        dist = dot3(d, d);
        if (best < 0 || dist < best) {
            best = dist;
            t = o->t[i];
        }
    }
    for (int it = 0; it < 30; it++) {
        double s[3], v[3], d[3], dt;

        orc_orbit_state(o, t, s, v);
        for (int k = 0; k < 3; k++)
            d[k] = p[k] - s[k];
        dt = dot3(v, d) / dot3(v, v);
        t += dt;
        if (fabs(dt) < 1e-10)
            break;
    }
    *tz = t;
    return (t < o->t[0] || t > o->t[o->n - 1]) ? -1 : 0;
}

static double det3(double m[3][3])
{
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

/* geometry.c:73-98 */
static int solve3(double a[3][3], const double *b, double *x)
{
    const double det = det3(a);

    if (det == 0.0)
        return 0;
    for (int c = 0; c < 3; c++) {
        double m[3][3];

        memcpy(m, a, sizeof(m));
        for (int r = 0; r < 3; r++)
            m[r][c] = b[r];
        x[c] = det3(m) / det;
    }
    return 1;
}

/* geometry.c:100-148; -1 singular, -2 no convergence. */
int orc_geolocate(const orc_orbit *o, double t, double range, double h, int have_guess,
                  double *p)
{
    const double a = GEO_A + h, b = GEO_B + h;
    double s[3], v[3];

    orc_orbit_state(o, t, s, v);
    if (!have_guess) {
        double rs = sqrt(dot3(s, s)), right[3], nr, ground;

        right[0] = v[1] * s[2] - v[2] * s[1];
        right[1] = v[2] * s[0] - v[0] * s[2];
        right[2] = v[0] * s[1] - v[1] * s[0];
        nr = sqrt(dot3(right, right));
        ground = sqrt(fmax(range * range - (rs - a) * (rs - a), 0.0));
        for (int k = 0; k < 3; k++)
            p[k] = s[k] * a / rs + right[k] / nr * ground;
    }
    for (int it = 0; it < 50; it++) {
        double d[3], jac[3][3], f[3], dx[3], dist;

        for (int k = 0; k < 3; k++)
            d[k] = p[k] - s[k];
        dist = sqrt(dot3(d, d));
        f[0] = -dot3(v, d);
        f[1] = -(dist - range);
        f[2] = -((p[0] * p[0] + p[1] * p[1]) / (a * a) + p[2] * p[2] / (b * b) - 1.0);
        for (int k = 0; k < 3; k++) {
            jac[0][k] = v[k];
            jac[1][k] = d[k] / dist;
        }
        jac[2][0] = 2.0 * p[0] / (a * a);
        jac[2][1] = 2.0 * p[1] / (a * a);
        jac[2][2] = 2.0 * p[2] / (b * b);
        if (!solve3(jac, f, dx))
            return -1;
        for (int k = 0; k < 3; k++)
            p[k] += dx[k];
        if (sqrt(dot3(dx, dx)) < 1e-6)
            return 0;
    }
    return -2;
}

/* Grid shape and height levels (geometry.c:201-216). */
void orc_geometry_shape(const orc_geometry *g, int *grid_rows, int *grid_cols, int *nheights,
                        double *heights)
{
    *grid_rows = (g->rows - 1) / GEO_STEP + 2;
    *grid_cols = (g->cols - 1) / GEO_STEP + 2;
    if (g->hmax - g->hmin < 1.0) {
        *nheights = 1;
        heights[0] = 0.5 * (g->hmin + g->hmax);
        heights[1] = heights[2] = 0.0;
    }
    else {
        *nheights = 3;
        heights[0] = g->hmin;
        heights[1] = 0.5 * (g->hmin + g->hmax);
        heights[2] = g->hmax;
    }
}

/* The phase grid [grid_rows][grid_cols][nheights][ndates] (geometry.c:218-254).
   Returns 0, -1 (geolocation failed) or -2 (a point outside an orbit). */
int orc_geometry_grid(const orc_geometry *g, const orc_orbit *orbits, double *grid)
{
    const int n = g->ndates;
    int gr_n, gc_n, nh;
    double hs[3];

    orc_geometry_shape(g, &gr_n, &gc_n, &nh, hs);
    for (int gr = 0; gr < gr_n; gr++) {
        const double line = g->line0 + (double)gr * GEO_STEP;
        const double t = g->first_line_time + line * g->azimuth_time_interval;

        for (int gc = 0; gc < gc_n; gc++) {
            const double sample = g->sample0 + (double)gc * GEO_STEP;
            const double range =
                0.5 * GEO_C * (g->slant_range_time + sample / g->range_sampling_rate);
            double p[3];

            for (int hl = 0; hl < nh; hl++) {
                double *ph = grid + (((size_t)gr * gc_n + gc) * nh + hl) * n;
                double r_ref = 0.0;

                if (orc_geolocate(&orbits[g->ref], t, range, hs[hl], hl > 0, p) < 0)
                    return -1;
                for (int k = 0; k < n; k++) {
                    double s[3], v[3], d[3], tk;

                    if (orc_zero_doppler(&orbits[k], p, &tk) < 0)
                        return -2;
                    orc_orbit_state(&orbits[k], tk, s, v);
                    for (int c = 0; c < 3; c++)
                        d[c] = p[c] - s[c];
                    ph[k] = sqrt(dot3(d, d));
                    if (k == g->ref)
                        r_ref = ph[k];
                }
                for (int k = 0; k < n; k++)
                    ph[k] = 4.0 * M_PI / g->wavelength * (ph[k] - r_ref);
            }
        }
    }
    return 0;
}

/* geometry.c:256-291 */
void orc_geometry_phases(const orc_geometry *g, const double *grid, int row, int col, double h,
                         double *phase)
{
    const int n = g->ndates;
    int gr_n, gc_n, nh;
    double hs[3], wh[3] = {1.0, 0.0, 0.0};

    orc_geometry_shape(g, &gr_n, &gc_n, &nh, hs);
    const int gr = row / GEO_STEP, gc = col / GEO_STEP;
    const double fr = (double)(row - gr * GEO_STEP) / GEO_STEP;
    const double fc = (double)(col - gc * GEO_STEP) / GEO_STEP;

    if (nh == 3) {
        const double *x = hs;

        wh[0] = (h - x[1]) * (h - x[2]) / ((x[0] - x[1]) * (x[0] - x[2]));
        wh[1] = (h - x[0]) * (h - x[2]) / ((x[1] - x[0]) * (x[1] - x[2]));
        wh[2] = (h - x[0]) * (h - x[1]) / ((x[2] - x[0]) * (x[2] - x[1]));
    }
    for (int k = 0; k < n; k++)
        phase[k] = 0.0;
    for (int hl = 0; hl < nh; hl++) {
        const size_t stride = (size_t)nh * n;
        const double *p00 = grid + (((size_t)gr * gc_n + gc) * nh + hl) * n;
        const double *p01 = p00 + stride;
        const double *p10 = p00 + (size_t)gc_n * stride;
        const double *p11 = p10 + stride;

        for (int k = 0; k < n; k++)
            phase[k] += wh[hl] * ((1.0 - fr) * ((1.0 - fc) * p00[k] + fc * p01[k]) +
                                  fr * ((1.0 - fc) * p10[k] + fc * p11[k]));
    }
}

/* main.c:52-127: the padded strip of region rows row0 .. row0 + padded_rows
   - 1 from raw I/Q planes re, im [ndates][padded_rows][cols] (rows outside
   the region are ignored), with halo_cols invalid columns on each side.
   elevation [padded_rows][cols] or NULL; g and grid NULL for no geometry.
   Outputs slc [padded_rows][cols + 2 halo][n][2], amp [..][n], valid. */
void orc_prepare_strip(int n, const float *re, const float *im, const double *elevation,
                       int row0, int region_rows, int padded_rows, int cols, int halo_cols,
                       const orc_geometry *g, const double *grid, float *slc, float *amp,
                       unsigned char *valid)
{
    const int W = cols + 2 * halo_cols;
    const size_t npad = (size_t)padded_rows * W;
    double phase[64];

    memset(valid, 0, npad);
    memset(slc, 0, npad * n * 2 * sizeof(float));
    memset(amp, 0, npad * n * sizeof(float));
    for (int r = 0; r < padded_rows; r++) {
        const int row = row0 + r;

        if (row < 0 || row >= region_rows)
            continue;
        for (int c = 0; c < cols; c++) {
            const size_t pix = (size_t)r * W + halo_cols + c;
            float *s = slc + pix * n * 2;
            float *a = amp + pix * n;
            int ok = 1;

            for (int k = 0; k < n; k++) {
                const float vi = re[((size_t)k * padded_rows + r) * cols + c];
                const float vq = im[((size_t)k * padded_rows + r) * cols + c];

                if (isnan(vi) || isnan(vq) || (vi == 0.0f && vq == 0.0f))
                    ok = 0;
                s[2 * k] = vi;
                s[2 * k + 1] = vq;
            }
            if (elevation && isnan(elevation[(size_t)r * cols + c]))
                ok = 0;
            if (!ok) {
                memset(s, 0, (size_t)n * 2 * sizeof(float));
                continue;
            }
            valid[pix] = 1;
            for (int k = 0; k < n; k++) {
                const float v = sqrtf(s[2 * k] * s[2 * k] + s[2 * k + 1] * s[2 * k + 1]);
                int j = k;

                while (j > 0 && a[j - 1] > v) {
                    a[j] = a[j - 1];
                    j--;
                }
                a[j] = v;
            }
            if (g) {
                orc_geometry_phases(g, grid, row, c,
                                    elevation ? elevation[(size_t)r * cols + c] : g->h0, phase);
                for (int k = 0; k < n; k++) {
                    const double cs = cos(phase[k]), sn = sin(phase[k]);
                    const double vr = s[2 * k], vi = s[2 * k + 1];

                    s[2 * k] = (float)(vr * cs - vi * sn);
                    s[2 * k + 1] = (float)(vr * sn + vi * cs);
                }
            }
        }
    }
}
