/* Flat-earth / topographic phase and the strip preparation, on the device.
 *
 * Phase grid (geometry.c:161-254): for every node of a grid every 16 lines
 * and samples of the region, and every height level (one, or hmin, mid,
 * hmax), the ground point seen by the reference date is located on the
 * WGS84 ellipsoid raised by the height (Newton on the range-Doppler
 * equations, geometry.c:100-148), then every date's zero-Doppler time of
 * that point is found by Newton from its closest state vector
 * (geometry.c:33-71), orbits being interpolated by 8-point Lagrange
 * polynomials (orbit.c:324-346); the phase of date k is
 * 4 pi / lambda (R_k - R_ref). All FP64, one thread per grid node (its
 * height levels in turn, each starting from the previous level's point as
 * the reference does). The grid is small (a few thousand nodes for a large
 * region) and computed once per run.
 *
 * Strip preparation (main.c:52-127), one thread per padded-strip cell, from
 * raw I/Q planes of the strip's rows: a cell is valid when it lies in the
 * region, no date is NULL (NaN) or zero in both components, and its height
 * (when an elevation map is given) is not NULL; amplitudes sqrtf(I^2 + Q^2)
 * are rounded exactly as the reference's C (no contraction) and sorted
 * ascending (a bitonic network in registers; any correct sort gives the
 * same floats); with a geometry, date k is rotated by exp(i phase_k) in
 * double, phase_k interpolated from the grid bilinearly in line and sample
 * and quadratically in height (geometry.c:256-291), and rounded to float.
 * Invalid cells are zero.
 */
#include "tcoh_internal.h"

#include <math.h>
#include <vector>

namespace {

constexpr int GEO_STEP = 16;
constexpr int LAGRANGE = 8;
constexpr double SPEED_OF_LIGHT = 299792458.0;
constexpr double WGS84_A = 6378137.0;
constexpr double WGS84_B = 6356752.314245;

__device__ int g_geo_fault;

__device__ __forceinline__ double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

struct DevOrbit {
    int n;
    const double *t, *pos, *vel;
};

__device__ DevOrbit dev_orbit(const TcOrbitSet &o, int k)
{
    DevOrbit d;
    const int off = o.offset[k];

    d.n = o.count[k];
    d.t = o.t + off;
    d.pos = o.pos + 3 * off;
    d.vel = o.vel + 3 * off;
    return d;
}

__device__ void orbit_state(const DevOrbit &o, double t, double *pos, double *vel)
{
    int first = 0;

    while (first + LAGRANGE < o.n && o.t[first + LAGRANGE / 2] < t)
        first++;
    for (int k = 0; k < 3; k++)
        pos[k] = vel[k] = 0.0;
    for (int i = first; i < first + LAGRANGE; i++) {
        double w = 1.0;

        for (int j = first; j < first + LAGRANGE; j++)
            if (j != i)
                w *= (t - o.t[j]) / (o.t[i] - o.t[j]);
        for (int k = 0; k < 3; k++) {
            pos[k] += w * o.pos[3 * i + k];
            vel[k] += w * o.vel[3 * i + k];
        }
    }
}

/* false when the time falls outside the orbit */
__device__ bool zero_doppler(const DevOrbit &o, const double *p, double &tz)
{
    double t = o.t[0], best = -1.0;

    for (int i = 0; i < o.n; i++) {
        double d[3];

        for (int k = 0; k < 3; k++)
            d[k] = p[k] - o.pos[3 * i + k];
        const double dist = dot3(d, d);

        if (best < 0 || dist < best) {
            best = dist;
            t = o.t[i];
        }
    }
    for (int it = 0; it < 30; it++) {
        double s[3], v[3], d[3];

        orbit_state(o, t, s, v);
        for (int k = 0; k < 3; k++)
            d[k] = p[k] - s[k];
        const double dt = dot3(v, d) / dot3(v, v);

        t += dt;
        if (fabs(dt) < 1e-10)
            break;
    }
    tz = t;
    return !(t < o.t[0] || t > o.t[o.n - 1]);
}

__device__ double det3(const double (&m)[3][3])
{
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

/* Cramer's rule; false when singular */
__device__ bool solve3(const double (&a)[3][3], const double *b, double *x)
{
    const double det = det3(a);

    if (det == 0.0)
        return false;
    for (int c = 0; c < 3; c++) {
        double m[3][3];

        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++)
                m[r][q] = q == c ? b[r] : a[r][q];
        x[c] = det3(m) / det;
    }
    return true;
}

/* false when singular or not converged */
__device__ bool geolocate(const DevOrbit &o, double t, double range, double h, bool have_guess,
                          double *p)
{
    const double a = WGS84_A + h, b = WGS84_B + h;
    double s[3], v[3];

    orbit_state(o, t, s, v);
    if (!have_guess) {
        double right[3];
        const double rs = sqrt(dot3(s, s));

        right[0] = v[1] * s[2] - v[2] * s[1];
        right[1] = v[2] * s[0] - v[0] * s[2];
        right[2] = v[0] * s[1] - v[1] * s[0];
        const double nr = sqrt(dot3(right, right));
        const double ground = sqrt(fmax(range * range - (rs - a) * (rs - a), 0.0));

        for (int k = 0; k < 3; k++)
            p[k] = s[k] * a / rs + right[k] / nr * ground;
    }
    for (int it = 0; it < 50; it++) {
        double d[3], jac[3][3], f[3], dx[3];

        for (int k = 0; k < 3; k++)
            d[k] = p[k] - s[k];
        const double dist = sqrt(dot3(d, d));

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
            return false;
        for (int k = 0; k < 3; k++)
            p[k] += dx[k];
        if (sqrt(dot3(dx, dx)) < 1e-6)
            return true;
    }
    return false;
}

__global__ void tc_geometry_grid_kernel(TcGeo g, TcOrbitSet orbits, double *grid)
{
    const int node = blockIdx.x * blockDim.x + threadIdx.x;

    if (node >= g.grid_rows * g.grid_cols)
        return;
    const int gr = node / g.grid_cols, gc = node - gr * g.grid_cols, n = g.ndates;
    const double line = g.line0 + (double)gr * GEO_STEP;
    const double t = g.first_line_time + line * g.azimuth_time_interval;
    const double sample = g.sample0 + (double)gc * GEO_STEP;
    const double range = 0.5 * SPEED_OF_LIGHT * (g.slant_range_time + sample / g.range_sampling_rate);
    const DevOrbit ref = dev_orbit(orbits, g.ref);
    double p[3] = {0.0, 0.0, 0.0};

    for (int hl = 0; hl < g.nheights; hl++) {
        double *ph = grid + ((size_t)node * g.nheights + hl) * n;
        double r_ref = 0.0;

        if (!geolocate(ref, t, range, g.heights[hl], hl > 0, p)) {
            atomicOr(&g_geo_fault, 1);
            return;
        }
        for (int k = 0; k < n; k++) {
            const DevOrbit o = dev_orbit(orbits, k);
            double tk, s[3], v[3], d[3];

            if (!zero_doppler(o, p, tk)) {
                atomicOr(&g_geo_fault, 2);
                return;
            }
            orbit_state(o, tk, s, v);
            for (int c = 0; c < 3; c++)
                d[c] = p[c] - s[c];
            ph[k] = sqrt(dot3(d, d));
            if (k == g.ref)
                r_ref = ph[k];
        }
        for (int k = 0; k < n; k++)
            ph[k] = 4.0 * M_PI / g.wavelength * (ph[k] - r_ref);
    }
}

/* Bitonic sort of NP floats in registers, ascending. */
template <int NP>
__device__ __forceinline__ void bitonic(float (&a)[NP])
{
#pragma unroll
    for (int k = 2; k <= NP; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < NP; i++) {
                const int l = i ^ j;

                if (l > i) {
                    const float x = a[i], y = a[l];
                    const bool up = (i & k) == 0;

                    a[i] = up ? fminf(x, y) : fmaxf(x, y);
                    a[l] = up ? fmaxf(x, y) : fminf(x, y);
                }
            }
}

/* Interpolated phase of date k at region cell (row, col) and height h. */
__device__ __forceinline__ double grid_phase(const TcGeo &g, const double *grid, int gr, int gc,
                                             double fr, double fc, const double (&wh)[3], int k)
{
    const int n = g.ndates;
    const size_t stride = (size_t)g.nheights * n;
    double ph = 0.0;

#pragma unroll
    for (int hl = 0; hl < 3; hl++) {
        if (hl >= g.nheights)
            break;
        const double *p00 = grid + (((size_t)gr * g.grid_cols + gc) * g.nheights + hl) * n;
        const double *p01 = p00 + stride;
        const double *p10 = p00 + (size_t)g.grid_cols * stride;
        const double *p11 = p10 + stride;

        ph += wh[hl] * ((1.0 - fr) * ((1.0 - fc) * p00[k] + fc * p01[k]) +
                        fr * ((1.0 - fc) * p10[k] + fc * p11[k]));
    }
    return ph;
}

/* One thread per strip cell; the outputs are pixel-major ([pixel][date]),
   so each warp stages its 32 pixels' amplitudes, then their samples, in
   shared memory (row stride n | 1, conflict-free for the 4-byte
   amplitudes) and writes them out as one contiguous run. */
template <int NP>
__global__ void __launch_bounds__(256, NP <= 32 ? 3 : 1)
tc_prep_raw_kernel(int n, const float *__restrict__ re, const float *__restrict__ im,
                   const double *__restrict__ elev, int row0, int region_rows, int padded_rows,
                   int cols, int halo, int use_geo, TcGeo g, const double *__restrict__ grid,
                   const double *__restrict__ dh, const float *__restrict__ psi,
                   float2 *__restrict__ slc, float *__restrict__ amp,
                   unsigned char *__restrict__ valid)
{
    extern __shared__ float2 prep_stage[];
    const int W = cols + 2 * halo, ld = n | 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long total = (long long)padded_rows * W;
    const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long wpix = pix - lane;
    const int wcount = (int)min(32LL, total - wpix);
    float2 *wb = prep_stage + warp * 32 * ld;
    float *wa = (float *)wb;
    const bool live = pix < total;
    const int r = (int)(pix / W), c = (int)(pix - (long long)r * W) - halo, row = row0 + r;
    const size_t plane = (size_t)padded_rows * cols;
    const size_t at = (size_t)r * cols + c;
    bool ok = live && row >= 0 && row < region_rows && c >= 0 && c < cols;
    float a[NP];

    if (wcount <= 0)
        return; /* the whole warp lies past the strip */
    if (ok && elev && isnan(elev[at]))
        ok = false;
#pragma unroll
    for (int k = 0; k < NP; k++) {
        a[k] = INFINITY;
        if (k < n && ok) {
            const float vi = re[k * plane + at], vq = im[k * plane + at];

            if (isnan(vi) || isnan(vq) || (vi == 0.f && vq == 0.f))
                ok = false;
            /* rounded as the reference's C: no contraction */
            a[k] = sqrtf(__fadd_rn(__fmul_rn(vi, vi), __fmul_rn(vq, vq)));
        }
    }
    if (live)
        valid[pix] = ok ? 1 : 0;
    if (ok)
        bitonic<NP>(a);
#pragma unroll
    for (int k = 0; k < NP; k++)
        if (k < n)
            wa[lane * ld + k] = ok ? a[k] : 0.f;
    __syncwarp();
    for (int e = lane; e < wcount * n; e += 32) {
        const int p = e / n;

        amp[wpix * n + e] = wa[p * ld + (e - p * n)];
    }
    __syncwarp();
    if (!ok) {
        for (int k = 0; k < n; k++)
            wb[lane * ld + k] = make_float2(0.f, 0.f);
    }
    else if (!use_geo && !psi) {
        for (int k = 0; k < n; k++)
            wb[lane * ld + k] = make_float2(re[k * plane + at], im[k * plane + at]);
    }
    else {
        const int gr = row / GEO_STEP, gc = c / GEO_STEP;
        const double fr = (double)(row - gr * GEO_STEP) / GEO_STEP;
        const double fc = (double)(c - gc * GEO_STEP) / GEO_STEP;
        /* the adjoint's variables: a height error and a phase screen */
        const double h = (elev ? elev[at] : g.h0) + (dh ? dh[at] : 0.0);
        double wh[3] = {1.0, 0.0, 0.0};

        if (use_geo && g.nheights == 3) {
            const double *x = g.heights;

            wh[0] = (h - x[1]) * (h - x[2]) / ((x[0] - x[1]) * (x[0] - x[2]));
            wh[1] = (h - x[0]) * (h - x[2]) / ((x[1] - x[0]) * (x[1] - x[2]));
            wh[2] = (h - x[0]) * (h - x[1]) / ((x[2] - x[0]) * (x[2] - x[1]));
        }
        for (int k = 0; k < n; k++) {
            const double ph = (use_geo ? grid_phase(g, grid, gr, gc, fr, fc, wh, k) : 0.0) +
                              (psi ? (double)psi[k * plane + at] : 0.0);
            double sn, cs;

            sincos(ph, &sn, &cs);
            const double vr = re[k * plane + at], vi = im[k * plane + at];

            /* (vr cs - vi sn, vr sn + vi cs) in double without contraction,
               as main.c:117-121, then rounded to float */
            wb[lane * ld + k] = make_float2((float)__dadd_rn(__dmul_rn(vr, cs), -__dmul_rn(vi, sn)),
                                            (float)__dadd_rn(__dmul_rn(vr, sn), __dmul_rn(vi, cs)));
        }
    }
    __syncwarp();
    for (int e = lane; e < wcount * n; e += 32) {
        const int p = e / n;

        slc[wpix * n + e] = wb[p * ld + (e - p * n)];
    }
}

template <int NP>
cudaError_t launch_prep_raw(unsigned blocks, int n, const float *re, const float *im,
                            const double *elev, int row0, int region_rows, int padded_rows,
                            int cols, int halo, int use, const TcGeo &g, const double *grid,
                            const double *dh, const float *psi, float2 *s, float *amp,
                            unsigned char *valid, cudaStream_t st)
{
    const int bytes = 8 * 32 * (n | 1) * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(tc_prep_raw_kernel<NP>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);

    if (e != cudaSuccess)
        return e;
    tc_prep_raw_kernel<NP><<<blocks, 256, bytes, st>>>(n, re, im, elev, row0, region_rows,
                                                      padded_rows, cols, halo, use, g, grid, dh,
                                                      psi, s, amp, valid);
    return cudaGetLastError();
}

} // namespace

int tc_geometry_shape(const struct tc_geometry &in, TcGeo &g)
{
    if (in.ndates < 2 || in.ndates > TC_MAX_DATES || in.ref < 0 || in.ref >= in.ndates)
        return tc_error(TC_ERR_ARG, "geometry: %d dates, reference date %d", in.ndates, in.ref);
    if (in.rows < 1 || in.cols < 1)
        return tc_error(TC_ERR_ARG, "geometry: empty region %d x %d", in.rows, in.cols);
    if (!(in.wavelength > 0.0) || !(in.range_sampling_rate > 0.0) ||
        !(in.azimuth_time_interval > 0.0))
        return tc_error(TC_ERR_ARG, "geometry: wavelength, range sampling rate and azimuth "
                        "time interval must be positive");
    if (!(in.hmax >= in.hmin))
        return tc_error(TC_ERR_ARG, "geometry: height range %g .. %g", in.hmin, in.hmax);
    g.ndates = in.ndates;
    g.ref = in.ref;
    g.grid_rows = (in.rows - 1) / GEO_STEP + 2;
    g.grid_cols = (in.cols - 1) / GEO_STEP + 2;
    if (in.hmax - in.hmin < 1.0) {
        g.nheights = 1;
        g.heights[0] = 0.5 * (in.hmin + in.hmax);
        g.heights[1] = g.heights[2] = 0.0;
    }
    else {
        g.nheights = 3;
        g.heights[0] = in.hmin;
        g.heights[1] = 0.5 * (in.hmin + in.hmax);
        g.heights[2] = in.hmax;
    }
    g.first_line_time = in.first_line_time;
    g.azimuth_time_interval = in.azimuth_time_interval;
    g.slant_range_time = in.slant_range_time;
    g.range_sampling_rate = in.range_sampling_rate;
    g.wavelength = in.wavelength;
    g.line0 = in.line0;
    g.sample0 = in.sample0;
    g.h0 = in.h0;
    return TC_OK;
}

int tc_geometry_grid(const TcGeo &g, const struct tc_orbit *orbits, double *grid_host,
                     cudaStream_t st)
{
    const int n = g.ndates;
    std::vector<int> count(n), offset(n);
    int total = 0;

    for (int k = 0; k < n; k++) {
        const struct tc_orbit &o = orbits[k];

        if (o.n < LAGRANGE || !o.t || !o.pos || !o.vel)
            return tc_error(TC_ERR_ARG, "orbit of date %d: %d state vectors, at least %d needed",
                            k, o.n, LAGRANGE);
        for (int i = 1; i < o.n; i++)
            if (!(o.t[i] > o.t[i - 1]))
                return tc_error(TC_ERR_ARG, "orbit of date %d: state vector times not "
                                "increasing at %d", k, i);
        count[k] = o.n;
        offset[k] = total;
        total += o.n;
    }
    const size_t nodes = (size_t)g.grid_rows * g.grid_cols;
    const size_t grid_bytes = nodes * g.nheights * n * sizeof(double);
    double *d_t = nullptr, *d_pos = nullptr, *d_vel = nullptr, *d_grid = nullptr;
    int *d_count = nullptr, *d_off = nullptr;
    cudaError_t e = cudaSuccess;
    int rc = TC_OK, fault = 0;
    const int zero = 0;

#define GEO_CK(call)                                                                     \
    do {                                                                                 \
        if (e == cudaSuccess)                                                            \
            e = (call);                                                                  \
    } while (0)
    GEO_CK(cudaMalloc(&d_t, total * sizeof(double)));
    GEO_CK(cudaMalloc(&d_pos, 3 * total * sizeof(double)));
    GEO_CK(cudaMalloc(&d_vel, 3 * total * sizeof(double)));
    GEO_CK(cudaMalloc(&d_count, n * sizeof(int)));
    GEO_CK(cudaMalloc(&d_off, n * sizeof(int)));
    GEO_CK(cudaMalloc(&d_grid, grid_bytes));
    for (int k = 0; k < n && e == cudaSuccess; k++) {
        GEO_CK(cudaMemcpyAsync(d_t + offset[k], orbits[k].t, count[k] * sizeof(double),
                               cudaMemcpyHostToDevice, st));
        GEO_CK(cudaMemcpyAsync(d_pos + 3 * offset[k], orbits[k].pos,
                               3 * count[k] * sizeof(double), cudaMemcpyHostToDevice, st));
        GEO_CK(cudaMemcpyAsync(d_vel + 3 * offset[k], orbits[k].vel,
                               3 * count[k] * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    GEO_CK(cudaMemcpyAsync(d_count, count.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    GEO_CK(cudaMemcpyAsync(d_off, offset.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    GEO_CK(cudaMemcpyToSymbolAsync(g_geo_fault, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                   st));
    if (e == cudaSuccess) {
        TcOrbitSet os;

        os.count = d_count;
        os.offset = d_off;
        os.t = d_t;
        os.pos = d_pos;
        os.vel = d_vel;
        tc_geometry_grid_kernel<<<(unsigned)((nodes + 127) / 128), 128, 0, st>>>(g, os, d_grid);
        e = cudaGetLastError();
    }
    GEO_CK(cudaMemcpyAsync(grid_host, d_grid, grid_bytes, cudaMemcpyDeviceToHost, st));
    GEO_CK(cudaMemcpyFromSymbolAsync(&fault, g_geo_fault, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                     st));
    GEO_CK(cudaStreamSynchronize(st));
#undef GEO_CK
    if (e != cudaSuccess)
        rc = tc_error(e == cudaErrorMemoryAllocation ? TC_ERR_MEMORY : TC_ERR_CUDA,
                      "geometry grid: %s", cudaGetErrorString(e));
    else if (fault & 2)
        rc = tc_error(TC_ERR_ARG, "A ground point is seen outside of an orbit's coverage: is "
                      "the stack coregistered on the reference date?");
    else if (fault & 1)
        rc = tc_error(TC_ERR_ARG, "Geolocation failed (singular geometry or no convergence)");
    cudaFree(d_t);
    cudaFree(d_pos);
    cudaFree(d_vel);
    cudaFree(d_count);
    cudaFree(d_off);
    cudaFree(d_grid);
    return rc;
}

cudaError_t tc_launch_prep_raw(int n, const float *re, const float *im, const double *elev,
                               int row0, int region_rows, int padded_rows, int cols, int halo,
                               const TcGeo *g, const double *grid, const double *dh,
                               const float *psi, float *slc, float *amp, unsigned char *valid,
                               cudaStream_t st)
{
    const long long cells = (long long)padded_rows * (cols + 2 * halo);
    const unsigned blocks = (unsigned)((cells + 255) / 256);
    const TcGeo none = {};
    const TcGeo &gg = g ? *g : none;
    const int use = g != nullptr;
    float2 *s = (float2 *)slc;

    if (n <= 8)
        return launch_prep_raw<8>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                  halo, use, gg, grid, dh, psi, s, amp, valid, st);
    if (n <= 16)
        return launch_prep_raw<16>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                   halo, use, gg, grid, dh, psi, s, amp, valid, st);
    if (n <= 32)
        return launch_prep_raw<32>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                   halo, use, gg, grid, dh, psi, s, amp, valid, st);
    return launch_prep_raw<64>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                               halo, use, gg, grid, dh, psi, s, amp, valid, st);
}
