/* Flat-earth / topographic phase and the strip preparation, on the device.
 *
 * Phase grid (what geometry.c:161-254 computes): for every node of a grid
 * every 16 lines and samples of the region and every height level (one, or
 * hmin, mid, hmax), the ground point that the reference date sees at the
 * node's azimuth time and slant range on the WGS84 ellipsoid raised by the
 * height, then every date's slant range to that point at its own
 * zero-Doppler time; the phase of date k is 4 pi / lambda (R_k - R_ref).
 * All in double precision, one warp per grid node:
 *
 * - orbits: each date's state vectors, interpolated by the polynomial of
 *   degree 7 through the 8 vectors around the time (the window of
 *   orbit.c:326-346), evaluated by Neville's scheme on the offsets from
 *   the window's middle vector, with the time derivative of the velocity;
 * - ground point (lanes 0 .. nheights - 1, one height level each): in the
 *   zero-Doppler plane of the reference orbit the point is
 *   s + R (cos a e1 + sin a e2), e1 pointing down, e2 to the right of the
 *   track, so that the Doppler and range equations hold by construction;
 *   the look angle a solves the ellipsoid equation by Newton's method from
 *   the law-of-cosines angle of a spherical Earth of the local radius;
 * - zero-Doppler times (the lanes over height levels x dates): the root of
 *   f(t) = v(t) . (p - s(t)) lies between the state vector nearest to p and
 *   its neighbour across the sign change of f; Newton's method from the
 *   secant point of that bracket, with f'(t) = v'(t) . (p - s(t)) - |v(t)|^2,
 *   converges quadratically. A point whose root is not bracketed inside the
 *   orbit is outside its coverage (the reference's fatal error).
 *
 * The grid is small (a few thousand nodes for a large region) and computed
 * once per run. For the strip preparation it is turned into coefficient
 * form (tc_launch_geometry_coef): per node and date the quadratic in height
 * through the three levels, so that a cell's phase is one bilinear blend of
 * three coefficients and a Horner step (TcGridCell).
 *
 * Strip preparation (main.c:52-127), one thread per padded-strip cell, from
 * raw I/Q planes of the strip's rows: a cell is valid when it lies in the
 * region, no date is NULL (NaN) or zero in both components, and its height
 * (when an elevation map is given) is not NULL; amplitudes sqrtf(I^2 + Q^2)
 * are rounded exactly as the reference's C (no contraction) and sorted
 * ascending (a bitonic network in registers; any correct sort gives the
 * same floats); with a geometry, date k is rotated by exp(i phase_k) in
 * double, phase_k interpolated from the grid at the cell's line, sample and
 * height, and rounded to float. Invalid cells are zero.
 */
#include "tcoh_internal.h"

#include <math.h>
#include <vector>

namespace {

constexpr int LAGRANGE = 8;       /* state vectors per interpolation window */
constexpr int GRID_WARPS = 4;     /* grid nodes per CTA */
constexpr double SPEED_OF_LIGHT = 299792458.0;
constexpr double WGS84_A = 6378137.0;
constexpr double WGS84_B = 6356752.314245;
constexpr unsigned FULL = 0xffffffffu;

__device__ int g_geo_fault;

struct V3 {
    double x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 operator*(double k, V3 a) { return v3(k * a.x, k * a.y, k * a.z); }
__host__ __device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ V3 unit(V3 a) { return (1.0 / sqrt(dot(a, a))) * a; }

/* One date's orbit: nsv state vectors, times increasing. */
struct Orbit {
    int nsv;
    const double *t, *pos, *vel; /* [nsv], [nsv][3], [nsv][3] */
};

__host__ __device__ __forceinline__ Orbit orbit_of(const TcOrbitSet &o, int k)
{
    const int off = o.offset[k];

    return {o.count[k], o.t + off, o.pos + 3 * off, o.vel + 3 * off};
}

__host__ __device__ __forceinline__ V3 row3(const double *a, int i)
{
    return v3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
}

struct State {
    V3 pos, vel, acc; /* acc: time derivative of the interpolated velocity */
};

/* First state vector of the interpolation window at time tt: LAGRANGE / 2
   vectors before the first one at or after tt, kept inside the orbit. */
__host__ __device__ int window_start(const Orbit &o, double tt)
{
    int lo = 0, hi = o.nsv;

    while (lo < hi) {
        const int mid = (lo + hi) >> 1;

        if (o.t[mid] < tt)
            lo = mid + 1;
        else
            hi = mid;
    }
    const int f = lo - LAGRANGE / 2;

    return f < 0 ? 0 : (f > o.nsv - LAGRANGE ? o.nsv - LAGRANGE : f);
}

/* Neville's scheme on the window's 8 points (times dt[i] relative to the
   evaluation time) for the values y, and the derivative when d is set. */
__host__ __device__ __forceinline__ double neville(const double (&dt)[LAGRANGE], double (&y)[LAGRANGE],
                                          double *d)
{
    double dy[LAGRANGE];

#pragma unroll
    for (int i = 0; i < LAGRANGE; i++)
        dy[i] = 0.0;
#pragma unroll
    for (int m = 1; m < LAGRANGE; m++)
#pragma unroll
        for (int i = 0; i + m < LAGRANGE; i++) {
            /* P_i,i+m(t) = ((t - t_i+m) P_i,i+m-1 + (t_i - t) P_i+1,i+m) / (t_i - t_i+m) */
            const double r = 1.0 / (dt[i] - dt[i + m]);

            if (d)
                dy[i] = (y[i] - y[i + 1] - dt[i + m] * dy[i] + dt[i] * dy[i + 1]) * r;
            y[i] = (dt[i] * y[i + 1] - dt[i + m] * y[i]) * r;
        }
    if (d)
        *d = dy[0];
    return y[0];
}

__host__ __device__ State orbit_state(const Orbit &o, double tt)
{
    const int f = window_start(o, tt), c = f + LAGRANGE / 2;
    double dt[LAGRANGE], y[LAGRANGE], out[6], der[3] = {0.0, 0.0, 0.0};

#pragma unroll
    for (int i = 0; i < LAGRANGE; i++)
        dt[i] = o.t[f + i] - tt;
#pragma unroll
    for (int comp = 0; comp < 6; comp++) {
        const double *src = comp < 3 ? o.pos : o.vel;
        const int q = comp % 3;
        /* offsets from the window's middle vector */
        const double base = src[3 * c + q];

#pragma unroll
        for (int i = 0; i < LAGRANGE; i++)
            y[i] = src[3 * (f + i) + q] - base;
        out[comp] = base + neville(dt, y, comp < 3 ? nullptr : der + q);
    }
    return {v3(out[0], out[1], out[2]), v3(out[3], out[4], out[5]), v3(der[0], der[1], der[2])};
}

/* Ground point at height h seen at slant range R from the state st (the
   reference orbit at the node's azimuth time), right-looking; false when
   Newton's method on the look angle does not settle. */
__host__ __device__ bool ground_point(const State &st, double R, double h, V3 &p)
{
    const double a = WGS84_A + h, b = WGS84_B + h;
    const double ia2 = 1.0 / (a * a), ib2 = 1.0 / (b * b);
    const V3 s = st.pos, v = st.vel;
    const V3 e1 = unit((dot(s, v) / dot(v, v)) * v - s); /* down, in the plane */
    const V3 e2 = unit(cross(v, s));                       /* right of the track */
    const double rho2 = dot(s, s);
    /* a sphere of the ellipsoid's radius below the satellite */
    const double z2 = s.z * s.z / rho2;
    const double re2 = a * a * b * b / (b * b * (1.0 - z2) + a * a * z2);
    const double c0 = (rho2 + R * R - re2) / (2.0 * sqrt(rho2) * R);
    double ang = acos(fmin(fmax(c0, -1.0), 1.0));

    for (int it = 0; it < 40; it++) {
        double sn, cs;

        sincos(ang, &sn, &cs);
        p = s + R * (cs * e1 + sn * e2);
        const V3 dp = R * (cs * e2 - sn * e1);
        const double F = (p.x * p.x + p.y * p.y) * ia2 + p.z * p.z * ib2 - 1.0;
        const double dF = 2.0 * ((p.x * dp.x + p.y * dp.y) * ia2 + p.z * dp.z * ib2);

        if (!(dF != 0.0))
            return false;
        const double step = F / dF;

        ang -= step;
        if (fabs(step) * R < 1e-8) {
            sincos(ang, &sn, &cs);
            p = s + R * (cs * e1 + sn * e2);
            return true;
        }
    }
    return false;
}

/* v . (p - s) at state vector i: positive before the point is passed */
__host__ __device__ __forceinline__ double doppler_at(const Orbit &o, int i, V3 p)
{
    return dot(row3(o.vel, i), p - row3(o.pos, i));
}

/* Slant range from p to orbit o at its zero-Doppler time; false when that
   time is not bracketed inside the orbit or Newton's method stalls. */
__host__ __device__ bool zero_doppler_range(const Orbit &o, V3 p, double &range)
{
    int near = 0;
    double best = INFINITY;

    for (int i = 0; i < o.nsv; i++) {
        const V3 d = p - row3(o.pos, i);
        const double d2 = dot(d, d);

        if (d2 < best) {
            best = d2;
            near = i;
        }
    }
    const int lo = doppler_at(o, near, p) >= 0.0 ? near : near - 1, hi = lo + 1;

    if (lo < 0 || hi >= o.nsv)
        return false;
    const double flo = doppler_at(o, lo, p), fhi = doppler_at(o, hi, p);

    if (!(flo >= 0.0 && fhi <= 0.0))
        return false;
    double t = flo > fhi ? o.t[lo] + flo / (flo - fhi) * (o.t[hi] - o.t[lo]) : o.t[lo];

    for (int it = 0; it < 20; it++) {
        const State st = orbit_state(o, t);
        const V3 d = p - st.pos;
        const double f = dot(st.vel, d), df = dot(st.acc, d) - dot(st.vel, st.vel);

        if (!(df < 0.0))
            return false;
        const double step = f / df;

        t -= step;
        if (fabs(step) < 1e-9) {
            if (t < o.t[0] || t > o.t[o.nsv - 1])
                return false;
            const V3 e = p - orbit_state(o, t).pos;

            range = sqrt(dot(e, e));
            return true;
        }
    }
    return false;
}

/* One warp per grid node: ground points on lanes (one height level each),
   then the (level, date) ranges over the lanes, then the phases. */
__global__ void __launch_bounds__(32 * GRID_WARPS)
tc_geometry_grid_kernel(TcGeo g, TcOrbitSet orbits, double *grid)
{
    __shared__ double s_range[GRID_WARPS][3][TC_MAX_DATES];
    __shared__ V3 s_point[GRID_WARPS][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int node = blockIdx.x * GRID_WARPS + warp;

    if (node >= g.grid_rows * g.grid_cols)
        return; /* the whole warp */
    const int gr = node / g.grid_cols, gc = node - gr * g.grid_cols, n = g.ndates;
    const int items = g.nheights * n;
    const double tt =
        g.first_line_time + (g.line0 + (double)gr * TC_GEO_STEP) * g.azimuth_time_interval;
    const double R = 0.5 * SPEED_OF_LIGHT *
                     (g.slant_range_time + (g.sample0 + (double)gc * TC_GEO_STEP) /
                                               g.range_sampling_rate);
    bool ok = true;

    if (lane < g.nheights) {
        const State st = orbit_state(orbit_of(orbits, g.ref), tt);

        ok = ground_point(st, R, g.heights[lane], s_point[warp][lane]);
    }
    if (!__all_sync(FULL, ok)) {
        if (lane == 0)
            atomicOr(&g_geo_fault, 1);
        return;
    }
    __syncwarp();
    for (int q = lane; q < items; q += 32) {
        const int hl = q / n, k = q - hl * n;

        ok &= zero_doppler_range(orbit_of(orbits, k), s_point[warp][hl], s_range[warp][hl][k]);
    }
    if (!__all_sync(FULL, ok)) {
        if (lane == 0)
            atomicOr(&g_geo_fault, 2);
        return;
    }
    __syncwarp();
    const double scale = 4.0 * M_PI / g.wavelength;

    for (int q = lane; q < items; q += 32) {
        const int hl = q / n, k = q - hl * n;

        grid[(size_t)node * items + q] = scale * (s_range[warp][hl][k] - s_range[warp][hl][g.ref]);
    }
}

/* Coefficient form (TcGridCell): one thread per node and date. With the
   levels h0 < h1 < h2 and their phases P0, P1, P2, the Newton form about
   h1 gives phase(h) = P1 + u (d12 - (h2 - h1) d012) + u^2 d012, u = h - h1,
   d12 and d012 the first and second divided differences. */
__global__ void tc_geometry_coef_kernel(TcGeo g, const double *__restrict__ grid,
                                        double *__restrict__ coef)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.ndates;

    if (q >= (long long)g.grid_rows * g.grid_cols * n)
        return;
    const long long node = q / n;
    const int k = (int)(q - node * n);
    double *out = coef + 3 * q;

    if (g.nheights == 3) {
        const double *P = grid + node * 3 * n + k;
        const double *h = g.heights;
        const double d01 = (P[n] - P[0]) / (h[1] - h[0]);
        const double d12 = (P[2 * n] - P[n]) / (h[2] - h[1]);
        const double d012 = (d12 - d01) / (h[2] - h[0]);

        out[0] = P[n];
        out[1] = d12 - (h[2] - h[1]) * d012;
        out[2] = d012;
    }
    else {
        out[0] = grid[node * n + k];
        out[1] = 0.0;
        out[2] = 0.0;
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

/* One thread per strip cell; the outputs are pixel-major ([pixel][date]),
   so each warp stages its 32 pixels' amplitudes, then their samples, in
   shared memory (row stride n | 1, conflict-free for the 4-byte
   amplitudes) and writes them out as one contiguous run. */
template <int NP>
__global__ void __launch_bounds__(256, NP <= 32 ? 3 : 1)
tc_prep_raw_kernel(int n, const float *__restrict__ re, const float *__restrict__ im,
                   const double *__restrict__ elev, int row0, int region_rows, int padded_rows,
                   int cols, int halo, long long cell0, long long cell1, int use_geo, TcGeo g,
                   const double *__restrict__ grid,
                   const double *__restrict__ dh, const float *__restrict__ psi,
                   float2 *__restrict__ slc, float *__restrict__ amp,
                   unsigned char *__restrict__ valid)
{
    extern __shared__ float2 prep_stage[];
    const int W = cols + 2 * halo, ld = n | 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long total = cell1;
    const long long pix = cell0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
        /* the adjoint's variables: a height error and a phase screen */
        const double h = (elev ? elev[at] : g.h0) + (dh ? dh[at] : 0.0);
        const TcGridCell cell = use_geo ? tc_grid_cell(g, grid, row, c, h) : TcGridCell{};

        for (int k = 0; k < n; k++) {
            const double ph = (use_geo ? cell.phase(k, nullptr) : 0.0) +
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
                            int cols, int halo, long long cell0, long long cell1, int use,
                            const TcGeo &g, const double *grid, const double *dh,
                            const float *psi, float2 *s, float *amp, unsigned char *valid,
                            cudaStream_t st)
{
    const int bytes = 8 * 32 * (n | 1) * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(tc_prep_raw_kernel<NP>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);

    if (e != cudaSuccess)
        return e;
    tc_prep_raw_kernel<NP><<<blocks, 256, bytes, st>>>(n, re, im, elev, row0, region_rows,
                                                      padded_rows, cols, halo, cell0, cell1, use,
                                                      g, grid, dh, psi, s, amp, valid);
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
    g.grid_rows = (in.rows - 1) / TC_GEO_STEP + 2;
    g.grid_cols = (in.cols - 1) / TC_GEO_STEP + 2;
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
        tc_geometry_grid_kernel<<<(unsigned)((nodes + GRID_WARPS - 1) / GRID_WARPS),
                                  32 * GRID_WARPS, 0, st>>>(g, os, d_grid);
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

cudaError_t tc_launch_geometry_coef(const TcGeo &g, const double *grid, double *coef,
                                    cudaStream_t st)
{
    const long long items = (long long)g.grid_rows * g.grid_cols * g.ndates;

    tc_geometry_coef_kernel<<<(unsigned)((items + 255) / 256), 256, 0, st>>>(g, grid, coef);
    return cudaGetLastError();
}

cudaError_t tc_launch_prep_raw(int n, const float *re, const float *im, const double *elev,
                               int row0, int region_rows, int padded_rows, int cols, int halo,
                               int prow0, int prow1, const TcGeo *g, const double *grid,
                               const double *dh, const float *psi, float *slc, float *amp,
                               unsigned char *valid, cudaStream_t st)
{
    const long long W = cols + 2 * halo;
    const long long cell0 = (long long)prow0 * W, cell1 = (long long)prow1 * W;
    const unsigned blocks = (unsigned)((cell1 - cell0 + 255) / 256);
    const TcGeo none = {};
    const TcGeo &gg = g ? *g : none;
    const int use = g != nullptr;
    float2 *s = (float2 *)slc;

    if (cell1 <= cell0)
        return cudaSuccess;
    if (n <= 8)
        return launch_prep_raw<8>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                  halo, cell0, cell1, use, gg, grid, dh, psi, s, amp, valid, st);
    if (n <= 16)
        return launch_prep_raw<16>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                   halo, cell0, cell1, use, gg, grid, dh, psi, s, amp, valid, st);
    if (n <= 32)
        return launch_prep_raw<32>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                                   halo, cell0, cell1, use, gg, grid, dh, psi, s, amp, valid, st);
    return launch_prep_raw<64>(blocks, n, re, im, elev, row0, region_rows, padded_rows, cols,
                               halo, cell0, cell1, use, gg, grid, dh, psi, s, amp, valid, st);
}
