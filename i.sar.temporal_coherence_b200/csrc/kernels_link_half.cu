/* Phase linking and temporal coherence for stacks of up to 32 dates: two
 * pixels per warp, one per 16-lane half.
 *
 * Lane l of a half owns rows l and l + 16 of its pixel's matrices, in
 * registers. The stages and their numerics are those of kernels_link.cu
 * (see there for the reference lines); this layout exists for speed: each
 * Householder step is gated by reductions and shared-memory round trips,
 * and with two pixels per warp (two rows per lane) every such latency and
 * every serial scalar computation serves two pixels, while the rank-2
 * updates of two rows per lane give the schedulers independent work.
 *
 * The Householder reduction runs in float. At step k the pivot column k of
 * a row sits in r[0] and its trailing columns k+1 .. n-1 in r[1 ..]; the
 * rank-2 update writes column j into r[j - 1], so register indices stay
 * static while k is a run-time loop (the code stays small). The Householder
 * vectors are parked in the lower triangle of T, which only mirrors the
 * upper one.
 *
 * EMI: |T| is inverted in double (Gauss-Jordan when every pivot exceeds
 * 1e-5; through |T|^2 when |T| is indefinite; Jacobi pseudo-inverse with the
 * absolute floor 1e-9 of tests/reference.py:151-156 when it is close to
 * singular). M = |T|^-1 o T is reduced in float. Where the gap of its two
 * smallest eigenvalues is small against its norm, the float eigenvector is
 * then refined in double: the residual r = M x - mu x (M and mu in double)
 * is mapped by the float Householder basis Q onto the tridiagonal, the
 * correction solves (tri - mu) t = Q^H r off the eigen-direction, and
 * x -= Q t; this step gives double accuracy whenever the float rounding of
 * M is small against that gap (one step squares the relative error).
 * Elsewhere the float eigen-solve adds less to gamma's error than the float
 * coherence sums do.
 */
#include "tcoh_internal.h"

#include <math.h>

#define FULL 0xffffffffu

/* EMI: refine the float eigenvector in double where the gap between M's
   two smallest eigenvalues is below this fraction of its norm. */
#ifndef TC_REFINE_GAP
#define TC_REFINE_GAP 0.005f
#endif
/* EMI: send a pixel to the exact tier where n max|inv| divided by M's
   relative eigengap exceeds this bound. */
#ifndef TC_EXACT_BOUND
#define TC_EXACT_BOUND 1.0e5
#endif

namespace {

struct Grp {
    int lane, gl, base;
    unsigned mask;
};

__device__ __forceinline__ Grp make_grp(int lane)
{
    Grp g;

    g.lane = lane;
    g.gl = lane & 15;
    g.base = lane & 16;
    g.mask = 0xFFFFu << g.base;
    return g;
}

template <typename T>
__device__ __forceinline__ T gsum(T v, const Grp &g)
{
#pragma unroll
    for (int o = 8; o; o >>= 1)
        v += __shfl_xor_sync(g.mask, v, o);
    return v;
}

__device__ __forceinline__ float gmaxf(float v, const Grp &g)
{
#pragma unroll
    for (int o = 8; o; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(g.mask, v, o));
    return v;
}

__device__ __forceinline__ float gminf(float v, const Grp &g)
{
#pragma unroll
    for (int o = 8; o; o >>= 1)
        v = fminf(v, __shfl_xor_sync(g.mask, v, o));
    return v;
}

__device__ __forceinline__ double gmaxd(double v, const Grp &g)
{
#pragma unroll
    for (int o = 8; o; o >>= 1)
        v = fmax(v, __shfl_xor_sync(g.mask, v, o));
    return v;
}

template <typename T>
__device__ __forceinline__ T gbcast(T v, int row, const Grp &g)
{
    return __shfl_sync(g.mask, v, g.base | (row & 15));
}

__device__ __forceinline__ void gsync(const Grp &g) { __syncwarp(g.mask); }

/* Per-group shared workspace (byte offsets, 16-byte aligned). */
struct HalfLayout {
    int n, ld;
    int off_T, off_G, off_vw, off_lu, off_tau, off_d, off_e, off_df, off_e2f, off_y,
        off_nrm, off_zs, off_rs, off_lam, off_x, off_Db;
    int per_group;
};

struct HWs {
    int n;
    float2 *T;
    double *G;
    float4 *vw;
    float4 *lu;
    float2 *tau;
    float *d, *e, *df, *e2f, *y, *nrm; /* nrm: 1 / sqrt(C_ii) */
    float2 *zs;
    double *rs, *lam;
    double2 *x; /* scratch vectors of the adjoint's solves (2 x 32) */
};

__device__ __forceinline__ HWs hws(unsigned char *base, const HalfLayout &L)
{
    HWs w;

    w.n = L.n;
    w.T = (float2 *)(base + L.off_T);
    w.G = (double *)(base + L.off_G);
    w.vw = (float4 *)(base + L.off_vw);
    w.lu = (float4 *)(base + L.off_lu);
    w.tau = (float2 *)(base + L.off_tau);
    w.d = (float *)(base + L.off_d);
    w.e = (float *)(base + L.off_e);
    w.df = (float *)(base + L.off_df);
    w.e2f = (float *)(base + L.off_e2f);
    w.y = (float *)(base + L.off_y);
    w.nrm = (float *)(base + L.off_nrm);
    w.zs = (float2 *)(base + L.off_zs);
    w.rs = (double *)(base + L.off_rs);
    w.lam = nullptr;
    w.x = (double2 *)(base + L.off_x);
    return w;
}

/* ------------------------------------------------------------------ */
/* Householder reduction of the group's matrix (rows in r0, r1).       */
/* ------------------------------------------------------------------ */

/* Norm of the sub-pivot part of the pivot column, the sub-diagonal and the
   diagonal of step k, from the pivot column values c0, c1 of rows i0, i1. */
struct StepHead {
    float xn2;
    float2 alpha;
    float dk;
};

__device__ __forceinline__ StepHead step_head(float2 c0, float2 c1, int k, int n, const Grp &g)
{
    const int i0 = g.gl, i1 = g.gl + 16;
    StepHead h;
    float x = (i0 >= k + 2 && i0 < n ? c0.x * c0.x + c0.y * c0.y : 0.f) +
              (i1 >= k + 2 && i1 < n ? c1.x * c1.x + c1.y * c1.y : 0.f);
    const float2 sa = k + 1 < 16 ? c0 : c1;

    h.alpha = make_float2(gbcast(sa.x, k + 1, g), gbcast(sa.y, k + 1, g));
    h.dk = gbcast(k < 16 ? c0.x : c1.x, k, g);
    h.xn2 = gsum(x, g);
    return h;
}

/* One element of the rank-2 update: t - (v conj(wj) + w conj(vj)), with
   nv = -v and nw = -w (four FMAs per component). */
__device__ __forceinline__ float2 r2(float2 t, float2 nv, float2 nw, float4 q)
{
    t.x = fmaf(nv.x, q.z, t.x);
    t.x = fmaf(nv.y, q.w, t.x);
    t.x = fmaf(nw.x, q.x, t.x);
    t.x = fmaf(nw.y, q.y, t.x);
    t.y = fmaf(nv.y, q.z, t.y);
    t.y = fmaf(-nv.x, q.w, t.y);
    t.y = fmaf(nw.y, q.x, t.y);
    t.y = fmaf(-nw.x, q.y, t.y);
    return t;
}

__device__ void householder(float2 (&r0)[32], float2 (&r1)[32], int n, const HWs &w, int ld,
                            const Grp &g)
{
    const int i0 = g.gl, i1 = g.gl + 16;

    /* Entries 32..63 stay zero: whole blocks of 4 columns may run past n. */
    w.vw[32 + g.gl] = make_float4(0.f, 0.f, 0.f, 0.f);
    w.vw[48 + g.gl] = make_float4(0.f, 0.f, 0.f, 0.f);
    StepHead hd = step_head(r0[0], r1[0], 0, n, g);

    for (int k = 0; k < n - 1; k++) {
        const int len = n - 1 - k;
        const float2 c0 = r0[0], c1 = r1[0];
        const float2 alpha = hd.alpha;
        const float xn2 = hd.xn2;
        float beta, tr = 0.f, ti = 0.f, sr = 0.f, si = 0.f;

        if (xn2 == 0.f && alpha.y == 0.f)
            beta = alpha.x;
        else {
            beta = -copysignf(sqrtf(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
            const float ib = __frcp_rn(beta);

            tr = (beta - alpha.x) * ib;
            ti = -alpha.y * ib;
            const float dr = alpha.x - beta, di = alpha.y;
            const float iden = __frcp_rn(dr * dr + di * di);

            sr = dr * iden;
            si = -di * iden;
        }
        const bool refl = !(tr == 0.f && ti == 0.f);
        float2 v0 = make_float2(0.f, 0.f), v1 = make_float2(0.f, 0.f);

        if (i0 == k + 1)
            v0 = make_float2(1.f, 0.f);
        else if (i0 > k + 1 && i0 < n)
            v0 = refl ? make_float2(c0.x * sr - c0.y * si, c0.x * si + c0.y * sr) : c0;
        if (i1 == k + 1)
            v1 = make_float2(1.f, 0.f);
        else if (i1 > k + 1 && i1 < n)
            v1 = refl ? make_float2(c1.x * sr - c1.y * si, c1.x * si + c1.y * sr) : c1;
        if (i0 > k && i0 < n)
            w.T[i0 * ld + k] = v0;
        if (i1 > k && i1 < n)
            w.T[i1 * ld + k] = v1;
        if (g.gl == 0) {
            w.d[k] = hd.dk;
            w.e[k] = beta;
            w.tau[k] = make_float2(tr, ti);
        }
        /* With tau = 0 the update below is an exact zero: only the shift. */
        ((float2 *)w.vw)[2 * i0] = v0;
        ((float2 *)w.vw)[2 * i1] = v1;
        gsync(g);
        const float4 *vwk = w.vw + k;
        float2 p0a = make_float2(0.f, 0.f), p0b = p0a, p1a = p0a, p1b = p0a;

#pragma unroll
        for (int jb = 1; jb < 32; jb += 4) {
            if (jb > len)
                break;
#pragma unroll
            for (int jj = jb; jj < jb + 4 && jj < 32; jj++) {
                const float2 vj = *(const float2 *)&vwk[jj];
                float2 &q0 = (jj & 1) ? p0b : p0a;
                float2 &q1 = (jj & 1) ? p1b : p1a;

                q0.x = fmaf(r0[jj].x, vj.x, fmaf(-r0[jj].y, vj.y, q0.x));
                q0.y = fmaf(r0[jj].x, vj.y, fmaf(r0[jj].y, vj.x, q0.y));
                q1.x = fmaf(r1[jj].x, vj.x, fmaf(-r1[jj].y, vj.y, q1.x));
                q1.y = fmaf(r1[jj].x, vj.y, fmaf(r1[jj].y, vj.x, q1.y));
            }
        }
        const float2 p0 = make_float2(p0a.x + p0b.x, p0a.y + p0b.y);
        const float2 p1 = make_float2(p1a.x + p1b.x, p1a.y + p1b.y);
        float2 w0 = make_float2(tr * p0.x - ti * p0.y, tr * p0.y + ti * p0.x);
        float2 w1 = make_float2(tr * p1.x - ti * p1.y, tr * p1.y + ti * p1.x);
        float pr = (i0 > k ? w0.x * v0.x + w0.y * v0.y : 0.f) +
                   (i1 > k ? w1.x * v1.x + w1.y * v1.y : 0.f);
        float pi = (i0 > k ? w0.x * v0.y - w0.y * v0.x : 0.f) +
                   (i1 > k ? w1.x * v1.y - w1.y * v1.x : 0.f);

        pr = gsum(pr, g);
        pi = gsum(pi, g);
        const float hr = -0.5f * (tr * pr - ti * pi), hi = -0.5f * (tr * pi + ti * pr);

        w0.x += hr * v0.x - hi * v0.y;
        w0.y += hr * v0.y + hi * v0.x;
        w1.x += hr * v1.x - hi * v1.y;
        w1.y += hr * v1.y + hi * v1.x;
        if (i0 <= k)
            w0 = make_float2(0.f, 0.f);
        if (i1 <= k)
            w1 = make_float2(0.f, 0.f);
        ((float2 *)w.vw)[2 * i0 + 1] = w0;
        ((float2 *)w.vw)[2 * i1 + 1] = w1;
        gsync(g);
        const float2 nv0 = make_float2(-v0.x, -v0.y), nv1 = make_float2(-v1.x, -v1.y);
        const float2 nw0 = make_float2(-w0.x, -w0.y), nw1 = make_float2(-w1.x, -w1.y);

        /* Column k + 1 first: it is the next pivot column, so the next
           step's reductions overlap the rest of this update. */
        {
            const float4 q = vwk[1];

            r0[0] = r2(r0[1], nv0, nw0, q);
            r1[0] = r2(r1[1], nv1, nw1, q);
        }
        hd = step_head(r0[0], r1[0], k + 1, n, g); /* unused after the last step */
#pragma unroll
        for (int jj = 2; jj < 6; jj++) {
            const float4 q = vwk[jj];

            r0[jj - 1] = r2(r0[jj], nv0, nw0, q);
            r1[jj - 1] = r2(r1[jj], nv1, nw1, q);
        }
#pragma unroll
        for (int jb = 6; jb < 32; jb += 4) {
            if (jb > len)
                break;
#pragma unroll
            for (int jj = jb; jj < jb + 4 && jj < 32; jj++) {
                const float4 q = vwk[jj];

                r0[jj - 1] = r2(r0[jj], nv0, nw0, q);
                r1[jj - 1] = r2(r1[jj], nv1, nw1, q);
            }
        }
        gsync(g);
    }
    {
        const float dl = gbcast(n - 1 < 16 ? r0[0].x : r1[0].x, n - 1, g);

        if (g.gl == 0)
            w.d[n - 1] = dl;
    }
    gsync(g);
}

/* ------------------------------------------------------------------ */
/* Tridiagonal eigenvector.                                            */
/* ------------------------------------------------------------------ */

/* x <- Q^H x (adjoint) or Q x, Q = H_0 H_1 .. H_{n-2}, H_k = I - tau_k v_k v_k^H
   (v_k in T's lower triangle, column k), on the group's rows (i0, i1).
   The reflectors go in blocks of four in application order; per block the
   four products v^H x and the six v_m^H v_j within the block are reduced
   over the group at once, then
       s_m = v_m^H x - sum_{j<m} (v_m^H v_j) h_j,  h_m = tau'_m s_m,
       x  -= sum_m v_m h_m
   (tau' = conj(tau) for Q^H), which is the sequential application
   rearranged. */
__device__ void apply_q(int n, int ld, const HWs &w, const Grp &g, bool adjoint, float2 &x0,
                        float2 &x1)
{
    const int i0 = g.gl, i1 = g.gl + 16, nk = n - 1;

    for (int b = 0; b < nk; b += 4) {
        float2 v0[4], v1[4], ta[4];

#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int pos = b + m, k = adjoint ? pos : nk - 1 - pos;
            const bool ok = pos < nk;
            const float2 t = ok ? w.tau[k] : make_float2(0.f, 0.f);

            ta[m] = adjoint ? make_float2(t.x, -t.y) : t;
            v0[m] = ok && i0 > k && i0 < n ? w.T[i0 * ld + k] : make_float2(0.f, 0.f);
            v1[m] = ok && i1 > k && i1 < n ? w.T[i1 * ld + k] : make_float2(0.f, 0.f);
        }
        /* r[2m], r[2m+1]: v_m^H x; r[8 + 2p], r[9 + 2p]: v_m^H v_j, pairs
           p = (1,0), (2,0), (2,1), (3,0), (3,1), (3,2) */
        float r[20];

#pragma unroll
        for (int m = 0; m < 4; m++) {
            r[2 * m] = v0[m].x * x0.x + v0[m].y * x0.y + v1[m].x * x1.x + v1[m].y * x1.y;
            r[2 * m + 1] = v0[m].x * x0.y - v0[m].y * x0.x + v1[m].x * x1.y - v1[m].y * x1.x;
        }
        {
            int p = 0;

#pragma unroll
            for (int m = 1; m < 4; m++)
#pragma unroll
                for (int j = 0; j < m; j++, p++) {
                    r[8 + 2 * p] = v0[m].x * v0[j].x + v0[m].y * v0[j].y + v1[m].x * v1[j].x +
                                   v1[m].y * v1[j].y;
                    r[9 + 2 * p] = v0[m].x * v0[j].y - v0[m].y * v0[j].x + v1[m].x * v1[j].y -
                                   v1[m].y * v1[j].x;
                }
        }
#pragma unroll
        for (int e = 0; e < 20; e++)
            r[e] = gsum(r[e], g);
        float2 h[4];

        {
            int p = 0;

#pragma unroll
            for (int m = 0; m < 4; m++) {
                float sx = r[2 * m], sy = r[2 * m + 1];

#pragma unroll
                for (int j = 0; j < m; j++, p++) {
                    const float gx = r[8 + 2 * p], gy = r[9 + 2 * p];

                    sx -= gx * h[j].x - gy * h[j].y;
                    sy -= gx * h[j].y + gy * h[j].x;
                }
                h[m] = make_float2(ta[m].x * sx - ta[m].y * sy, ta[m].x * sy + ta[m].y * sx);
            }
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            x0.x -= v0[m].x * h[m].x - v0[m].y * h[m].y;
            x0.y -= v0[m].x * h[m].y + v0[m].y * h[m].x;
            x1.x -= v1[m].x * h[m].x - v1[m].y * h[m].y;
            x1.y -= v1[m].x * h[m].y + v1[m].y * h[m].x;
        }
    }
}


__device__ __forceinline__ int sturm16(const float *d, const float *e2, int n, float x,
                                       float pivmin)
{
    float q = d[0] - x;
    int c = q < 0.f;

    for (int i = 1; i < n; i++) {
        if (fabsf(q) < pivmin)
            q = -pivmin;
        q = d[i] - x - __fdividef(e2[i - 1], q);
        c += q < 0.f;
    }
    return c;
}

/* Eigenvalue of rank `index` of the group's tridiagonal (w.d, w.e), by
   17-way multisection of its Gershgorin interval. */
__device__ float tri_eigenvalue(int n, int index, const HWs &w, const Grp &g, float &norm,
                                unsigned &status)
{
    const int i0 = g.gl, i1 = g.gl + 16;
    float lo = INFINITY, hi = -INFINITY;

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;

        if (r < n) {
            const float rad = (r > 0 ? fabsf(w.e[r - 1]) : 0.f) + (r < n - 1 ? fabsf(w.e[r]) : 0.f);

            lo = fminf(lo, w.d[r] - rad);
            hi = fmaxf(hi, w.d[r] + rad);
            if (r < n - 1)
                w.e2f[r] = w.e[r] * w.e[r];
        }
    }
    lo = gminf(lo, g);
    hi = gmaxf(hi, g);
    norm = fmaxf(fabsf(lo), fabsf(hi));
    lo -= 1.0e-6f * norm + 1.0e-30f;
    hi += 1.0e-6f * norm + 1.0e-30f;
    gsync(g);
    const float pivmin = 1.0e-30f + 1.0e-14f * norm;
    int round = 0;

    for (; round < 20; round++) {
        /* 1e-7 of the spectrum's scale is all that the inverse iteration
           and the solves off the eigenvector need (the eigenvector's
           accuracy comes from those); the smallest eigenvalues of EMI would
           otherwise take several more rounds down to their own ulp */
        if (hi - lo <= 1.0e-7f * norm)
            break;
        const float xq = lo + (hi - lo) * ((float)(g.gl + 1) * (1.0f / 17.0f));
        const int cnt = sturm16(w.d, w.e2f, n, xq, pivmin);
        const unsigned gt = (__ballot_sync(g.mask, cnt > index) >> g.base) & 0xFFFFu;
        float nlo, nhi;

        if (gt == 0u) {
            nlo = gbcast(xq, 15, g);
            nhi = hi;
        }
        else {
            const int f = __ffs(gt) - 1;

            nhi = gbcast(xq, f, g);
            nlo = gbcast(xq, f > 0 ? f - 1 : 0, g);
            if (f == 0)
                nlo = lo;
        }
        nlo = fmaxf(nlo, lo);
        nhi = fminf(nhi, hi);
        if (!(nlo > lo || nhi < hi))
            break;
        lo = nlo;
        hi = nhi;
    }
    if (round == 20)
        status |= TC_STATUS_ITER_CAP;
    return 0.5f * (lo + hi);
}

/* The LU's reciprocals (pivots of a shifted tridiagonal) need no correct
   rounding: the hardware approximation, within two ulps. */
__device__ __forceinline__ float rcpx(float x) { return __fdividef(1.0f, x); }

/* Partially pivoted LU of tri - lambda I, into w.lu (written by the first
   lane of the group); returns the pivot bits. Every lane computes it. */
template <typename R>
__device__ unsigned long long tri_lu(int n, R lambda, R tiny, const HWs &w, const Grp &g)
{
    R dd = (R)w.d[0] - lambda, s1 = n > 1 ? (R)w.e[0] : (R)0;
    unsigned long long piv = 0ull;

    for (int k = 0; k < n - 1; k++) {
        const R sub = w.e[k], nd = (R)w.d[k + 1] - lambda;
        const R ns = k + 1 < n - 1 ? (R)w.e[k + 1] : (R)0;
        float4 f;

        if (fabs(dd) >= fabs(sub)) {
            if (fabs(dd) < tiny)
                dd = dd < (R)0 ? -tiny : tiny;
            const R rd = rcpx(dd), l = sub * rd;

            f = make_float4((float)rd, (float)s1, 0.f, (float)l);
            dd = nd - l * s1;
            s1 = ns;
        }
        else {
            const R rs = rcpx(sub), l = dd * rs;

            piv |= 1ull << k;
            f = make_float4((float)rs, (float)nd, (float)ns, (float)l);
            dd = s1 - l * nd;
            s1 = -l * ns;
        }
        if (g.gl == 0)
            w.lu[k] = f;
    }
    if (fabs(dd) < tiny)
        dd = dd < (R)0 ? -tiny : tiny;
    if (g.gl == 0)
        w.lu[n - 1] = make_float4((float)rcpx(dd), 0.f, 0.f, 0.f);
    gsync(g);
    return piv;
}

/* Solve (tri - lambda) with the LU of tri_lu, in place on yr (every lane,
   same values). */
__device__ __forceinline__ void tri_solve(float (&yr)[32], int n, unsigned long long piv,
                                          const HWs &w)
{
#pragma unroll
    for (int k = 0; k < 31; k++) {
        if (k >= n - 1)
            break;
        if ((piv >> k) & 1ull) {
            const float t = yr[k];

            yr[k] = yr[k + 1];
            yr[k + 1] = t;
        }
        yr[k + 1] -= w.lu[k].w * yr[k];
    }
#pragma unroll
    for (int k = 31; k >= 0; k--) {
        if (k > n - 1)
            continue;
        const float4 u = w.lu[k];
        float v = yr[k];

        if (k + 1 < n)
            v -= u.y * yr[k + 1];
        if (k + 2 < n)
            v -= u.z * yr[k + 2];
        yr[k] = v * u.x;
    }
}

/* The eigenvector of rank `index` of the reduced matrix, back-transformed:
   returns the components of rows i0, i1 in z0, z1; y (tridiagonal vector)
   is left in yr. */
__device__ unsigned eigvec(int n, int index, const HWs &w, int ld, const Grp &g, float2 &z0,
                           float2 &z1, float (&yr)[32], float &lambda, float &norm,
                           unsigned long long &piv)
{
    unsigned status = 0;

    lambda = tri_eigenvalue(n, index, w, g, norm, status);
    const float tiny = 1.0e-6f * fmaxf(norm, 1.0e-30f);

    piv = tri_lu<float>(n, lambda, tiny, w, g);

#pragma unroll
    for (int k = 0; k < 32; k++)
        yr[k] = 1.f;
    for (int it = 0; it < 3; it++) {
        tri_solve(yr, n, piv, w);
        float nrm = 0.f;

#pragma unroll
        for (int k = 0; k < 32; k++)
            if (k < n)
                nrm = fmaxf(nrm, fabsf(yr[k]));
        const float inv = __frcp_rn(nrm);

#pragma unroll
        for (int k = 0; k < 32; k++)
            yr[k] *= inv;
    }
    const int i0 = g.gl, i1 = g.gl + 16;
    float y0 = 0.f, y1 = 0.f;

#pragma unroll
    for (int k = 0; k < 32; k++) {
        if (k == i0)
            y0 = yr[k];
        if (k == i1)
            y1 = yr[k];
    }
    z0 = make_float2(i0 < n ? y0 : 0.f, 0.f);
    z1 = make_float2(i1 < n ? y1 : 0.f, 0.f);
    /* z = H_0 .. H_{n-2} y */
    apply_q(n, ld, w, g, false, z0, z1);
    return status;
}

/* ------------------------------------------------------------------ */
/* EMI: |T|^-1 in double.                                              */
/* ------------------------------------------------------------------ */

/* 1 / d by two Newton-Raphson steps y <- y + y (1 - d y) from the hardware's
   approximate FP64 reciprocal (within an ulp of the quotient; |d| here is a
   pivot above the sweep's floor, never denormal or zero). */
__device__ __forceinline__ double rcp_newton(double d)
{
    double y;

    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);

    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

/* Symmetric sweep (Gauss-Jordan elimination without pivoting in the form
   that keeps the matrix symmetric; Goodnight, The American Statistician 33,
   1979) of the group's matrix: rows i0, i1 in g0, g1, columns >= n zero.
   Sweeping pivot k maps
       a_ij -> a_ij - a_ik a_kj / a_kk,  a_ik, a_kj -> a_ik / a_kk,
       a_kk -> -1 / a_kk,
   and sweeping every pivot leaves -A^-1. Because the matrix stays
   symmetric, pivot row k is assembled from every lane's own column-k
   entries. The register columns rotate by one per step so that the pivot
   column is always g[0] (the step loop stays a run-time loop): on return
   register column p holds true column (p + n) & 31. rs holds 2 x 32
   doubles (alternate steps use alternate halves). False when a pivot's
   magnitude is not above `floor`. */
__device__ bool sweep16(double (&g0)[32], double (&g1)[32], int n, double floor, double *rs,
                        const Grp &g)
{
    const int i0 = g.gl, i1 = g.gl + 16;

    for (int k = 0; k < n; k++) {
        double *r = rs + 32 * (k & 1);

        /* a_ik, in the order of the registers: rs[p] = a_k,(p + k) & 31 */
        r[(i0 - k) & 31] = g0[0];
        r[(i1 - k) & 31] = g1[0];
        gsync(g);
        const double d = r[0];

        if (!(fabs(d) > floor))
            return false;
        const double id = rcp_newton(d);
        const bool piv0 = i0 == k, piv1 = i1 == k;
        /* the pivot row scales by 1 / a_kk: a_kj - (1 - 1 / a_kk) a_kj, with
           a_kj from rs (equal to the row's own value up to rounding) */
        const double f0 = piv0 ? 1.0 - id : g0[0] * id, f1 = piv1 ? 1.0 - id : g1[0] * id;

#pragma unroll
        for (int q = 0; q < 32; q += 2) {
            const double2 a = *(const double2 *)&r[q];

            if (q > 0) {
                g0[q - 1] = fma(-f0, a.x, g0[q]);
                g1[q - 1] = fma(-f1, a.x, g1[q]);
            }
            g0[q] = fma(-f0, a.y, g0[q + 1]);
            g1[q] = fma(-f1, a.y, g1[q + 1]);
        }
        g0[31] = piv0 ? -id : f0;
        g1[31] = piv1 ? -id : f1;
    }
    return true;
}

/* Rows i0, i1 of a matrix whose register column p is true column
   (p + rot) & 31, scaled by s, into dst (n x ld). */
__device__ __forceinline__ void store_rows(double *dst, int ld, int n, int rot, double s,
                                           const double (&g0)[32], const double (&g1)[32],
                                           const Grp &g)
{
    const int i0 = g.gl, i1 = g.gl + 16;

#pragma unroll
    for (int p = 0; p < 32; p++) {
        const int j = (p + rot) & 31;

        if (j < n) {
            if (i0 < n)
                dst[i0 * ld + j] = s * g0[p];
            if (i1 < n)
                dst[i1 * ld + j] = s * g1[p];
        }
    }
}

/* (o0, o1) = rows i0, i1 of A times B; A and B n x ld (memory). */
__device__ void rows_times(const double *A, const double *B, int ld, int n, int i0, int i1,
                           double (&o0)[32], double (&o1)[32])
{
#pragma unroll
    for (int j = 0; j < 32; j++) {
        o0[j] = 0.0;
        o1[j] = 0.0;
    }
    for (int k = 0; k < n; k++) {
        const double *row = B + k * ld;
        const double x0 = i0 < n ? A[i0 * ld + k] : 0.0, x1 = i1 < n ? A[i1 * ld + k] : 0.0;

#pragma unroll
        for (int j = 0; j < 32; j++)
            if (j < n) {
                const double b = row[j];

                o0[j] = fma(x0, b, o0[j]);
                o1[j] = fma(x1, b, o1[j]);
            }
    }
}

/* Jacobi pseudo-inverse of G (n x ld double, shared) in place, V (n x ld)
   workspace; eigenvalues |l| < 1e-9 dropped (tests/reference.py:151-156). */
__device__ unsigned jacobi_pinv16(int n, int ld, double *G, double *V, double *lam,
                                  const Grp &g)
{
    unsigned status = TC_STATUS_ITER_CAP;

    for (int r = g.gl; r < n; r += 16)
        for (int j = 0; j < n; j++)
            V[r * ld + j] = r == j ? 1.0 : 0.0;
    gsync(g);
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0, dg = 0.0;

        for (int r = g.gl; r < n; r += 16)
            for (int j = 0; j < n; j++) {
                const double x = G[r * ld + j];

                if (j == r)
                    dg += x * x;
                else
                    off += x * x;
            }
        off = gsum(off, g);
        dg = gsum(dg, g);
        if (off <= 1.0e-30 * dg) {
            status = 0;
            break;
        }
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = G[p * ld + q];

                if (apq == 0.0)
                    continue;
                const double app = G[p * ld + p], aqq = G[q * ld + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                                 (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;

                gsync(g);
                for (int r = g.gl; r < n; r += 16) {
                    if (r != p && r != q) {
                        const double akp = G[r * ld + p], akq = G[r * ld + q];

                        G[r * ld + p] = c * akp - s * akq;
                        G[r * ld + q] = s * akp + c * akq;
                    }
                    const double vkp = V[r * ld + p], vkq = V[r * ld + q];

                    V[r * ld + p] = c * vkp - s * vkq;
                    V[r * ld + q] = s * vkp + c * vkq;
                }
                gsync(g);
                for (int r = g.gl; r < n; r += 16)
                    if (r != p && r != q) {
                        G[p * ld + r] = G[r * ld + p];
                        G[q * ld + r] = G[r * ld + q];
                    }
                if (g.gl == 0) {
                    G[p * ld + p] = app - t * apq;
                    G[q * ld + q] = aqq + t * apq;
                    G[p * ld + q] = 0.0;
                    G[q * ld + p] = 0.0;
                }
                gsync(g);
            }
    }
    for (int r = g.gl; r < n; r += 16)
        lam[r] = G[r * ld + r];
    gsync(g);
    for (int i = g.gl; i < n; i += 16)
        for (int j = 0; j < n; j++) {
            double s = 0.0;

            for (int k = 0; k < n; k++) {
                const double l = lam[k];

                if (fabs(l) >= 1.0e-9)
                    s += V[i * ld + k] * V[j * ld + k] / l;
            }
            G[i * ld + j] = s;
        }
    gsync(g);
    return status;
}

/* Packed entry (i, j) of a symmetric matrix, either triangle. */
__device__ __forceinline__ int sym_idx(int n, int i, int j)
{
    return i <= j ? tc_pidx(n, i, j) : tc_pidx(n, j, i);
}

/* |T| in double into w.G (packed upper triangle), from T (n <= 32); lane l
   takes rows l and n - 1 - l, so that every lane has n + 1 entries. */
__device__ void packed_abs_t(int n, int ld, const HWs &w, const Grp &g)
{
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? n - 1 - g.gl : g.gl;

        if (r < n && (t == 0 ? r <= n - 1 - g.gl : r > g.gl))
            for (int j = r; j < n; j++) {
                const float2 v = w.T[r * ld + j];

                w.G[tc_pidx(n, r, j)] = hypot((double)v.x, (double)v.y);
            }
    }
    gsync(g);
}

/* |T| in full into A (n x ld, global scratch), from its packed copy. */
__device__ void full_abs_t(double *A, int n, int ld, const double *Gp, const Grp &g)
{
    for (int r = g.gl; r < n; r += 16)
        for (int j = 0; j < n; j++)
            A[r * ld + j] = Gp[sym_idx(n, r, j)];
    gsync(g);
}

/* |T|^-1 into w.G (packed upper triangle, double), from T. The rare
   fallback tiers work on full matrices A, V (n x ld each) and lam (n) in
   the group's global scratch. Returns status bits. */
/* |T|^-1 into w.G; inv_max receives n max|inv_ij| (infinite when a
   fallback tier ran). */
__device__ unsigned emi_inverse(int n, int ld, const HWs &w, double *A, double *V, double *lam,
                                const Grp &g, double &inv_max)
{
    const int i0 = g.gl, i1 = g.gl + 16;
    double g0[32], g1[32];
    unsigned st = 0;
    int rot = n;
    bool full = false;

    packed_abs_t(n, ld, w, g);
#pragma unroll
    for (int j = 0; j < 32; j++) {
        g0[j] = (i0 < n && j < n) ? w.G[sym_idx(n, i0, j)] : 0.0;
        g1[j] = (i1 < n && j < n) ? w.G[sym_idx(n, i1, j)] : 0.0;
    }
    bool ok = sweep16(g0, g1, n, 1.0e-5, w.rs, g);

    if (!ok) {
        /* a pivot of |T| is close to zero: (|T|^2)^-1 |T|, with the
           intermediate inverse in V */
        st |= TC_STATUS_EMI_PINV;
        gsync(g);
        full_abs_t(A, n, ld, w.G, g);
        full = true;
        rows_times(A, A, ld, n, i0, i1, g0, g1);
        ok = sweep16(g0, g1, n, 1.0e-300, w.rs, g);
        if (ok) {
            store_rows(V, ld, n, n, -1.0, g0, g1, g);
            gsync(g);
            rows_times(V, A, ld, n, i0, i1, g0, g1);
            rot = 0;
        }
    }
    if (ok) {
        /* every |eigenvalue| of |T| above 1e-9, where the pseudo-inverse of
           reference.py is the inverse: n max|inv_ij| < 1e8 ensures it. */
        double mx = 0.0;

#pragma unroll
        for (int j = 0; j < 32; j++)
            mx = fmax(mx, fmax(fabs(g0[j]), fabs(g1[j])));
        mx = gmaxd(mx, g);
        ok = mx == mx && n * mx < 1.0e8;
        inv_max = ok && !full ? n * mx : INFINITY;
    }
    else
        inv_max = INFINITY;
    gsync(g);
    if (ok) {
        const double sc = rot ? -1.0 : 1.0;

#pragma unroll
        for (int p = 0; p < 32; p++) {
            const int j = (p + rot) & 31;

            if (j < n) {
                if (i0 <= j)
                    w.G[tc_pidx(n, i0, j)] = sc * g0[p];
                if (i1 <= j)
                    w.G[tc_pidx(n, i1, j)] = sc * g1[p];
            }
        }
    }
    else {
        if (!full)
            full_abs_t(A, n, ld, w.G, g);
        st |= TC_STATUS_EMI_PINV | jacobi_pinv16(n, ld, A, V, lam, g);
        for (int r = g.gl; r < n; r += 16)
            for (int j = r; j < n; j++)
                w.G[tc_pidx(n, r, j)] = A[r * ld + j];
    }
    gsync(g);
    return st;
}

/* M_ij = inv_ij T_ij (double) */
__device__ __forceinline__ double2 mval(const HWs &w, int ld, int i, int j)
{
    const double gg = w.G[sym_idx(w.n, i, j)];
    const float2 t = w.T[i < j ? i * ld + j : j * ld + i];

    return make_double2(gg * (double)t.x, i < j ? gg * (double)t.y : -gg * (double)t.y);
}

/* t = Q (tri - lambda)^+ Q^H b off the eigen-direction, rows (i0, i1):
   Q and tri are the float reduction of the group's matrix (Householder
   vectors in T's lower triangle, tau), lambda the eigenvalue of the
   tridiagonal eigenvector y, piv / w.lu the LU of (tri - lambda). b is
   mapped by Q^H, its component along y removed, the real and imaginary
   parts solved with the LU, the y component removed again, and the result
   mapped back by Q. Scratch: the first 32 float2 of w.x. */
__device__ void solve_off(int n, int ld, const HWs &w, const Grp &g, const float (&yr)[32],
                          unsigned long long piv, float2 b0, float2 b1, float2 &t0, float2 &t1)
{
    const int i0 = g.gl, i1 = g.gl + 16;

    /* b = Q^H b = H_{n-2} .. H_0 b */
    apply_q(n, ld, w, g, true, b0, b1);
    /* b is in the real-tridiagonal basis but complex-valued: solve the real
       and imaginary parts with the float LU of (tri - lambda), off y. */
    float2 *bs = (float2 *)w.x;

    bs[i0] = b0;
    bs[i1] = b1;
    gsync(g);
    float tr_[32], ti_[32];
    float ynrm = 0.f, cr = 0.f, ci = 0.f;

#pragma unroll
    for (int k = 0; k < 32; k++) {
        const float2 bk = k < n ? bs[k] : make_float2(0.f, 0.f);

        ynrm = fmaf(yr[k], yr[k], ynrm);
        cr = fmaf(yr[k], bk.x, cr);
        ci = fmaf(yr[k], bk.y, ci);
        tr_[k] = bk.x;
        ti_[k] = bk.y;
    }
    gsync(g);
    cr /= ynrm;
    ci /= ynrm;
#pragma unroll
    for (int k = 0; k < 32; k++) {
        tr_[k] = fmaf(-cr, yr[k], tr_[k]);
        ti_[k] = fmaf(-ci, yr[k], ti_[k]);
    }
    /* one solve per lane: the real parts in lanes 0-7, the imaginary parts
       in lanes 8-15, exchanged afterwards */
    {
        float v[32];

#pragma unroll
        for (int k = 0; k < 32; k++)
            v[k] = g.gl >= 8 ? ti_[k] : tr_[k];
        tri_solve(v, n, piv, w);
#pragma unroll
        for (int k = 0; k < 32; k++) {
            tr_[k] = __shfl_sync(g.mask, v[k], g.base);
            ti_[k] = __shfl_sync(g.mask, v[k], g.base | 8);
        }
    }
    float dr = 0.f, di = 0.f;

#pragma unroll
    for (int k = 0; k < 32; k++)
        if (k < n) {
            dr = fmaf(yr[k], tr_[k], dr);
            di = fmaf(yr[k], ti_[k], di);
        }
    dr /= ynrm;
    di /= ynrm;
    t0 = make_float2(0.f, 0.f);
    t1 = t0;
#pragma unroll
    for (int k = 0; k < 32; k++) {
        if (k == i0 && k < n)
            t0 = make_float2(fmaf(-dr, yr[k], tr_[k]), fmaf(-di, yr[k], ti_[k]));
        if (k == i1 && k < n)
            t1 = make_float2(fmaf(-dr, yr[k], tr_[k]), fmaf(-di, yr[k], ti_[k]));
    }
    /* t = Q t = H_0 .. H_{n-2} t */
    apply_q(n, ld, w, g, false, t0, t1);
}

/* One refinement step of the eigenpair of M for the eigenvector (z0, z1)
   of rows (i0, i1): see the file comment. tri and Q are the float
   reduction of M; y is the tridiagonal eigenvector. The residual is formed
   in double; the correction, a small vector that needs only float relative
   accuracy, is mapped through Q in float after scaling the residual to a
   unit maximum. */
__device__ void refine(int n, int ld, const HWs &w, const Grp &g, double2 &x0, double2 &x1,
                       const float (&yr)[32], unsigned long long piv)
{
    const int i0 = g.gl, i1 = g.gl + 16;

    /* normalize, publish x */
    double nn = x0.x * x0.x + x0.y * x0.y + x1.x * x1.x + x1.y * x1.y;

    nn = gsum(nn, g);
    const double inrm = 1.0 / sqrt(nn);

    x0.x *= inrm;
    x0.y *= inrm;
    x1.x *= inrm;
    x1.y *= inrm;
    w.x[i0] = x0;
    w.x[i1] = x1;
    gsync(g);
    /* u = M x (rows i0, i1), mu = x^H u */
    double2 u0 = make_double2(0.0, 0.0), u1 = u0;

    for (int j = 0; j < n; j++) {
        const double2 xj = w.x[j];

        if (i0 < n) {
            const double2 m = mval(w, ld, i0, j);

            u0.x += m.x * xj.x - m.y * xj.y;
            u0.y += m.x * xj.y + m.y * xj.x;
        }
        if (i1 < n) {
            const double2 m = mval(w, ld, i1, j);

            u1.x += m.x * xj.x - m.y * xj.y;
            u1.y += m.x * xj.y + m.y * xj.x;
        }
    }
    double mu = x0.x * u0.x + x0.y * u0.y + x1.x * u1.x + x1.y * u1.y;

    mu = gsum(mu, g);
    /* r = u - mu x, scaled to a unit maximum */
    double2 r0 = make_double2(u0.x - mu * x0.x, u0.y - mu * x0.y);
    double2 r1 = make_double2(u1.x - mu * x1.x, u1.y - mu * x1.y);

    if (i0 >= n)
        r0 = make_double2(0.0, 0.0);
    if (i1 >= n)
        r1 = make_double2(0.0, 0.0);
    const double rmax = gmaxd(fmax(fmax(fabs(r0.x), fabs(r0.y)), fmax(fabs(r1.x), fabs(r1.y))), g);

    gsync(g);
    if (!(rmax > 0.0))
        return;
    const double sc = 1.0 / rmax;
    float2 t0, t1;

    solve_off(n, ld, w, g, yr, piv, make_float2((float)(r0.x * sc), (float)(r0.y * sc)),
              make_float2((float)(r1.x * sc), (float)(r1.y * sc)), t0, t1);
    /* x -= Q (tri - mu)^+ Q^H r */
    x0.x -= rmax * t0.x;
    x0.y -= rmax * t0.y;
    x1.x -= rmax * t1.x;
    x1.y -= rmax * t1.y;
    gsync(g);
}

/* ------------------------------------------------------------------ */
/* Common stages.                                                      */
/* ------------------------------------------------------------------ */

/* One batch of the packed entries q = gl + 16 t (t = t0 .. t0 + B - 1):
   T_ij = C_ij / (nrm_i nrm_j), bias-corrected, both triangles. */
template <int B>
__device__ __forceinline__ void load_T_batch(const float2 (&gv)[B], int t0, int n, int npu, bool active,
                                             int looks, const TcLinkConst &k,
                                             const unsigned short *upper_tab, const HWs &w,
                                             int ld, const Grp &g, bool &boundary)
{
    const float fl = (float)looks;
    const bool debias = k.bias && looks > 1;
    const float ilm1 = debias ? __frcp_rn(fl - 1.0f) : 0.f;

#pragma unroll
    for (int t = 0; t < B; t++) {
        const int q = g.gl + 16 * (t0 + t);

        if (q >= npu)
            continue;
        const int i = upper_tab[q] >> 8, j = upper_tab[q] & 255;

        if (i == j) {
            w.T[i * ld + i] = make_float2(1.f, 0.f);
            continue;
        }
        float re = 0.f, im = 0.f;

        if (active) {
            /* w.nrm holds 1 / sqrt(C_ii) (0 for an empty date) */
            const float2 gq = gv[t];
            const float rd = w.nrm[i] * w.nrm[j];

            if (rd > 0.f) {
                re = gq.x * rd;
                im = gq.y * rd;
                if (debias) {
                    /* f^2 = m2c / m2, m2c = (L m2 - 1) / (L - 1) */
                    const float m2 = re * re + im * im;
                    const float lm1 = fmaf(fl, m2, -1.0f);
                    const float m2c = lm1 * ilm1;

                    boundary |= fabsf(lm1) < TC_BIAS_BAND * fl * m2;
                    const float f2 = m2 > 0.f && m2c > 0.f ? m2c * __fdividef(1.0f, m2) : 0.f;
                    const float f = f2 > 0.f ? f2 * rsqrtf(f2) : 0.f;

                    re *= f;
                    im *= f;
                }
            }
        }
        w.T[i * ld + j] = make_float2(re, im);
        w.T[j * ld + i] = make_float2(re, -im);
    }
}

/* The first batch of a pixel's packed Gram sums (entries gl + 16 t, t < 17)
   and its two diagonal sums, loaded for load_T (zero where out of range).
   The link kernel issues these loads for the next pixel pair during the
   last stage of the current one, so that they arrive while gamma runs. */
struct TFirst {
    float2 ga[17];
    float d0, d1;
};

__device__ __forceinline__ void t_first(TFirst &f, int n, int p, bool inrange,
                                        const float2 *__restrict__ gram, const Grp &g)
{
    const int npu = tc_npu(n), i0 = g.gl, i1 = g.gl + 16;

    f.d0 = (inrange && i0 < n) ? gram[tc_gram_at(npu, p, tc_pidx(n, i0, i0))].x : 1.f;
    f.d1 = (inrange && i1 < n) ? gram[tc_gram_at(npu, p, tc_pidx(n, i1, i1))].x : 1.f;
#pragma unroll
    for (int t = 0; t < 17; t++) {
        const int q = g.gl + 16 * t;

        f.ga[t] = (inrange && q < npu) ? gram[tc_gram_at(npu, p, q)] : make_float2(0.f, 0.f);
    }
}

/* T of the group's pixel from its packed Gram sums (tcoh.cl:611-636);
   identity for an inactive group. The entries come in two batches of 17
   (f, loaded ahead) and 16 per lane, each batch's loads issued before any
   use (one batch of 33 held 66 registers through the processing and
   spilled); upper_tab is the CTA's shared-memory copy of the packed-entry
   table. */
__device__ void load_T(const TcStrip &s, const TcChunk &c, const TcLinkConst &k, int p, bool active,
                       int looks, const float2 *__restrict__ gram, const TFirst &f,
                       const unsigned short *upper_tab, const HWs &w, int ld, const Grp &g,
                       bool &boundary)
{
    const int n = s.n, npu = tc_npu(n);
    const int i0 = g.gl, i1 = g.gl + 16;
    float2 gb[16];
    const float d0 = active ? f.d0 : 1.f, d1 = active ? f.d1 : 1.f;

    if (i0 < n)
        w.nrm[i0] = d0 > 0.f ? __frcp_rn(__fsqrt_rn(d0)) : 0.f;
    if (i1 < n)
        w.nrm[i1] = d1 > 0.f ? __frcp_rn(__fsqrt_rn(d1)) : 0.f;
    gsync(g);
    load_T_batch<17>(f.ga, 0, n, npu, active, looks, k, upper_tab, w, ld, g, boundary);
#pragma unroll
    for (int t = 0; t < 16; t++) {
        const int q = g.gl + 16 * (17 + t);

        gb[t] = (active && q < npu) ? gram[tc_gram_at(npu, p, q)] : make_float2(0.f, 0.f);
    }
    load_T_batch<16>(gb, 17, n, npu, active, looks, k, upper_tab, w, ld, g, boundary);
    gsync(g);
    boundary = __any_sync(g.mask, boundary);
}

/* Whether the non-zero coherences link all dates (n <= 32). */
__device__ bool linked16(int n, int ld, const float2 *T, const Grp &g)
{
    unsigned adj[2] = {0u, 0u};

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = g.gl + 16 * t;

        if (r < n)
            for (int j = 0; j < n; j++) {
                const float2 v = T[r * ld + j];

                if (j != r && (v.x != 0.f || v.y != 0.f))
                    adj[t] |= 1u << j;
            }
    }
    const unsigned all = n == 32 ? ~0u : (1u << n) - 1u;
    unsigned reached = 1u, frontier = 1u;

    for (int it = 0; it < n; it++) {
        unsigned mine = 0u;

        if ((frontier >> g.gl) & 1u)
            mine |= adj[0];
        if (g.gl + 16 < n && ((frontier >> (g.gl + 16)) & 1u))
            mine |= adj[1];
#pragma unroll
        for (int o = 8; o; o >>= 1)
            mine |= __shfl_xor_sync(g.mask, mine, o);
        const unsigned nw = mine & ~reached;

        if (!nw)
            break;
        reached |= nw;
        frontier = nw;
    }
    return reached == all;
}

/* Unit phasors relative to the median date (tcoh.cl:700-724) into w.zs,
   then the goodness of fit (tcoh.cl:728-744), pairs spread evenly over the
   lanes. */
__device__ float gamma16(int n, int ld, const HWs &w, const Grp &g, double2 z0d, double2 z1d,
                         const unsigned short *__restrict__ upper_tab, float2 *sum = nullptr)
{
    /* the phasors in float, as the reference kernel forms them: the
       eigenvector's components carry float accuracy at best */
    const float2 z0 = make_float2((float)z0d.x, (float)z0d.y);
    const float2 z1 = make_float2((float)z1d.x, (float)z1d.y);
    const int i0 = g.gl, i1 = g.gl + 16;
    const float m0 = i0 < n ? hypotf(z0.x, z0.y) : 0.f, m1 = i1 < n ? hypotf(z1.x, z1.y) : 0.f;
    const float mx = gmaxf(fmaxf(m0, m1), g);
    int ref = n / 2;
    const float mref = gbcast(ref < 16 ? m0 : m1, ref, g);

    if (mref <= 1.0e-3f * mx) {
        int last = -1;

        if (i0 < n && m0 == mx)
            last = i0;
        if (i1 < n && m1 == mx)
            last = i1;
#pragma unroll
        for (int o = 8; o; o >>= 1)
            last = max(last, __shfl_xor_sync(g.mask, last, o));
        ref = last;
    }
    const float zrx = gbcast(ref < 16 ? z0.x : z1.x, ref, g);
    const float zry = gbcast(ref < 16 ? z0.y : z1.y, ref, g);
    const float refm = hypotf(zrx, zry);
    const float refr = zrx / refm, refi = -zry / refm;
    const float floor_ = mx * 1.0e-3f;

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;
        const float2 z = t ? z1 : z0;

        if (r < n) {
            const float re = z.x * refr - z.y * refi, im = z.x * refi + z.y * refr;
            const float mm = hypotf(re, im);

            w.zs[r] = mm > floor_ ? make_float2(re / mm, im / mm) : make_float2(1.f, 0.f);
        }
    }
    gsync(g);
    float sr = 0.f, si = 0.f;
    const int npu = tc_npu(n);

    for (int q = g.gl; q < npu; q += 16) {
        const int i = upper_tab[q] >> 8, j = upper_tab[q] & 255;

        if (i == j)
            continue;
        const float2 tv = w.T[i * ld + j];
        const float m2 = tv.x * tv.x + tv.y * tv.y;
        float ur = 1.f, ui = 0.f;

        if (m2 > 0.f) {
            const float r = rsqrtf(m2);

            ur = tv.x * r;
            ui = tv.y * r;
        }
        const float2 zi = w.zs[i], zj = w.zs[j];
        const float wr = zi.x * zj.x + zi.y * zj.y;
        const float wi = zi.x * zj.y - zi.y * zj.x;

        sr += ur * wr - ui * wi;
        si += ur * wi + ui * wr;
    }
    sr = gsum(sr, g);
    si = gsum(si, g);
    if (sum)
        *sum = make_float2(sr, si);
    return hypotf(sr, si) / (0.5f * n * (n - 1));
}

/* ------------------------------------------------------------------ */
/* Adjoint.                                                            */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmulc(float2 a, float2 b) /* a conj(b) */
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

/* T_ij of either triangle from the upper one (the lower holds the
   Householder vectors). */
__device__ __forceinline__ float2 t_full(const HWs &w, int ld, int i, int j)
{
    if (i == j)
        return make_float2(1.f, 0.f);
    const float2 t = w.T[(i < j ? i : j) * ld + (i < j ? j : i)];

    return i < j ? t : make_float2(t.x, -t.y);
}

/* Gradient of gamma with respect to the pixel's coherence sums, written as
   the Hermitian matrix G (upper triangle, gbar[pidx][p]) such that
   d gamma = Re sum_ij conj(G_ij) dC_ij. The chain, in reverse:
   gamma = |S| / npairs, S = sum_{i<j} unit(T_ij) conj(e_i) e_j; phasors
   e_k = unit(z_k conj(z_ref)) (1 below the 1e-3 floor); the eigenvector z
   of X (X = T for EVD, M = |T|^-1 o T for EMI) through
   dz = (lambda - X)^+ dX z, applied with the float reduction of X
   (solve_off); for EMI, M-bar = y z^H gives T-bar += |T|^-1 o M-bar and
   |T|-bar = -|T|^-1 Re(conj(M-bar) o T) |T|^-1 (double); the bias correction
   |T| = sqrt((L |t|^2 - 1) / (L - 1)); the normalization
   t_ij = C_ij / sqrt(C_ii C_jj) (C_ii does not depend on the phases).
   z0, z1: the final eigenvector rows; S: the sum of gamma16. The rows
   (i0, i1) of T-bar stay in registers (those of the reduction are free by
   now); once solve_off, the last reader of the Householder vectors, is
   done, their strictly lower parts go to T's lower triangle so that the
   owner of row i forms G_ij = (T-bar_ij + conj(T-bar_ji)) / 2 for j > i.
   Db: n x ld double scratch (EMI). An inactive pixel gets G = 0. */
template <bool EMI>
__device__ void backward16(int n, int ld, const HWs &w, const Grp &g, double2 z0d, double2 z1d,
                           float2 S, const float (&yr)[32], unsigned long long piv, int looks,
                           bool bias, bool active, double *Db, float2 *gbar, long long npix,
                           long long p)
{
    const int i0 = g.gl, i1 = g.gl + 16;

    /* unit-norm z in float; the phasor decisions (reference date, floor)
       are those of gamma16, made on the rows rounded to float */
    const float mf0 = i0 < n ? hypotf((float)z0d.x, (float)z0d.y) : 0.f;
    const float mf1 = i1 < n ? hypotf((float)z1d.x, (float)z1d.y) : 0.f;
    const float mxf = gmaxf(fmaxf(mf0, mf1), g);
    const double m0 = i0 < n ? hypot(z0d.x, z0d.y) : 0.0, m1 = i1 < n ? hypot(z1d.x, z1d.y) : 0.0;
    int ref = n / 2;
    const float mref = gbcast(ref < 16 ? mf0 : mf1, ref, g);

    if (mref <= 1.0e-3f * mxf) {
        int last = -1;

        if (i0 < n && mf0 == mxf)
            last = i0;
        if (i1 < n && mf1 == mxf)
            last = i1;
#pragma unroll
        for (int o = 8; o; o >>= 1)
            last = max(last, __shfl_xor_sync(g.mask, last, o));
        ref = last;
    }
    const bool big0 = i0 < n && mf0 > mxf * 1.0e-3f, big1 = i1 < n && mf1 > mxf * 1.0e-3f;
    const double nn = gsum(m0 * m0 + m1 * m1, g);
    const double inv = nn > 0.0 ? 1.0 / sqrt(nn) : 0.0;
    const float2 z0 = make_float2((float)(z0d.x * inv), (float)(z0d.y * inv));
    const float2 z1 = make_float2((float)(z1d.x * inv), (float)(z1d.y * inv));
    float2 *zb = (float2 *)w.x + 32;

    zb[i0] = i0 < n ? z0 : make_float2(0.f, 0.f);
    zb[i1] = i1 < n ? z1 : make_float2(0.f, 0.f);
    gsync(g);
    const float2 zr = zb[ref];
    /* S-bar */
    const float P = 0.5f * n * (n - 1), sm = hypotf(S.x, S.y);
    const float2 Sb = sm > 0.f ? make_float2(S.x / (sm * P), S.y / (sm * P)) : make_float2(0.f, 0.f);
    const float2 Sc = make_float2(Sb.x, -Sb.y);
    float2 tb0[32], tb1[32]; /* T-bar rows i0, i1 */
    float2 vb[2];

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;
        float2 eb = make_float2(0.f, 0.f);
        const float2 er = r < n ? w.zs[r] : make_float2(1.f, 0.f);

#pragma unroll
        for (int j = 0; j < 32; j++) {
            float2 tb = make_float2(0.f, 0.f);

            if (r < n && j < n && j != r) {
                const float2 tv = t_full(w, ld, r, j);
                const float m2 = tv.x * tv.x + tv.y * tv.y;
                const float im = m2 > 0.f ? rsqrtf(m2) : 0.f;
                const float2 wv = m2 > 0.f ? make_float2(tv.x * im, tv.y * im)
                                           : make_float2(1.f, 0.f);
                const float2 ej = w.zs[j];
                /* j > r: e-bar_r += conj(S-bar) w_rj e_j; j < r: e-bar_r +=
                   S-bar conj(w_jr) e_j = S-bar w_rj e_j */
                const float2 c = cmul(cmul(j > r ? Sc : Sb, wv), ej);

                eb = make_float2(eb.x + c.x, eb.y + c.y);
                if (j > r && m2 > 0.f) {
                    /* w-bar_rj = S-bar e_r conj(e_j), through w = T / |T| */
                    const float2 wb = cmul(Sb, cmulc(er, ej));
                    const float rr = wv.x * wb.x + wv.y * wb.y;

                    tb = make_float2((wb.x - wv.x * rr) * im, (wb.y - wv.y * rr) * im);
                }
            }
            if (t)
                tb1[j] = tb;
            else
                tb0[j] = tb;
        }
        /* v-bar_r = (e-bar - e Re(conj(e) e-bar)) / |v_r| */
        vb[t] = make_float2(0.f, 0.f);
        if (t ? big1 : big0) {
            const float2 zv = t ? z1 : z0;
            const float vm = hypotf(zv.x, zv.y) * hypotf(zr.x, zr.y);
            const float rr = er.x * eb.x + er.y * eb.y;

            vb[t] = make_float2((eb.x - er.x * rr) / vm, (eb.y - er.y * rr) / vm);
        }
    }
    /* v_k = z_k conj(z_ref): z-bar_k = v-bar_k z_ref, z-bar_ref += sum_k conj(v-bar_k) z_k */
    float2 zbar[2] = {cmul(vb[0], zr), cmul(vb[1], zr)};
    {
        const float2 c0 = cmul(make_float2(vb[0].x, -vb[0].y), z0);
        const float2 c1 = cmul(make_float2(vb[1].x, -vb[1].y), z1);
        const float cx = gsum(c0.x + c1.x, g), cy = gsum(c0.y + c1.y, g);

        if (i0 == ref) {
            zbar[0].x += cx;
            zbar[0].y += cy;
        }
        if (i1 == ref) {
            zbar[1].x += cx;
            zbar[1].y += cy;
        }
    }
    /* r = (I - z z^H) z-bar */
    float2 al = make_float2(z0.x * zbar[0].x + z0.y * zbar[0].y + z1.x * zbar[1].x + z1.y * zbar[1].y,
                            z0.x * zbar[0].y - z0.y * zbar[0].x + z1.x * zbar[1].y - z1.y * zbar[1].x);

    al.x = gsum(al.x, g);
    al.y = gsum(al.y, g);
    float2 b0 = make_float2(zbar[0].x - cmul(z0, al).x, zbar[0].y - cmul(z0, al).y);
    float2 b1 = make_float2(zbar[1].x - cmul(z1, al).x, zbar[1].y - cmul(z1, al).y);

    if (i0 >= n)
        b0 = make_float2(0.f, 0.f);
    if (i1 >= n)
        b1 = make_float2(0.f, 0.f);
    /* y = (lambda - X)^+ r = -(X - lambda)^+ r; X-bar = y z^H */
    float2 y0, y1;

    solve_off(n, ld, w, g, yr, piv, b0, b1, y0, y1);
    y0 = make_float2(-y0.x, -y0.y);
    y1 = make_float2(-y1.x, -y1.y);
    gsync(g);
    if (!EMI) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const float2 zj = j < n ? zb[j] : make_float2(0.f, 0.f);
            const float2 x0 = cmulc(y0, zj), x1 = cmulc(y1, zj);

            tb0[j].x += x0.x;
            tb0[j].y += x0.y;
            tb1[j].x += x1.x;
            tb1[j].y += x1.y;
        }
    }
    else {
        /* M = A o T with A = |T|^-1 (packed, double): T-bar += A o M-bar,
           A-bar = Re(conj(M-bar) o T) (rows to Db) */
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = t ? i1 : i0;
            const float2 yv = t ? y1 : y0;

#pragma unroll
            for (int j = 0; j < 32; j++)
                if (r < n && j < n) {
                    const float2 mb = cmulc(yv, zb[j]);
                    const double a = w.G[sym_idx(n, r, j)];
                    const float2 tv = t_full(w, ld, r, j);

                    if (t) {
                        tb1[j].x += (float)a * mb.x;
                        tb1[j].y += (float)a * mb.y;
                    } else {
                        tb0[j].x += (float)a * mb.x;
                        tb0[j].y += (float)a * mb.y;
                    }
                    Db[r * ld + j] = (double)mb.x * tv.x + (double)mb.y * tv.y;
                }
        }
        /* |T|-bar = -A (A-bar A): first Q = A-bar A, each lane's rows in
           place (it reads only its own rows of A-bar) */
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = t ? i1 : i0;

            if (r < n) {
                double q[32];

#pragma unroll
                for (int j = 0; j < 32; j++)
                    q[j] = 0.0;
                for (int l = 0; l < n; l++) {
                    const double ab = Db[r * ld + l];

#pragma unroll
                    for (int j = 0; j < 32; j++)
                        if (j < n)
                            q[j] = fma(ab, w.G[sym_idx(n, l, j)], q[j]);
                }
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < n)
                        Db[r * ld + j] = q[j];
            }
        }
        gsync(g);
        /* then |T|-bar_rj = -(A Q)_rj, into T-bar through |T| */
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = t ? i1 : i0;

#pragma unroll
            for (int j = 0; j < 32; j++)
                if (r < n && j < n && j != r) {
                    double bb = 0.0;

                    for (int k = 0; k < n; k++)
                        bb = fma(w.G[sym_idx(n, r, k)], Db[k * ld + j], bb);
                    const float2 tv = t_full(w, ld, r, j);
                    const float m = hypotf(tv.x, tv.y);

                    if (m > 0.f) {
                        const float b = (float)-bb;

                        if (t) {
                            tb1[j].x += b * tv.x / m;
                            tb1[j].y += b * tv.y / m;
                        } else {
                            tb0[j].x += b * tv.x / m;
                            tb0[j].y += b * tv.y / m;
                        }
                    }
                }
        }
    }
    /* bias correction and normalization: C-bar_rj = t-bar_rj / (nrm_r nrm_j) */
    const float L = (float)looks;

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;

#pragma unroll
        for (int j = 0; j < 32; j++) {
            float2 tb = t ? tb1[j] : tb0[j];

            if (r >= n || j >= n || j == r)
                tb = make_float2(0.f, 0.f);
            else if (bias && looks > 1) {
                const float2 tv = t_full(w, ld, r, j);
                const float mT = hypotf(tv.x, tv.y);

                if (mT > 0.f) {
                    /* t = unit(T) |t|, |t|^2 = ((L - 1) |T|^2 + 1) / L */
                    const float m2 = ((L - 1.f) * mT * mT + 1.f) / L;
                    const float mt = sqrtf(m2), c = mT / mt;
                    const float2 tt = make_float2(tv.x / c, tv.y / c);
                    const float kap = (tb.x * tt.x + tb.y * tt.y) / (c * (L - 1.f) * m2 * m2);

                    tb = make_float2(c * tb.x + kap * tt.x, c * tb.y + kap * tt.y);
                }
                else
                    tb = make_float2(0.f, 0.f);
            }
            if (r < n && j < n) {
                const float sc = w.nrm[r] * w.nrm[j];

                tb = make_float2(tb.x * sc, tb.y * sc);
            }
            if (t)
                tb1[j] = tb;
            else
                tb0[j] = tb;
        }
    }
    /* the strictly lower parts of the rows to T's lower triangle (the
       Householder vectors were last read by solve_off) */
    gsync(g);
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;

#pragma unroll
        for (int j = 0; j < 32; j++)
            if (r < n && j < r)
                w.T[r * ld + j] = t ? tb1[j] : tb0[j];
    }
    gsync(g);
    /* G_rj = (C-bar_rj + conj(C-bar_jr)) / 2 for j >= r (zero on the
       diagonal), by the owner of row r */
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = t ? i1 : i0;

        if (r < n) {
            float2 *row = gbar + (long long)tc_pidx(n, r, r) * npix + p;

            row[0] = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 1; j < 32; j++)
                if (j > r && j < n) {
                    float2 v = make_float2(0.f, 0.f);

                    if (active) {
                        const float2 a = t ? tb1[j] : tb0[j], b = w.T[j * ld + r];

                        v = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
                    }
                    row[(long long)(j - r) * npix] = v;
                }
        }
    }
    gsync(g);
}

/* ADJ: after gamma, backward16 writes the gradient of gamma with respect
   to the pixel's coherence sums into gbar (same layout as gram). */
template <bool EMI, bool ADJ>
__global__ void __launch_bounds__(EMI || ADJ ? 256 : 384)
tc_link_half_kernel(TcStrip s, TcChunk c, TcLinkConst k, HalfLayout L,
                    const float2 *__restrict__ gram, const int *__restrict__ count,
                    const unsigned short *__restrict__ upper_tab,
                    const unsigned short *__restrict__ pair_tab, double *__restrict__ scratch,
                    float *__restrict__ coh, float *__restrict__ pairs,
                    float *__restrict__ phases, unsigned char *__restrict__ status,
                    float2 *__restrict__ gbar, const uint32_t *__restrict__ mask,
                    int *__restrict__ queue, int qstride)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const Grp g = make_grp(lane);
    const int grp = warp * 2 + (lane >> 4);
    const HWs w = hws(smem + (size_t)grp * L.per_group, L);
    const int n = s.n, ld = L.ld;
    const long long plane = (long long)s.rows * s.cols;
    double *V = scratch + ((size_t)blockIdx.x * wpb * 2 + grp) * (size_t)(2 * n * ld + 32);
    const int i0 = g.gl, i1 = g.gl + 16;
    /* the packed-entry table, read in every stage, from shared memory */
    unsigned short *s_upper = (unsigned short *)(smem + (size_t)wpb * 2 * L.per_group);

    for (int e = threadIdx.x; e < tc_npu(n); e += blockDim.x)
        s_upper[e] = upper_tab[e];
    __syncthreads();

    /* The warps of a CTA take pixel pairs qb + warp and run each stage
       together, separated by CTA barriers: the stages' code is far larger
       than the instruction cache, and warps in different stages would keep
       evicting each other's instructions. */
    const int nq = (c.npix + 1) / 2;

    /* pixel of this group in the pair block starting at qb: its output
       index (-1 outside the output) */
    auto locate = [&](int qb, int &p) -> long long {
        const int q = qb + warp;
        int y = 0, x = 0;

        p = 2 * q + (lane >> 4);
        if (q < nq)
            tc_pixel_yx(c, p, y, x);
        const bool inrange =
            q < nq && p < c.npix && y < c.row0 + c.nrows && y < s.rows && x < s.cols;
        return inrange ? (long long)y * s.cols + x : -1ll;
    };
    TFirst tf;
    int next_p = 0;
    long long next_out = locate(blockIdx.x * wpb, next_p);
    int next_looks = next_out >= 0 ? count[next_out] : -1;

    t_first(tf, n, next_p, next_out >= 0, gram, g);
    for (int qb = blockIdx.x * wpb; qb < nq; qb += gridDim.x * wpb) {
        const int q = qb + warp;
        const int p = next_p;
        const bool inrange = next_out >= 0;
        const long long out = inrange ? next_out : 0;
        const int looks = next_looks;
        bool active = inrange && looks >= k.min_looks;
        unsigned st = 0;

        if (inrange && !active) {
            if (g.gl == 0)
                coh[out] = NAN;
            for (int t = g.gl; t < k.npairs; t += 16)
                pairs[t * plane + out] = NAN;
            if (phases)
                for (int r = g.gl; r < n; r += 16)
                    phases[out * n + r] = NAN;
            if (status && g.gl == 0)
                status[out] = 0;
        }
        bool run = __any_sync(FULL, active);

        /* stage 1: coherence matrix, pair coherences, connectivity */
        bool sent = false; /* the pixel is on the exact tier's list */

        if (run) {
            bool boundary = false;

            load_T(s, c, k, p, active, looks, gram, tf, s_upper, w, ld, g, boundary);
            if (queue && active && boundary) {
                sent = true;
                if (g.gl == 0)
                    tc_exact_push(queue, qstride, out, mask, c.npix, p);
            }
            if (active)
                for (int t = g.gl; t < k.npairs; t += 16) {
                    const int i = pair_tab[t] >> 8, j = pair_tab[t] & 255;
                    const float2 tv = w.T[i * ld + j];

                    pairs[t * plane + out] = hypotf(tv.x, tv.y);
                }
            if (k.bias && active && !linked16(n, ld, w.T, g)) {
                if (g.gl == 0)
                    coh[out] = NAN;
                if (phases)
                    for (int r = g.gl; r < n; r += 16)
                        phases[out * n + r] = NAN;
                if (status && g.gl == 0)
                    status[out] = TC_STATUS_UNLINKED;
                active = false;
            }
            gsync(g);
            if (!active) {
                /* a well-conditioned stand-in keeps the group in step */
                for (int r = g.gl; r < n; r += 16)
                    for (int j = 0; j < n; j++)
                        w.T[r * ld + j] = make_float2(r == j ? 1.f : 0.f, 0.f);
                gsync(g);
            }
            run = __any_sync(FULL, active);
        }
        __syncthreads();

        float2 r0[32], r1[32];
        double2 z0 = make_double2(0.0, 0.0), z1 = z0;
        float yr[32], lambda = 0.f, norm = 0.f;
        double inv_max = INFINITY;
        float2 f0 = make_float2(0.f, 0.f), f1 = f0;
        unsigned long long piv = 0ull;

        if (!EMI) {
            /* stage 2: Householder reduction of T */
            if (run) {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    r0[j] = (i0 < n && j < n) ? w.T[i0 * ld + j] : make_float2(0.f, 0.f);
                    r1[j] = (i1 < n && j < n) ? w.T[i1 * ld + j] : make_float2(0.f, 0.f);
                }
                gsync(g);
                householder(r0, r1, n, w, ld, g);
            }
            __syncthreads();
            /* stage 3: its dominant eigenvector */
            if (run) {
                st |= eigvec(n, n - 1, w, ld, g, f0, f1, yr, lambda, norm, piv);
                z0 = make_double2(f0.x, f0.y);
                z1 = make_double2(f1.x, f1.y);
            }
            __syncthreads();
        }
        else {
            /* stage 2: |T|^-1 in double */
            if (run)
                st |= emi_inverse(n, ld, w, V, V + n * ld, V + 2 * n * ld, g, inv_max);
            __syncthreads();
            /* stage 3: M = |T|^-1 o T in float rows, Householder reduction */
            if (run) {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    r0[j] = make_float2(0.f, 0.f);
                    r1[j] = make_float2(0.f, 0.f);
                    if (j < n) {
                        if (i0 < n) {
                            const double2 m = mval(w, ld, i0, j);

                            r0[j] = make_float2((float)m.x, (float)m.y);
                        }
                        if (i1 < n) {
                            const double2 m = mval(w, ld, i1, j);

                            r1[j] = make_float2((float)m.x, (float)m.y);
                        }
                    }
                }
                gsync(g);
                /* The reduction parks its vectors in T's lower triangle,
                   which mval no longer reads (it takes T_ij from i < j). */
                householder(r0, r1, n, w, ld, g);
            }
            __syncthreads();
            /* stage 4: eigenvector of the smallest eigenvalue, refined
               where its gap is small */
            if (run) {
                st |= eigvec(n, 0, w, ld, g, f0, f1, yr, lambda, norm, piv);
                z0 = make_double2(f0.x, f0.y);
                z1 = make_double2(f1.x, f1.y);
                /* The float eigen-solve's error in gamma is about
                   3 eps_f norm / gap (gap between the two smallest
                   eigenvalues of M): 2e-5 at a relative gap of 0.005.
                   Pixels whose gap is below TC_REFINE_GAP of the norm (two
                   eigenvalues under lambda + TC_REFINE_GAP norm) refine
                   their eigenvector once in double (the golden incoherent
                   case that float EMI misses without it has a relative
                   gap of 1.6e-3). Against the bound 0.02, 0.005 left the
                   largest error over 896k pixels of the 30-date AD/EMI/-b
                   workload unchanged (3.4e-5) at 6 % less link time. */
                if (active && sturm16(w.d, w.e2f, n, lambda + TC_REFINE_GAP * norm,
                                      1.0e-30f + 1.0e-14f * norm) >= 2)
                    refine(n, ld, w, g, z0, z1, yr, piv);
                /* Pixels whose gamma the float rounding of T may move by
                   more than ~1e-5 go to the exact tier: the first-order
                   sensitivity of M's eigenvector to T grows with
                   n max|inv| / (relative eigengap of M). The gap is below
                   delta when the tridiagonal has two eigenvalues under
                   lambda + delta (one Sturm count). Calibrated against the
                   FP64 oracle on nine 320 x 320 crops (896k pixels) of the
                   30-date AD/EMI/-b workload: the bounds 3e4 and 1e5 give
                   the same largest error, 3.4e-5 (3.2 % and 1.6 % of the
                   pixels flagged), 3e5 gives 7.2e-5 (1.0 %). */
                if (queue && active && !sent) {
                    const double delta = inv_max * (double)norm / TC_EXACT_BOUND;
                    bool flag = !(delta < (double)norm);

                    if (!flag)
                        flag = sturm16(w.d, w.e2f, n, lambda + (float)delta,
                                       1.0e-30f + 1.0e-14f * norm) >= 2;
                    if (flag && g.gl == 0)
                        tc_exact_push(queue, qstride, out, mask, c.npix, p);
                }
            }
            __syncthreads();
        }
        /* last stage: phasors, temporal coherence, outputs; the next pair's
           first sums load meanwhile (after the backward stage with ADJ,
           which needs the registers) */
        auto prefetch_next = [&]() {
            next_out = locate(qb + gridDim.x * wpb, next_p);
            next_looks = next_out >= 0 ? count[next_out] : -1;
            t_first(tf, n, next_p, next_out >= 0, gram, g);
        };
        if (!ADJ)
            prefetch_next();
        float2 ssum = make_float2(0.f, 0.f);

        if (run) {
            const float gamma = gamma16(n, ld, w, g, z0, z1, s_upper, &ssum);

            if (active) {
                if (g.gl == 0)
                    coh[out] = gamma;
                if (phases)
#pragma unroll
                    for (int t = 0; t < 2; t++) {
                        const int r = t ? i1 : i0;

                        if (r < n) {
                            const float2 u = w.zs[r];

                            phases[out * n + r] = atan2f(u.y, u.x);
                        }
                    }
                if (status && g.gl == 0)
                    status[out] = (unsigned char)st;
            }
        }
        if (ADJ && q < nq) {
            if (run)
                backward16<EMI>(n, ld, w, g, z0, z1, ssum, yr, piv, looks, k.bias != 0, active,
                                (double *)(smem + (size_t)grp * L.per_group + L.off_Db), gbar,
                                c.npix, p);
            else
                for (int t = g.gl; t < tc_npu(n); t += 16)
                    gbar[(long long)t * c.npix + p] = make_float2(0.f, 0.f);
        }
        if (ADJ)
            prefetch_next();
        __syncthreads();
    }
}

HalfLayout half_layout(int n, int emi, int adj = 0)
{
    HalfLayout L;
    int off = 0;
    auto take = [&](int bytes) {
        const int o = off;

        off += (bytes + 15) & ~15;
        return o;
    };

    L.n = n;
    L.ld = n | 1;
    L.off_T = take(8 * n * L.ld);
    L.off_G = take(emi ? 8 * tc_npu(n) : 0);
    /* stage-local: the sweep's pivot rows (inverse), the Householder
       vectors (reduction) and the adjoint's vectors share one region */
    L.off_vw = take(16 * 64);
    L.off_rs = L.off_vw;
    L.off_x = L.off_vw;
    L.off_lu = take(16 * 32);
    L.off_tau = take(8 * 32);
    L.off_d = take(4 * 32);
    L.off_e = take(4 * 32);
    L.off_df = take(4 * 32);
    L.off_e2f = take(4 * 32);
    L.off_y = take(4 * 32);
    L.off_nrm = take(4 * 32);
    L.off_zs = take(8 * 32);
    L.off_lam = 0;
    L.off_Db = take(adj && emi ? 8 * n * L.ld : 0);
    L.per_group = off;
    return L;
}

} // namespace

size_t tc_link_half_scratch_bytes(int n, int sms)
{
    /* EMI only, per group (two per warp, at most 8 warps per CTA, one CTA
       per SM): |T|, the Jacobi eigenvectors and eigenvalues of the fallback
       tiers. Stacks of more than 32 dates take the shared-memory kernel. */
    if (n > 32)
        return 256;
    return (size_t)sms * 16 * (2 * n * (n | 1) + 32) * sizeof(double);
}

template <bool EMI, bool ADJ>
static cudaError_t launch_half(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                               const float2 *gram, const int *count,
                               const unsigned short *upper_tab, const unsigned short *pair_tab,
                               double *scratch, float *coh, float *pairs, float *phases,
                               unsigned char *status, float2 *gbar, const uint32_t *mask,
                               int *queue, int qstride, int sms,
                               cudaStream_t st)
{
    const HalfLayout L = half_layout(s.n, EMI, ADJ);
    const size_t per_warp = 2 * (size_t)L.per_group;
    const size_t tab = ((size_t)tc_npu(s.n) * 2 + 15) & ~(size_t)15;
    const int max_warps = EMI || ADJ ? 8 : 12;
    int wpb = (int)((227 * 1024 - tab) / per_warp);

    if (wpb > max_warps)
        wpb = max_warps;
    if (wpb < 1)
        return cudaErrorInvalidConfiguration;
    const size_t smem = per_warp * wpb + tab;
    const int want = (c.npix / 2 + wpb - 1) / wpb;
    const int blocks = want < sms ? want : sms;
    cudaError_t e = cudaFuncSetAttribute(tc_link_half_kernel<EMI, ADJ>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);

    if (e != cudaSuccess)
        return e;
    tc_link_half_kernel<EMI, ADJ><<<blocks, wpb * 32, smem, st>>>(
        s, c, k, L, gram, count, upper_tab, pair_tab, scratch, coh, pairs, phases, status, gbar,
        mask, queue, qstride);
    return cudaGetLastError();
}

cudaError_t tc_launch_link_half(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                const float2 *gram, const uint32_t *mask, const int *count,
                                const unsigned short *upper_tab, const unsigned short *pair_tab,
                                double *scratch, float *coh, float *pairs, float *phases,
                                unsigned char *status, int *queue, int qstride, int sms,
                                cudaStream_t st)
{
    if (k.emi)
        return launch_half<true, false>(s, c, k, gram, count, upper_tab, pair_tab, scratch, coh,
                                        pairs, phases, status, nullptr, mask, queue, qstride,
                                        sms, st);
    return launch_half<false, false>(s, c, k, gram, count, upper_tab, pair_tab, scratch, coh,
                                     pairs, phases, status, nullptr, mask, queue, qstride, sms,
                                     st);
}

cudaError_t tc_launch_link_adjoint(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                   const float2 *gram, const int *count,
                                   const unsigned short *upper_tab,
                                   const unsigned short *pair_tab, double *scratch, float *coh,
                                   float *pairs, float2 *gbar, int sms, cudaStream_t st)
{
    if (s.n > 32)
        return cudaErrorInvalidValue;
    if (k.emi)
        return launch_half<true, true>(s, c, k, gram, count, upper_tab, pair_tab, scratch, coh,
                                       pairs, nullptr, nullptr, gbar, nullptr, nullptr, 0, sms,
                                       st);
    return launch_half<false, true>(s, c, k, gram, count, upper_tab, pair_tab, scratch, coh,
                                    pairs, nullptr, nullptr, gbar, nullptr, nullptr, 0, sms, st);
}
