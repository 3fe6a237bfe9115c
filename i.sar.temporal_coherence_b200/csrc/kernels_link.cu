/* Phase linking and temporal coherence of every output pixel, from its
 * masked covariance (the packed upper triangle produced by a Gram kernel).
 *
 * One warp per pixel. Stages (tcoh.cl:603-744):
 *
 *   coherence matrix T_ij = C_ij / sqrt(C_ii C_jj), optional magnitude bias
 *   correction, in float with round-to-nearest intrinsics in the
 *   reference's order (tcoh.cl:610-636), kept in shared memory;
 *   pair coherences |T_ij| (tcoh.cl:515-527, 639);
 *   connectivity of the non-zero T_ij under the bias correction, as a
 *   bit-parallel breadth-first search (tcoh.cl:494-513, 644-647);
 *   EVD: eigenvector of the largest eigenvalue of T, in float (as
 *   tcoh.cl:649-656); EMI: eigenvector of the smallest eigenvalue of
 *   M = |T|^-1 o T (tcoh.cl:657-694), all in double: |T| is inverted by
 *   the symmetric sweep (Gauss-Jordan without pivoting, which takes the
 *   indefinite |T| of noisy stacks) when its pivots stay above 1e-5 in
 *   magnitude and the inverse stays moderate, else by its Jacobi
 *   eigen-pseudo-inverse with the absolute eigenvalue floor 1e-9 of
 *   tests/reference.py:151-156; the two differ only near singularity,
 *   since the pseudo-inverse of a matrix whose eigenvalues all exceed 1e-9
 *   in magnitude is its inverse;
 *   the eigenvector is one Householder reduction to a real tridiagonal
 *   (LAPACK zhetd2 form), a 33-way multisection on Sturm counts for the
 *   wanted eigenvalue, inverse iteration on the tridiagonal and the
 *   back-transformation (the method of tcoh.cl:201-444);
 *   unit phasors relative to the median date (or the strongest component
 *   when it is negligible) and the Pepe-Lanari goodness of fit
 *   (tcoh.cl:696-744).
 *
 * This file holds the path for 33 to 64 dates, where the matrices stay in
 * shared memory, two rows per lane. With EMI, |T| and its inverse occupy
 * the first half of the working matrix's region (the Jacobi fallback's
 * eigenvectors the second half) until M is formed over them, so that a
 * warp needs T plus one complex double matrix: two warps per SM at 60
 * dates. Up to 32 dates the
 * faster register path of kernels_link_half.cu runs instead (same stages,
 * same numerics, two pixels per warp).
 */
#include "tcoh_internal.h"

#include <math.h>

#define FULL 0xffffffffu

namespace {

/* ------------------------------------------------------------------ */
/* Scalars and complex numbers of either precision.                    */
/* ------------------------------------------------------------------ */

template <typename R> struct Cx;
template <> struct Cx<float> {
    typedef float2 T;
};
template <> struct Cx<double> {
    typedef double2 T;
};

template <typename R>
__device__ __forceinline__ typename Cx<R>::T mk(R x, R y)
{
    typename Cx<R>::T c;

    c.x = x;
    c.y = y;
    return c;
}

template <typename R>
__device__ __forceinline__ R wsum(R v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ float wmax(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

__device__ __forceinline__ float wmin(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v = fminf(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

/* ------------------------------------------------------------------ */
/* Per-warp shared workspace (8-byte units).                           */
/* ------------------------------------------------------------------ */

struct LinkLayout {
    int n, ld;        /* dates, odd leading dimension >= n */
    int nv;           /* vector length: max(n, 32) */
    int off_T, off_G, off_A, off_vec;
    int per_warp;
};

struct Ws {
    float2 *T;   /* n x ld normalized coherence */
    double *G;   /* n x ld |T| and its inverse (EMI) */
    void *A;     /* n x ld working matrix of the shared-memory path */
    /* vectors */
    void *d, *e, *y;   /* tridiagonal, eigenvector (R) */
    void *lu;          /* 4 n (R): LU of the shifted tridiagonal */
    void *tau;         /* n (complex R) */
    void *vw;          /* 4 nv units: Householder v, w / Gauss-Jordan row */
    float *df, *e2f;   /* float copies for the Sturm counts */
    float *nrm;        /* sqrt(C_ii) */
    float2 *zs;        /* unit phasors */
    double *lam;       /* eigenvalues of |T| (pseudo-inverse) */
};

/* Offsets are kept even (16-byte aligned) for the float4 / double2 arrays. */
__host__ __device__ __forceinline__ int even(int x) { return (x + 1) & ~1; }

__device__ __forceinline__ Ws workspace(double *base, const LinkLayout &L)
{
    Ws w;
    double *v = base + L.off_vec;
    const int an = even(L.n), nv = L.nv;

    w.T = (float2 *)(base + L.off_T);
    w.G = base + L.off_G;
    w.A = base + L.off_A;
    w.d = v;
    w.e = v + an;
    w.y = v + 2 * an;
    w.lu = v + 3 * an;                    /* 4n */
    w.tau = v + 7 * an;                   /* 2n */
    w.vw = v + 9 * an;                    /* 4 nv */
    w.df = (float *)(v + 9 * an + 4 * nv);
    w.e2f = (float *)(v + 10 * an + 4 * nv);
    w.nrm = (float *)(v + 11 * an + 4 * nv);
    w.zs = (float2 *)(v + 12 * an + 4 * nv);
    w.lam = v + 13 * an + 4 * nv;
    return w;
}

#define VEC_UNITS(n, nv) (14 * even(n) + 4 * even(nv))

/* ------------------------------------------------------------------ */
/* Tridiagonal eigenvector.                                            */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp(double x) { return 1.0 / x; }

/* Number of eigenvalues of the double tridiagonal (d, e) below x. Only the
   signs matter: 1/q comes from the float reciprocal and one Newton step
   (relative error ~1e-14). */
__device__ __forceinline__ int sturmd(const double *d, const double *e2, int n, double x,
                                      double pivmin)
{
    double q = d[0] - x;
    int c = q < 0.0;

    for (int i = 1; i < n; i++) {
        if (fabs(q) < pivmin)
            q = -pivmin;
        double r = (double)__frcp_rn((float)q);

        r = r * fma(-q, r, 2.0);
        q = d[i] - x - e2[i - 1] * r;
        c += q < 0.0;
    }
    return c;
}

__device__ __forceinline__ int sturmf(const float *d, const float *e2, int n, float x,
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

/* One round of 33-way multisection of [lo, hi] for the eigenvalue of rank
   `index`. Returns false when the interval stopped shrinking. */
template <typename R, typename F>
__device__ __forceinline__ bool multisect(R &lo, R &hi, int index, int lane, F count)
{
    const R xq = lo + (hi - lo) * ((R)(lane + 1) / (R)33);
    const int cnt = count(xq);
    const unsigned gt = __ballot_sync(FULL, cnt > index);
    R nlo, nhi;

    if (gt == 0u) {
        nlo = __shfl_sync(FULL, xq, 31);
        nhi = hi;
    }
    else {
        const int f = __ffs(gt) - 1;

        nhi = __shfl_sync(FULL, xq, f);
        nlo = __shfl_sync(FULL, xq, f > 0 ? f - 1 : 0);
        if (f == 0)
            nlo = lo;
    }
    nlo = nlo > lo ? nlo : lo;
    nhi = nhi < hi ? nhi : hi;
    if (!(nlo > lo || nhi < hi))
        return false;
    lo = nlo;
    hi = nhi;
    return true;
}

/* Eigenvalue of rank `index` of the tridiagonal (w.d, w.e) (R), then its
   eigenvector into w.y by inverse iteration (lane 0). The counts run in
   float; for double tridiagonals three double rounds refine the float
   interval. Returns status bits. */
template <typename R>
__device__ unsigned tridiag_vector(int n, int index, const Ws &w, int lane)
{
    R *d = (R *)w.d, *e = (R *)w.e, *y = (R *)w.y;
    R *lu = (R *)w.lu;
    unsigned status = 0;
    float lo = INFINITY, hi = -INFINITY;

    for (int r = lane; r < n; r += 32) {
        const R rad = (r > 0 ? fabs(e[r - 1]) : (R)0) + (r < n - 1 ? fabs(e[r]) : (R)0);

        lo = fminf(lo, (float)(d[r] - rad));
        hi = fmaxf(hi, (float)(d[r] + rad));
        w.df[r] = (float)d[r];
        if (r < n - 1)
            w.e2f[r] = (float)(e[r] * e[r]);
    }
    lo = wmin(lo);
    hi = wmax(hi);
    /* Gershgorin bounds in float: widen by a relative 1e-6 for safety. */
    const float normf = fmaxf(fabsf(lo), fabsf(hi));

    lo -= 1.0e-6f * normf + 1.0e-30f;
    hi += 1.0e-6f * normf + 1.0e-30f;
    __syncwarp();
    {
        const float pivmin = 1.0e-30f + 1.0e-14f * normf;
        auto cf = [&](float x) { return sturmf(w.df, w.e2f, n, x, pivmin); };
        int round = 0;

        for (; round < 16; round++)
            if (!multisect<float>(lo, hi, index, lane, cf))
                break;
        if (round == 16)
            status |= TC_STATUS_ITER_CAP;
    }
    R lambda;

    if constexpr (sizeof(R) == 8) {
        /* The float interval can be off by the rounding of the float
           counts: widen it by a few of its ulps, then three double rounds. */
        const R norm = (R)normf;
        R dlo = (R)lo - (R)4.0e-7 * norm - (R)1e-300;
        R dhi = (R)hi + (R)4.0e-7 * norm + (R)1e-300;
        R *e2 = (R *)w.lu; /* scratch before the LU */

        for (int r = lane; r < n - 1; r += 32)
            e2[r] = e[r] * e[r];
        __syncwarp();
        const R pivmin = (R)1e-290 + (R)1e-28 * norm;
        auto cd = [&](R x) { return sturmd((const double *)d, (const double *)e2, n, (double)x, (double)pivmin); };

        for (int round = 0; round < 3; round++)
            if (!multisect<R>(dlo, dhi, index, lane, cd))
                break;
        lambda = (R)0.5 * (dlo + dhi);
        __syncwarp();
    }
    else
        lambda = (R)0.5 * (R)(lo + hi);

    /* Inverse iteration: LU of T - lambda I with partial pivoting, three
       solves from a vector of ones (tcoh.cl:342-410). Every lane runs it
       on the same values (lane 0 stores the factors), with the iterate in
       registers; lane r then keeps y[r]. */
    const R norm = (R)normf;
    const R tiny = (sizeof(R) == 8 ? (R)1.0e-13 : (R)1.0e-6) * (norm > (R)1e-30 ? norm : (R)1e-30);
    unsigned long long piv = 0ull;
    {
        R dd = d[0] - lambda, s1 = n > 1 ? e[0] : (R)0;

        for (int k = 0; k < n - 1; k++) {
            const R sub = e[k], nd = d[k + 1] - lambda;
            const R ns = k + 1 < n - 1 ? e[k + 1] : (R)0;

            if (fabs(dd) >= fabs(sub)) {
                if (fabs(dd) < tiny)
                    dd = dd < (R)0 ? -tiny : tiny;
                const R rd = rcp(dd), l = sub * rd;

                if (lane == 0) {
                    lu[4 * k] = rd;
                    lu[4 * k + 1] = s1;
                    lu[4 * k + 2] = 0;
                    lu[4 * k + 3] = l;
                }
                dd = nd - l * s1;
                s1 = ns;
            }
            else {
                const R rs = rcp(sub), l = dd * rs;

                piv |= 1ull << k;
                if (lane == 0) {
                    lu[4 * k] = rs;
                    lu[4 * k + 1] = nd;
                    lu[4 * k + 2] = ns;
                    lu[4 * k + 3] = l;
                }
                dd = s1 - l * nd;
                s1 = -l * ns;
            }
        }
        if (fabs(dd) < tiny)
            dd = dd < (R)0 ? -tiny : tiny;
        if (lane == 0) {
            lu[4 * (n - 1)] = rcp(dd);
            lu[4 * (n - 1) + 1] = 0;
            lu[4 * (n - 1) + 2] = 0;
        }
    }
    __syncwarp();
    if (n > 32) {
        /* Lane 0 alone, on the shared copy. */
        if (lane == 0) {
            for (int k = 0; k < n; k++)
                y[k] = 1;
            for (int it = 0; it < 3; it++) {
                R nrm = 0;

                for (int k = 0; k < n - 1; k++) {
                    if ((piv >> k) & 1ull) {
                        const R t = y[k];

                        y[k] = y[k + 1];
                        y[k + 1] = t;
                    }
                    y[k + 1] -= lu[4 * k + 3] * y[k];
                }
                for (int k = n - 1; k >= 0; k--) {
                    R v = y[k];

                    if (k + 1 < n)
                        v -= lu[4 * k + 1] * y[k + 1];
                    if (k + 2 < n)
                        v -= lu[4 * k + 2] * y[k + 2];
                    y[k] = v * lu[4 * k];
                    nrm = fmax(nrm, fabs(y[k]));
                }
                const R inv = rcp(nrm);

                for (int k = 0; k < n; k++)
                    y[k] *= inv;
            }
        }
        __syncwarp();
        return status;
    }
    R yr[32];

#pragma unroll
    for (int k = 0; k < 32; k++)
        yr[k] = 1;
    for (int it = 0; it < 3; it++) {
#pragma unroll
        for (int k = 0; k < 31; k++) {
            if (k >= n - 1)
                break;
            if ((piv >> k) & 1ull) {
                const R t = yr[k];

                yr[k] = yr[k + 1];
                yr[k + 1] = t;
            }
            yr[k + 1] -= lu[4 * k + 3] * yr[k];
        }
        R nrm = 0;

#pragma unroll
        for (int k = 31; k >= 0; k--) {
            if (k > n - 1)
                continue;
            R v = yr[k];

            if (k + 1 < n)
                v -= lu[4 * k + 1] * yr[k + 1];
            if (k + 2 < n)
                v -= lu[4 * k + 2] * yr[k + 2];
            yr[k] = v * lu[4 * k];
            nrm = fmax(nrm, fabs(yr[k]));
        }
        const R inv = rcp(nrm);

#pragma unroll
        for (int k = 0; k < 32; k++)
            yr[k] *= inv;
    }
    R mine = 0;

#pragma unroll
    for (int k = 0; k < 32; k++)
        if (k == lane)
            mine = yr[k];
    if (lane < n)
        y[lane] = mine;
    __syncwarp();
    return status;
}

/* ------------------------------------------------------------------ */
/* Shared-memory path (N <= 64).                                       */
/* ------------------------------------------------------------------ */

template <typename R>
__device__ unsigned heig_smem(int n, int ld, typename Cx<R>::T *A, int index, const Ws &ws,
                              int lane, typename Cx<R>::T (&zo)[2])
{
    typedef typename Cx<R>::T C;
    R *d = (R *)ws.d, *e = (R *)ws.e;
    C *tau = (C *)ws.tau;
    C *vv = (C *)ws.vw, *wwv = vv + n;

    for (int k = 0; k < n - 1; k++) {
        R xn2 = 0;

        for (int r = lane; r < n; r += 32)
            if (r >= k + 2) {
                const C a = A[r * ld + k];

                xn2 += a.x * a.x + a.y * a.y;
            }
        xn2 = wsum<R>(xn2);
        const C alpha = A[(k + 1) * ld + k];
        const R dk = A[k * ld + k].x;
        R beta, tr = 0, ti = 0;

        __syncwarp();
        if (xn2 == (R)0 && alpha.y == (R)0)
            beta = alpha.x;
        else {
            beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
            tr = (beta - alpha.x) / beta;
            ti = -alpha.y / beta;
            const R dr = alpha.x - beta, di = alpha.y, den = dr * dr + di * di;
            const R sr = dr / den, si = -di / den;

            for (int r = lane; r < n; r += 32)
                if (r >= k + 2) {
                    const C a = A[r * ld + k];

                    A[r * ld + k] = mk<R>(a.x * sr - a.y * si, a.x * si + a.y * sr);
                }
        }
        if (lane == 0) {
            d[k] = dk;
            e[k] = beta;
            tau[k] = mk<R>(tr, ti);
            A[(k + 1) * ld + k] = mk<R>(1, 0);
        }
        __syncwarp();
        if (tr == (R)0 && ti == (R)0)
            continue;
        for (int r = lane; r < n; r += 32)
            vv[r] = r > k ? A[r * ld + k] : mk<R>(0, 0);
        __syncwarp();
        C wl[2];
        R pr = 0, pi = 0;

#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = lane + 32 * t;

            wl[t] = mk<R>(0, 0);
            if (r > k && r < n) {
                R sr = 0, si = 0;
                const C *row = A + r * ld;

                for (int j = k + 1; j < n; j++) {
                    const C a = row[j], v = vv[j];

                    sr += a.x * v.x - a.y * v.y;
                    si += a.x * v.y + a.y * v.x;
                }
                wl[t] = mk<R>(tr * sr - ti * si, tr * si + ti * sr);
                const C v = vv[r];

                pr += wl[t].x * v.x + wl[t].y * v.y;
                pi += wl[t].x * v.y - wl[t].y * v.x;
            }
        }
        pr = wsum<R>(pr);
        pi = wsum<R>(pi);
        const R hr = (R)-0.5 * (tr * pr - ti * pi), hi = (R)-0.5 * (tr * pi + ti * pr);

#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = lane + 32 * t;

            if (r > k && r < n) {
                const C v = vv[r];

                wl[t].x += hr * v.x - hi * v.y;
                wl[t].y += hr * v.y + hi * v.x;
                wwv[r] = wl[t];
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = lane + 32 * t;

            if (r > k && r < n) {
                const C vr = vv[r], wr = wwv[r];
                C *row = A + r * ld;

                for (int j = k + 1; j < n; j++) {
                    const C vj = vv[j], wj = wwv[j];
                    C a = row[j];

                    a.x -= vr.x * wj.x + vr.y * wj.y + wr.x * vj.x + wr.y * vj.y;
                    a.y -= vr.y * wj.x - vr.x * wj.y + wr.y * vj.x - wr.x * vj.y;
                    row[j] = a;
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0)
        d[n - 1] = A[(n - 1) * ld + n - 1].x;
    __syncwarp();
    unsigned status = tridiag_vector<R>(n, index, ws, lane);
    const R *y = (const R *)ws.y;
    C z[2];

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = lane + 32 * t;

        z[t] = mk<R>(r < n ? y[r] : (R)0, 0);
    }
    for (int k = n - 2; k >= 0; k--) {
        const C ta = tau[k];

        if (ta.x == (R)0 && ta.y == (R)0)
            continue;
        R sr = 0, si = 0;

#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = lane + 32 * t;

            if (r > k && r < n) {
                const C v = A[r * ld + k];

                sr += v.x * z[t].x + v.y * z[t].y;
                si += v.x * z[t].y - v.y * z[t].x;
            }
        }
        sr = wsum<R>(sr);
        si = wsum<R>(si);
        const R hr = ta.x * sr - ta.y * si, hi2 = ta.x * si + ta.y * sr;

#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int r = lane + 32 * t;

            if (r > k && r < n) {
                const C v = A[r * ld + k];

                z[t].x -= v.x * hr - v.y * hi2;
                z[t].y -= v.x * hi2 + v.y * hr;
            }
        }
    }
    zo[0] = z[0];
    zo[1] = z[1];
    return status;
}

/* In-place inverse of the symmetric W (double, full storage, shared
   memory) by the symmetric sweep (Gauss-Jordan elimination without
   pivoting in the form that keeps the matrix symmetric; Goodnight, The
   American Statistician 33, 1979): sweeping pivot k maps
       a_ij -> a_ij - a_ik a_kj / a_kk,  a_ik, a_kj -> a_ik / a_kk,
       a_kk -> -1 / a_kk,
   and sweeping every pivot leaves -W^-1. It takes indefinite matrices. row
   is n doubles of scratch (the pivot row before the step). False when a
   pivot's magnitude is not above 1e-5, or when the inverse is not finite or
   so large (n max|inv| >= 1e8) that an eigenvalue may lie below the
   pseudo-inverse floor 1e-9; W is then undefined. */
__device__ bool sweep_inverse_smem(int n, int ld, double *W, double *row, int lane)
{
    for (int k = 0; k < n; k++) {
        const double d = W[k * ld + k];

        if (!(fabs(d) > 1.0e-5))
            return false;
        const double id = 1.0 / d;

        for (int j = lane; j < n; j += 32)
            row[j] = W[k * ld + j];
        __syncwarp();
        for (int r = lane; r < n; r += 32) {
            double *wr = W + r * ld;

            if (r == k)
                for (int j = 0; j < n; j++)
                    wr[j] = j == k ? -id : row[j] * id;
            else {
                const double f = wr[k] * id;

                for (int j = 0; j < n; j++)
                    wr[j] = j == k ? f : fma(-f, row[j], wr[j]);
            }
        }
        __syncwarp();
    }
    double mx = 0.0;
    bool bad = false;

    for (int r = lane; r < n; r += 32)
        for (int j = 0; j < n; j++) {
            const double v = -W[r * ld + j];

            W[r * ld + j] = v;
            bad |= !(fabs(v) <= 1.0e300);
            mx = fmax(mx, fabs(v));
        }
#pragma unroll
    for (int o = 16; o; o >>= 1)
        mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
    bad = __any_sync(FULL, bad);
    __syncwarp();
    return !bad && n * mx < 1.0e8;
}

/* Pseudo-inverse of the symmetric W (double, full storage) in place, from
   its cyclic Jacobi eigendecomposition; eigenvalues |l| < 1e-9 are dropped
   (tests/reference.py:151-156). V is workspace (n x ld). Returns status
   bits. */
__device__ unsigned jacobi_pinv(int n, int ld, double *W, double *V, double *lam, int lane)
{
    unsigned status = TC_STATUS_ITER_CAP;

    for (int r = lane; r < n; r += 32)
        for (int j = 0; j < n; j++)
            V[r * ld + j] = r == j ? 1.0 : 0.0;
    __syncwarp();
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0, dg = 0.0;

        for (int r = lane; r < n; r += 32)
            for (int j = 0; j < n; j++) {
                const double w = W[r * ld + j];

                if (j == r)
                    dg += w * w;
                else
                    off += w * w;
            }
        off = wsum<double>(off);
        dg = wsum<double>(dg);
        if (off <= 1.0e-30 * dg) {
            status = 0;
            break;
        }
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = W[p * ld + q];

                if (apq == 0.0)
                    continue;
                const double app = W[p * ld + p], aqq = W[q * ld + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                                 (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;

                __syncwarp();
                for (int r = lane; r < n; r += 32) {
                    if (r != p && r != q) {
                        const double akp = W[r * ld + p], akq = W[r * ld + q];

                        W[r * ld + p] = c * akp - s * akq;
                        W[r * ld + q] = s * akp + c * akq;
                    }
                    const double vkp = V[r * ld + p], vkq = V[r * ld + q];

                    V[r * ld + p] = c * vkp - s * vkq;
                    V[r * ld + q] = s * vkp + c * vkq;
                }
                __syncwarp();
                for (int r = lane; r < n; r += 32)
                    if (r != p && r != q) {
                        W[p * ld + r] = W[r * ld + p];
                        W[q * ld + r] = W[r * ld + q];
                    }
                if (lane == 0) {
                    W[p * ld + p] = app - t * apq;
                    W[q * ld + q] = aqq + t * apq;
                    W[p * ld + q] = 0.0;
                    W[q * ld + p] = 0.0;
                }
                __syncwarp();
            }
    }
    for (int r = lane; r < n; r += 32)
        lam[r] = W[r * ld + r];
    __syncwarp();
    for (int i = lane; i < n; i += 32)
        for (int j = 0; j < n; j++) {
            double s = 0.0;

            for (int k = 0; k < n; k++) {
                const double l = lam[k];

                if (fabs(l) >= 1.0e-9)
                    s += V[i * ld + k] * V[j * ld + k] / l;
            }
            W[i * ld + j] = s;
        }
    __syncwarp();
    return status;
}

/* ------------------------------------------------------------------ */
/* Common stages.                                                      */
/* ------------------------------------------------------------------ */

struct PixelCtx {
    int n, ld;
    long long out, plane;
};

/* T from the packed Gram sums (tcoh.cl:611-636). */
__device__ void load_coherence(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                               int p, int looks, const float2 *__restrict__ gram,
                               const unsigned short *__restrict__ upper_tab, const Ws &w,
                               int ld, int lane)
{
    const int n = s.n, npu = tc_npu(n);

    for (int r = lane; r < n; r += 32)
        w.nrm[r] = __fsqrt_rn(gram[tc_gram_at(tc_npu(n), p, tc_pidx(n, r, r))].x);
    __syncwarp();
    const float fl = (float)looks;

    for (int q = lane; q < npu; q += 32) {
        const int i = upper_tab[q] >> 8, j = upper_tab[q] & 255;

        if (i == j) {
            w.T[i * ld + i] = make_float2(1.f, 0.f);
            continue;
        }
        const float2 g = gram[tc_gram_at(tc_npu(n), p, q)];
        const float dd = __fmul_rn(w.nrm[i], w.nrm[j]);
        float re = 0.f, im = 0.f;

        if (dd > 0.f) {
            re = __fdiv_rn(g.x, dd);
            im = __fdiv_rn(g.y, dd);
            if (k.bias && looks > 1) {
                const float m2 = __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im));
                const float m2c =
                    __fdiv_rn(__fsub_rn(__fmul_rn(fl, m2), 1.0f), __fsub_rn(fl, 1.0f));
                const float f = (m2 > 0.f && m2c > 0.f) ? __fsqrt_rn(__fdiv_rn(m2c, m2)) : 0.f;

                re = __fmul_rn(re, f);
                im = __fmul_rn(im, f);
            }
        }
        w.T[i * ld + j] = make_float2(re, im);
        w.T[j * ld + i] = make_float2(re, -im);
    }
    __syncwarp();
}

/* Whether the non-zero coherences link all dates. */
__device__ bool linked(int n, int ld, const float2 *T, int lane)
{
    unsigned long long adj[2] = {0ull, 0ull};

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = lane + 32 * t;

        if (r < n)
            for (int j = 0; j < n; j++) {
                const float2 v = T[r * ld + j];

                if (j != r && (v.x != 0.f || v.y != 0.f))
                    adj[t] |= 1ull << j;
            }
    }
    const unsigned long long all = n == 64 ? ~0ull : (1ull << n) - 1ull;
    unsigned long long reached = 1ull, frontier = 1ull;

    for (int it = 0; it < n; it++) {
        unsigned long long mine = 0ull;

        if ((frontier >> lane) & 1ull)
            mine |= adj[0];
        if (lane + 32 < n && ((frontier >> (lane + 32)) & 1ull))
            mine |= adj[1];
        const unsigned lo = __reduce_or_sync(FULL, (unsigned)mine);
        const unsigned hi = __reduce_or_sync(FULL, (unsigned)(mine >> 32));
        const unsigned long long nw = (((unsigned long long)hi << 32) | lo) & ~reached;

        if (!nw)
            break;
        reached |= nw;
        frontier = nw;
    }
    return reached == all;
}

/* Unit phasors relative to the median date (tcoh.cl:700-724) from the
   eigenvector components of rows lane and lane + 32 (R), into w.zs; then
   the goodness of fit (tcoh.cl:728-744). Returns gamma on every lane. */
template <typename R>
__device__ float phasors_and_gamma(int n, int ld, const Ws &w,
                                   const typename Cx<R>::T (&z)[2],
                                   const unsigned short *__restrict__ upper_tab, int lane)
{
    R m[2];

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = lane + 32 * t;

        m[t] = r < n ? hypot(z[t].x, z[t].y) : (R)0;
    }
    R mx = m[0] > m[1] ? m[0] : m[1];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const R other = __shfl_xor_sync(FULL, mx, o);

        mx = other > mx ? other : mx;
    }
    int ref = n / 2;
    {
        const R mref = __shfl_sync(FULL, ref < 32 ? m[0] : m[1], ref & 31);

        if (mref <= (R)1.0e-3 * mx) {
            int last = -1;

#pragma unroll
            for (int t = 0; t < 2; t++) {
                const int r = lane + 32 * t;

                if (r < n && m[t] == mx)
                    last = max(last, r);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1)
                last = max(last, __shfl_xor_sync(FULL, last, o));
            ref = last;
        }
    }
    const int rt = ref >> 5, rl = ref & 31;
    const R zrx = __shfl_sync(FULL, rt ? z[1].x : z[0].x, rl);
    const R zry = __shfl_sync(FULL, rt ? z[1].y : z[0].y, rl);
    const R refm = hypot(zrx, zry);
    const R refr = zrx / refm, refi = -zry / refm;
    const R floor_ = mx * (R)1.0e-3;
    float2 u[2];

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = lane + 32 * t;

        u[t] = make_float2(1.f, 0.f);
        if (r < n) {
            const R re = z[t].x * refr - z[t].y * refi;
            const R im = z[t].x * refi + z[t].y * refr;
            const R mm = hypot(re, im);

            if (mm > floor_)
                u[t] = make_float2((float)(re / mm), (float)(im / mm));
            w.zs[r] = u[t];
        }
    }
    __syncwarp();
    /* pairs spread evenly over the lanes */
    float sr = 0.f, si = 0.f;
    const int npu = tc_npu(n);

    for (int q = lane; q < npu; q += 32) {
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
    sr = wsum<float>(sr);
    si = wsum<float>(si);
    return hypotf(sr, si) / (0.5f * n * (n - 1));
}

/* ------------------------------------------------------------------ */
/* Kernels.                                                            */
/* ------------------------------------------------------------------ */

__global__ void __launch_bounds__(256)
tc_link_smem_kernel(TcStrip s, TcChunk c, TcLinkConst k, LinkLayout L,
                    const float2 *__restrict__ gram, const int *__restrict__ count,
                    const unsigned short *__restrict__ upper_tab,
                    const unsigned short *__restrict__ pair_tab, double *__restrict__ scratch,
                    float *__restrict__ coh, float *__restrict__ pairs,
                    float *__restrict__ phases, unsigned char *__restrict__ status)
{
    extern __shared__ double smd[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int n = s.n, ld = L.ld;
    const Ws w = workspace(smd + (size_t)warp * L.per_warp, L);
    const long long plane = (long long)s.rows * s.cols;

    (void)scratch;
    for (int p = blockIdx.x * wpb + warp; p < c.npix; p += gridDim.x * wpb) {
        int y, x;

        tc_pixel_yx(c, p, y, x);
        if (y >= c.row0 + c.nrows || y >= s.rows || x >= s.cols)
            continue;
        const long long out = (long long)y * s.cols + x;
        const int looks = count[out];

        if (looks < k.min_looks) {
            if (lane == 0)
                coh[out] = NAN;
            for (int q = lane; q < k.npairs; q += 32)
                pairs[q * plane + out] = NAN;
            if (phases)
                for (int r = lane; r < n; r += 32)
                    phases[out * n + r] = NAN;
            if (status && lane == 0)
                status[out] = 0;
            continue;
        }
        load_coherence(s, c, k, p, looks, gram, upper_tab, w, ld, lane);
        for (int q = lane; q < k.npairs; q += 32) {
            const int i = pair_tab[q] >> 8, j = pair_tab[q] & 255;
            const float2 t = w.T[i * ld + j];

            pairs[q * plane + out] = hypotf(t.x, t.y);
        }
        unsigned st = 0;

        if (k.bias && !linked(n, ld, w.T, lane)) {
            if (lane == 0)
                coh[out] = NAN;
            if (phases)
                for (int r = lane; r < n; r += 32)
                    phases[out * n + r] = NAN;
            if (status && lane == 0)
                status[out] = TC_STATUS_UNLINKED;
            __syncwarp();
            continue;
        }
        float gamma;

        if (!k.emi) {
            float2 *A = (float2 *)w.A;

            for (int r = lane; r < n; r += 32)
                for (int j = 0; j < n; j++)
                    A[r * ld + j] = w.T[r * ld + j];
            __syncwarp();
            float2 z[2];

            st |= heig_smem<float>(n, ld, A, n - 1, w, lane, z);
            gamma = phasors_and_gamma<float>(n, ld, w, z, upper_tab, lane);
        }
        else {
            /* |T| and its inverse in w.G, the first half of the working
               matrix's region; the second half holds the Jacobi fallback's
               eigenvectors */
            double2 *A = (double2 *)w.A;
            double *V = w.G + n * ld;

            for (int r = lane; r < n; r += 32)
                for (int j = 0; j < n; j++) {
                    const float2 t = w.T[r * ld + j];

                    w.G[r * ld + j] = hypot((double)t.x, (double)t.y);
                }
            __syncwarp();
            if (!sweep_inverse_smem(n, ld, w.G, (double *)w.vw, lane)) {
                __syncwarp();
                for (int r = lane; r < n; r += 32)
                    for (int j = 0; j < n; j++) {
                        const float2 t = w.T[r * ld + j];

                        w.G[r * ld + j] = hypot((double)t.x, (double)t.y);
                    }
                __syncwarp();
                st |= TC_STATUS_EMI_PINV | jacobi_pinv(n, ld, w.G, V, w.lam, lane);
            }
            /* M = |T|^-1 o T over the same region, 32 entries at a time from
               the last one down: complex entry q covers |T|^-1 entries 2q and
               2q + 1, which are above the block being read (or in it, read
               before the barrier) and so already consumed */
            const int total = n * ld;

            for (int base = (total - 1) & ~31; base >= 0; base -= 32) {
                const int q = base + lane;
                double2 v = make_double2(0.0, 0.0);

                if (q < total) {
                    const int r = q / ld, j = q - r * ld;

                    if (j < n) {
                        const float2 t = w.T[r * ld + j];
                        const double gg = w.G[q];

                        v = make_double2(gg * (double)t.x, gg * (double)t.y);
                    }
                }
                __syncwarp();
                if (q < total)
                    A[q] = v;
                __syncwarp();
            }
            double2 z[2];

            st |= heig_smem<double>(n, ld, A, 0, w, lane, z);
            gamma = phasors_and_gamma<double>(n, ld, w, z, upper_tab, lane);
        }
        if (lane == 0)
            coh[out] = gamma;
        if (phases)
            for (int r = lane; r < n; r += 32) {
                const float2 u = w.zs[r];

                phases[out * n + r] = atan2f(u.y, u.x);
            }
        if (status && lane == 0)
            status[out] = (unsigned char)st;
        __syncwarp();
    }
}

LinkLayout layout_for(int n, int emi, bool regs)
{
    LinkLayout L;

    L.n = n;
    L.ld = n | 1;
    L.nv = even(n > 32 ? n : 32);
    L.off_T = 0;
    if (emi && !regs) {
        /* |T| and its inverse share the working matrix's region */
        L.off_A = even(n * L.ld);
        L.off_G = L.off_A;
        L.off_vec = even(L.off_A + 2 * n * L.ld);
    }
    else {
        L.off_G = even(n * L.ld);
        L.off_A = even(L.off_G + (emi ? n * L.ld : 0));
        L.off_vec = even(L.off_A + (regs ? 0 : (emi ? 2 : 1) * n * L.ld));
    }
    L.per_warp = even(L.off_vec + VEC_UNITS(n, L.nv));
    return L;
}

} // namespace

size_t tc_link_scratch_bytes(int n, int sms)
{
    return tc_link_half_scratch_bytes(n, sms);
}

cudaError_t tc_launch_link(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                           const float2 *gram, const int *count,
                           const unsigned short *upper_tab, const unsigned short *pair_tab,
                           double *scratch, float *coh, float *pairs, float *phases,
                           unsigned char *status, int sms, cudaStream_t st)
{
    if (s.n <= 32)
        return tc_launch_link_half(s, c, k, gram, count, upper_tab, pair_tab, scratch, coh,
                                   pairs, phases, status, sms, st);
    const LinkLayout L = layout_for(s.n, k.emi, false);
    const size_t per_warp = (size_t)L.per_warp * sizeof(double);
    int wpb = (int)((227 * 1024) / per_warp);

    if (wpb > 8)
        wpb = 8;
    if (wpb < 1)
        return cudaErrorInvalidConfiguration;
    const size_t smem = per_warp * wpb;
    const int want = (c.npix + wpb - 1) / wpb;
    const int blocks = want < sms ? want : sms;
    cudaError_t e = cudaFuncSetAttribute(tc_link_smem_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);

    if (e == cudaSuccess)
        tc_link_smem_kernel<<<blocks, wpb * 32, smem, st>>>(
            s, c, k, L, gram, count, upper_tab, pair_tab, scratch, coh, pairs, phases, status);
    if (e != cudaSuccess)
        return e;
    return cudaGetLastError();
}
