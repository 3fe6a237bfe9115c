/* Phase linking and temporal coherence of every output pixel, from its
 * masked covariance (the packed upper triangle produced by a Gram kernel),
 * for stacks of 33 to 64 dates, and the exact tier of EMI (any number of
 * dates up to 64; see tc_link_exact_kernel below).
 *
 * EVD, one warp per pixel. Stages (tcoh.cl:603-744):
 *
 *   coherence matrix T_ij = C_ij / sqrt(C_ii C_jj), optional magnitude bias
 *   correction, in float with round-to-nearest intrinsics in the
 *   reference's order (tcoh.cl:610-636), kept in shared memory;
 *   pair coherences |T_ij| (tcoh.cl:515-527, 639);
 *   connectivity of the non-zero T_ij under the bias correction, as a
 *   bit-parallel breadth-first search (tcoh.cl:494-513, 644-647);
 *   the eigenvector of the largest eigenvalue of T, in float (as
 *   tcoh.cl:649-656): one Householder reduction to a real tridiagonal
 *   (LAPACK zhetd2 form), a 33-way multisection on Sturm counts for the
 *   wanted eigenvalue, inverse iteration on the tridiagonal and the
 *   back-transformation (the method of tcoh.cl:201-444);
 *   unit phasors relative to the median date (or the strongest component
 *   when it is negligible) and the Pepe-Lanari goodness of fit
 *   (tcoh.cl:696-744).
 *
 * The matrices stay in shared memory, two rows per lane. Up to 32 dates
 * the faster register path of kernels_link_half.cu runs instead (same
 * stages, same numerics, two pixels per warp).
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

__device__ __forceinline__ double wmaxd(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v = fmax(v, __shfl_xor_sync(FULL, v, o));
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
/* Per-warp shared workspace of the 33-64-date EVD kernel (4-byte      */
/* units).                                                             */
/* ------------------------------------------------------------------ */

struct LinkLayout {
    int n;
    int per_warp; /* floats, a multiple of 4 (16-byte aligned workspaces) */
};

/* Packed lower triangle with the diagonal: entry (r, j), j <= r. */
__host__ __device__ __forceinline__ int low_idx(int r, int j) { return (r * (r + 1) >> 1) + j; }

struct Ws {
    float2 *A;   /* n (n + 1) / 2: T's lower triangle, then the reduction */
    /* vectors */
    void *d, *e, *y;   /* tridiagonal, eigenvector (R = float) */
    void *lu;          /* 4 n: LU of the shifted tridiagonal */
    void *tau;         /* n complex */
    void *vw;          /* 2 n complex: Householder v, w */
    float *df, *e2f;   /* copies for the Sturm counts */
    float *nrm;        /* sqrt(C_ii) */
    float2 *zs;        /* unit phasors */
};

__host__ __device__ __forceinline__ int up4(int x) { return (x + 3) & ~3; }

__device__ __forceinline__ Ws workspace(float *base, const LinkLayout &L)
{
    Ws w;
    const int n = L.n, an = up4(n);
    float *v = base + up4(2 * tc_npu(n));

    w.A = (float2 *)base;
    w.d = v;
    w.e = v + an;
    w.y = v + 2 * an;
    w.lu = v + 3 * an;       /* 4n */
    w.tau = v + 7 * an;      /* 2n */
    w.vw = v + 9 * an;       /* 4n */
    w.df = v + 13 * an;
    w.e2f = v + 14 * an;
    w.nrm = v + 15 * an;
    w.zs = (float2 *)(v + 16 * an); /* 2n */
    return w;
}

#define VEC_FLOATS(n) (18 * up4(n))

/* ------------------------------------------------------------------ */
/* Tridiagonal eigenvector.                                            */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

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

/* sturmd's count from the three-term recurrence of the leading principal
   minors, p_i = (d_i - x) p_{i-1} - e2_{i-1} p_{i-2}, whose ratios
   q_i = p_i / p_{i-1} are sturmd's pivots (a negative pivot is a sign
   change between consecutive minors): one FMA on the dependency chain per
   step, no division. The minors are rescaled by powers of two to stay in
   range; a pivot of magnitude below pivmin becomes -pivmin, as in sturmd. */
__device__ __forceinline__ int sturmd_minors(const double *d, const double *e2, int n, double x,
                                             double pivmin)
{
    double pm = 1.0, p = d[0] - x;

    if (fabs(p) < pivmin)
        p = -pivmin;
    int c = p < 0.0;

    for (int i = 1; i < n; i++) {
        double pn = fma(d[i] - x, p, -e2[i - 1] * pm);

        if (fabs(pn) < pivmin * fabs(p))
            pn = -pivmin * p;
        c += (pn < 0.0) != (p < 0.0);
        pm = p;
        p = pn;
        const double a = fabs(p);

        if (a > 0x1p400 || a < 0x1p-400) {
            const double sc = a > 1.0 ? 0x1p-400 : 0x1p400;

            p *= sc;
            pm *= sc;
        }
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

/* The eigenvector of rank `index` of the Hermitian matrix held as its packed
   lower triangle with the diagonal (low_idx): Householder reduction in
   place, the reflectors' vectors left in its columns. */
template <typename R>
__device__ unsigned heig_smem(int n, typename Cx<R>::T *A, int index, const Ws &ws,
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
                const C a = A[low_idx(r, k)];

                xn2 += a.x * a.x + a.y * a.y;
            }
        xn2 = wsum<R>(xn2);
        const C alpha = A[low_idx(k + 1, k)];
        const R dk = A[low_idx(k, k)].x;
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
                    const C a = A[low_idx(r, k)];

                    A[low_idx(r, k)] = mk<R>(a.x * sr - a.y * si, a.x * si + a.y * sr);
                }
        }
        if (lane == 0) {
            d[k] = dk;
            e[k] = beta;
            tau[k] = mk<R>(tr, ti);
            A[low_idx(k + 1, k)] = mk<R>(1, 0);
        }
        __syncwarp();
        if (tr == (R)0 && ti == (R)0)
            continue;
        for (int r = lane; r < n; r += 32)
            vv[r] = r > k ? A[low_idx(r, k)] : mk<R>(0, 0);
        __syncwarp();
        C wl[2];
        R pr = 0, pi = 0;
        {
            /* w = tau M v over rows r0 = lane, r1 = lane + 32 in one loop
               (the same trip count on every lane): M_rj is entry (r, j)
               of the packed triangle for j <= r, the conjugate of (j, r)
               beyond; cj = low_idx(j, 0). Separate accumulators for the
               two products of each part keep the FMA chains short. */
            const int r0 = lane, r1 = lane + 32;
            const bool a0 = r0 > k && r0 < n, a1 = r1 > k && r1 < n;
            const int ro0 = low_idx(r0, 0), ro1 = low_idx(a1 ? r1 : 0, 0);
            R p0 = 0, q0 = 0, u0 = 0, x0 = 0, p1 = 0, q1 = 0, u1 = 0, x1 = 0;

            for (int j = k + 1, cj = low_idx(k + 1, 0); j < n; cj += ++j) {
                const C v = vv[j];

                if (a0) {
                    const bool lo = j <= r0;
                    const C m = A[lo ? ro0 + j : cj + r0];
                    const R my = lo ? m.y : -m.y;

                    p0 = fma(m.x, v.x, p0);
                    q0 = fma(my, v.y, q0);
                    u0 = fma(m.x, v.y, u0);
                    x0 = fma(my, v.x, x0);
                }
                if (a1) {
                    const bool lo = j <= r1;
                    const C m = A[lo ? ro1 + j : cj + r1];
                    const R my = lo ? m.y : -m.y;

                    p1 = fma(m.x, v.x, p1);
                    q1 = fma(my, v.y, q1);
                    u1 = fma(m.x, v.y, u1);
                    x1 = fma(my, v.x, x1);
                }
            }
            const R sr0 = p0 - q0, si0 = u0 + x0, sr1 = p1 - q1, si1 = u1 + x1;

            wl[0] = a0 ? mk<R>(tr * sr0 - ti * si0, tr * si0 + ti * sr0) : mk<R>(0, 0);
            wl[1] = a1 ? mk<R>(tr * sr1 - ti * si1, tr * si1 + ti * sr1) : mk<R>(0, 0);
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const int r = lane + 32 * t;

                if (r > k && r < n) {
                    const C v = vv[r];

                    pr += wl[t].x * v.x + wl[t].y * v.y;
                    pi += wl[t].x * v.y - wl[t].y * v.x;
                }
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
                C *row = A + low_idx(r, 0);

                for (int j = k + 1; j <= r; j++) {
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
        d[n - 1] = A[low_idx(n - 1, n - 1)].x;
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
                const C v = A[low_idx(r, k)];

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
                const C v = A[low_idx(r, k)];

                z[t].x -= v.x * hr - v.y * hi2;
                z[t].y -= v.x * hi2 + v.y * hr;
            }
        }
    }
    zo[0] = z[0];
    zo[1] = z[1];
    return status;
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

/* T_ij (i < j) from its Gram sum g and the date norms (tcoh.cl:611-636),
   in IEEE float without contraction; near: the bias decision lies within
   TC_BIAS_BAND of its threshold. The load and the goodness of fit both
   take T from here, so that they see the same values. */
__device__ __forceinline__ float2 t_entry(float2 g, float nrm_i, float nrm_j, float fl,
                                          bool debias, bool &near)
{
    const float dd = __fmul_rn(nrm_i, nrm_j);
    float re = 0.f, im = 0.f;

    if (dd > 0.f) {
        re = __fdiv_rn(g.x, dd);
        im = __fdiv_rn(g.y, dd);
        if (debias) {
            const float m2 = __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im));
            const float lm1 = __fsub_rn(__fmul_rn(fl, m2), 1.0f);
            const float m2c = __fdiv_rn(lm1, __fsub_rn(fl, 1.0f));

            near |= fabsf(lm1) < TC_BIAS_BAND * fl * m2;
            const float f = (m2 > 0.f && m2c > 0.f) ? __fsqrt_rn(__fdiv_rn(m2c, m2)) : 0.f;

            re = __fmul_rn(re, f);
            im = __fmul_rn(im, f);
        }
    }
    return make_float2(re, im);
}

/* T from the packed Gram sums into w.A, as its packed lower triangle
   (T_ji = conj(T_ij)); w.nrm receives sqrt(C_ii). boundary: whether an
   entry's bias decision lies within TC_BIAS_BAND of its threshold. */
__device__ void load_coherence(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                               int p, int looks, const float2 *__restrict__ gram,
                               const unsigned short *__restrict__ upper_tab, const Ws &w,
                               int lane, bool &boundary)
{
    bool near = false;

    const int n = s.n, npu = tc_npu(n);

    for (int r = lane; r < n; r += 32)
        w.nrm[r] = __fsqrt_rn(gram[tc_gram_at(tc_npu(n), p, tc_pidx(n, r, r))].x);
    __syncwarp();
    const float fl = (float)looks;
    const bool debias = k.bias && looks > 1;

    for (int q = lane; q < npu; q += 32) {
        const int i = upper_tab[q] >> 8, j = upper_tab[q] & 255;

        if (i == j) {
            w.A[low_idx(i, i)] = make_float2(1.f, 0.f);
            continue;
        }
        const float2 t = t_entry(gram[tc_gram_at(tc_npu(n), p, q)], w.nrm[i], w.nrm[j], fl,
                                 debias, near);

        w.A[low_idx(j, i)] = make_float2(t.x, -t.y);
    }
    boundary = __any_sync(FULL, near);
    __syncwarp();
}

/* Whether the non-zero coherences link all dates (T as its packed lower
   triangle). */
__device__ bool linked(int n, const float2 *A, int lane)
{
    unsigned long long adj[2] = {0ull, 0ull};

#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int r = lane + 32 * t;

        if (r < n)
            for (int j = 0; j < n; j++) {
                const float2 v = A[j < r ? low_idx(r, j) : low_idx(j, r)];

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
__device__ float phasors_and_gamma(int n, const Ws &w, const typename Cx<R>::T (&z)[2],
                                   const unsigned short *__restrict__ upper_tab,
                                   const float2 *__restrict__ gram, int p, int looks,
                                   bool debias, int lane)
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
        /* T_ij again from its Gram sum: the reduction overwrote w.A */
        bool near = false;
        const float2 tv = t_entry(gram[tc_gram_at(npu, p, q)], w.nrm[i], w.nrm[j],
                                  (float)looks, debias, near);
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

__global__ void __launch_bounds__(384)
tc_link_smem_kernel(TcStrip s, TcChunk c, TcLinkConst k, LinkLayout L,
                    const float2 *__restrict__ gram, const int *__restrict__ count,
                    const unsigned short *__restrict__ upper_tab,
                    const unsigned short *__restrict__ pair_tab, double *__restrict__ scratch,
                    float *__restrict__ coh, float *__restrict__ pairs,
                    float *__restrict__ phases, unsigned char *__restrict__ status,
                    const uint32_t *__restrict__ mask, int *__restrict__ queue, int qstride)
{
    extern __shared__ float4 smf4[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int n = s.n;
    const Ws w = workspace((float *)smf4 + (size_t)warp * L.per_warp, L);
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
        bool boundary = false;

        load_coherence(s, c, k, p, looks, gram, upper_tab, w, lane, boundary);
        if (queue && boundary && lane == 0)
            tc_exact_push(queue, qstride, out, mask, c.npix, p);
        for (int q = lane; q < k.npairs; q += 32) {
            const int i = pair_tab[q] >> 8, j = pair_tab[q] & 255;
            const float2 t = w.A[low_idx(j, i)]; /* conj(T_ij), i < j */

            pairs[q * plane + out] = hypotf(t.x, t.y);
        }
        unsigned st = 0;

        if (k.bias && !linked(n, w.A, lane)) {
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
        /* EVD (the EMI path of this many dates is tc_link_exact_kernel),
           reduced in place on T's packed lower triangle */
        float2 z[2];

        st |= heig_smem<float>(n, w.A, n - 1, w, lane, z);
        const float gamma = phasors_and_gamma<float>(n, w, z, upper_tab, gram, p, looks,
                                                     k.bias && looks > 1, lane);

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

/* ------------------------------------------------------------------ */
/* The exact tier: a pixel from double-precision coherence sums.       */
/* ------------------------------------------------------------------ */

/* EMI divides by |T|, whose condition number reaches 1e5 - 1e6 on noisy or
   highly coherent stacks: the float rounding of the coherence sums and of
   their normalisation (a few 1e-7 relative) then moves gamma by up to 1e-3,
   however exactly the rest is computed. And the bias correction zeroes an
   entry at L m2 <= 1, a jump of gamma by up to 2 / (n (n - 1)) that float
   sums may place on the other side of the threshold. This tier recomputes
   a pixel from its samples with everything in double: the masked sums
   C = sum over SHPs q of s_q s_q^H (tcoh.cl:567-602, as tests/reference.py
   sums them), T and its bias correction (tcoh.cl:610-636); for EMI |T|^-1
   (ex_inverse: the symmetric sweep, Gauss-Jordan with partial pivoting,
   or the Jacobi pseudo-inverse with the absolute floor 1e-9 of
   tests/reference.py:151-156) and M = |T|^-1 o T, for EVD T itself; the
   Householder reduction to a real tridiagonal, the wanted eigenvalue by
   multisection on Sturm counts, inverse iteration and the
   back-transformation; then the phasors and gamma (tcoh.cl:696-744). It
   runs every pixel of the 33-64-date EMI path, and the pixels that the
   float kernels flag: ill-conditioned EMI pixels up to 32 dates, and with
   the bias correction any pixel with an entry at its threshold.

   One CTA of four warps per pixel, every matrix in packed upper-triangle
   storage (index tc_pidx) in shared memory, so that three pixels fit an
   SM at 60 dates: the sums and T (then M, in place) in complex double,
   |T| and its inverse in double (then a float copy of T for gamma in the
   same place). The sums accumulate in registers, each thread one to three
   2 x BC blocks of the triangle, over the SHP samples staged 16 candidates
   at a time, converted to double once at staging (a conversion costs four
   double FMAs' issue). */

constexpr int EX_THREADS = 128;
/* CTAs per SM: register blocks of the sums per thread NB = 1 (up to 32
   dates, 71 blocks of 2 x 4 entries at most) leave room for 6, NB = 3 (up
   to 64 dates) for 3 */
__host__ __device__ constexpr int ex_ctas(int nb) { return nb == 1 ? 6 : 3; }
constexpr int EX_KC = 16;         /* candidates per staging block */
/* the multisection's spacing: EX_THREADS points split an interval into
   EX_THREADS + 1 parts */
constexpr double EX_INV_POINTS = 1.0 / (EX_THREADS + 1);
constexpr int EX_NB = 3;          /* register blocks per thread, n <= 64 */
__host__ __device__ constexpr int ex_nb_for(int n) { return n <= 32 ? 1 : EX_NB; }
/* Columns per register block (2 rows x BC): 2 while the triangle's blocks
   fit one per thread (up to 30 dates), else 4. */
__host__ __device__ inline int ex_blocks(int n, int bc)
{
    const int rp = (n + 1) / 2, cg = (n + bc - 1) / bc;
    int nb = 0;

    for (int ip = 0; ip < rp; ip++)
        nb += cg - (2 * ip) / bc;
    return nb;
}
__host__ __device__ inline int ex_bc_for(int n) { return ex_blocks(n, 2) <= EX_THREADS ? 2 : 4; }
/* Row stride of the staged samples: n rounded up to 4, zero-padded. */
__host__ __device__ inline int ex_sld(int n) { return (n + 3) & ~3; }

struct ExLayout {
    int n, npu, nblk, ld;
    int off_T, off_G, off_tab, off_blk, off_stage, off_cand, off_vec, off_adj;
    int bytes;
};

struct ExWs {
    double2 *T;       /* [npu] sums, then T, then M */
    double *G;        /* [npu] |T|, then its inverse */
    float2 *Tf;       /* [npu] T in float, over G once M is formed */
    unsigned short *tab, *blk, *cand;
    double2 *stage;   /* [EX_KC][ex_sld(n)] */
    double *d, *e, *e2, *y, *lu, *rrow, *nrm, *red;
    double2 *v, *w, *tau, *z;
    float2 *zs;
    unsigned long long *adj;
    int *ints;        /* [0] candidates, [1] flags, [2..5] per warp, [6] next queue entry */
};

__host__ __device__ inline ExLayout ex_layout(int n, int area)
{
    ExLayout L;
    int off = 0;
    auto take = [&](int bytes) {
        const int o = off;

        off += (bytes + 15) & ~15;
        return o;
    };
    L.n = n;
    L.npu = tc_npu(n);
    L.ld = n | 1;
    L.nblk = ex_blocks(n, ex_bc_for(n));
    L.off_T = take(16 * L.npu);
    L.off_G = take(8 * L.npu);
    L.off_tab = take(2 * L.npu);
    L.off_blk = take(2 * L.nblk);
    /* the staged samples; once the sums are formed, up to 32 dates, the
       full |T| of the Gauss-Jordan inverse tier */
    L.off_stage = take(n <= 32 && 8 * n * n > 16 * EX_KC * ex_sld(n) ? 8 * n * n
                                                                      : 16 * EX_KC * ex_sld(n));
    L.off_cand = take(2 * area);
    L.off_vec = take(8 * (8 * 64 + 16 + 4 * 64) + 16 * 5 * 64 + 8 * 64 + 16);
    L.off_adj = take(8 * 64);
    L.bytes = off;
    return L;
}

__device__ __forceinline__ ExWs ex_ws(unsigned char *base, const ExLayout &L)
{
    ExWs w;
    double *v = (double *)(base + L.off_vec);

    w.T = (double2 *)(base + L.off_T);
    w.G = (double *)(base + L.off_G);
    w.Tf = (float2 *)(base + L.off_G);
    w.tab = (unsigned short *)(base + L.off_tab);
    w.blk = (unsigned short *)(base + L.off_blk);
    w.stage = (double2 *)(base + L.off_stage);
    w.cand = (unsigned short *)(base + L.off_cand);
    w.d = v;
    w.e = v + 64;
    w.e2 = v + 128;
    w.y = v + 192;
    w.rrow = v + 256;
    w.nrm = v + 320;
    w.red = v + 384;        /* 2 x 8 */
    w.lu = v + 400;         /* 4 x 64 */
    double2 *c = (double2 *)(v + 400 + 256);

    w.v = c;
    w.w = c + 64;
    w.tau = c + 128;
    w.z = c + 192;
    w.zs = (float2 *)(c + 320);
    w.ints = (int *)(w.zs + 64);
    w.adj = (unsigned long long *)(base + L.off_adj);
    return w;
}

/* 1 / x in double: a float reciprocal refined by two Newton steps
   r <- r (2 - x r), each doubling the correct bits (24 -> 48 -> 96, so
   within an ulp or two of 1 / x). For |x| in the float range: the LU
   pivots here, clamped to at least 1e-13 of the tridiagonal's norm, which
   is of order 1 or more (T has a unit diagonal, |T|^-1 o T one of 1 or
   more, a pseudo-inverse's at least about 1 / n^2). */
__device__ __forceinline__ double ex_rcp(double x)
{
    double r = (double)__frcp_rn((float)x);

    r = r * fma(-x, r, 2.0);
    return r * fma(-x, r, 2.0);
}

/* 1 / x for any x: ex_rcp inside [1e-30, 1e30] in magnitude, else the
   division. */
__device__ __forceinline__ double ex_rcp_any(double x)
{
    const double a = fabs(x);

    return a > 1.0e-30 && a < 1.0e30 ? ex_rcp(x) : 1.0 / x;
}

/* Block sums over the CTA (every thread gets them); red holds 8 doubles. */
__device__ __forceinline__ double2 ex_sum2(double a, double b, double *red)
{
    a = wsum<double>(a);
    b = wsum<double>(b);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = a;
        red[4 + (threadIdx.x >> 5)] = b;
    }
    __syncthreads();
    return make_double2(red[0] + red[1] + red[2] + red[3], red[4] + red[5] + red[6] + red[7]);
}

/* The same without the leading barrier, for callers that alternate
   between two halves of red (red + 8 * parity) with a barrier between two
   uses of one half. */
__device__ __forceinline__ double2 ex_sum2p(double a, double b, double *red)
{
    a = wsum<double>(a);
    b = wsum<double>(b);
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = a;
        red[4 + (threadIdx.x >> 5)] = b;
    }
    __syncthreads();
    return make_double2(red[0] + red[1] + red[2] + red[3], red[4] + red[5] + red[6] + red[7]);
}

/* Packed (i, j) of the upper triangle for any order of i, j. */
__device__ __forceinline__ int ex_sym(int n, int i, int j)
{
    return i <= j ? tc_pidx(n, i, j) : tc_pidx(n, j, i);
}

/* M_ij (Hermitian) from packed upper storage. */
__device__ __forceinline__ double2 ex_m(const double2 *P, int n, int i, int j)
{
    if (i <= j)
        return P[tc_pidx(n, i, j)];
    const double2 m = P[tc_pidx(n, j, i)];

    return make_double2(m.x, -m.y);
}

/* The pixel's SHP candidates (window indices) into w.cand; their number.
   Mask word i of the pixel is words[i * stride]. */
__device__ int ex_candidates(const TcStrip &s, const uint32_t *words, long long stride,
                             const ExWs &w)
{
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t bits = lane < s.mask_words ? words[lane * stride] : 0u;

        if (lane == s.mask_words - 1 && (s.area & 31))
            bits &= (1u << (s.area & 31)) - 1u; /* candidates only */
        const int cnt = __popc(bits);
        int off = cnt;

#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, off, o);

            if (lane >= o)
                off += v;
        }
        if (lane == 31)
            w.ints[0] = off;
        off -= cnt;
        while (bits) {
            const int b = __ffs(bits) - 1;

            bits &= bits - 1;
            w.cand[off++] = (unsigned short)(lane * 32 + b);
        }
    }
    __syncthreads();
    return w.ints[0];
}

/* C = sum of s_q s_q^H over the candidates, in double, into w.T (packed);
   NB register blocks per thread (L.nblk <= NB * EX_THREADS). */
template <int NB, int BC>
__device__ void ex_gram(const TcStrip &s, const float2 *slc, int py0, int px0, int ncand,
                        const ExWs &w, const ExLayout &L)
{
    const int n = s.n, t = threadIdx.x;
    const int sld = ex_sld(n);
    double2 acc[NB][2][BC];
    int bi[NB], bj[NB];

#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int id = t + b * EX_THREADS;

        bi[b] = bj[b] = -1;
        if (id < L.nblk) {
            bi[b] = 2 * (w.blk[id] >> 8);
            bj[b] = BC * (w.blk[id] & 255);
        }
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int q = 0; q < BC; q++)
                acc[b][r][q] = make_double2(0.0, 0.0);
    }
    for (int c0 = 0; c0 < ncand; c0 += EX_KC) {
        const int kc = min(EX_KC, ncand - c0);

        for (int q = t >> 5; q < kc; q += EX_THREADS / 32) {
            const int u = w.cand[c0 + q], dy = u / s.wr, dx = u - dy * s.wr;
            const float2 *src = slc + ((long long)(py0 + dy) * s.W + px0 + dx) * n;

            for (int d = t & 31; d < sld; d += 32) {
                float2 v = d < n ? src[d] : make_float2(0.f, 0.f);

                if (!isfinite(v.x) || !isfinite(v.y))
                    v = make_float2(0.f, 0.f);
                w.stage[q * sld + d] = make_double2(v.x, v.y);
            }
        }
        __syncthreads();
#pragma unroll
        for (int b = 0; b < NB; b++) {
            if (bi[b] < 0)
                continue;
            for (int q = 0; q < kc; q++) {
                const double2 *row = w.stage + q * sld;
                double2 a[2], cj[BC];

#pragma unroll
                for (int r = 0; r < 2; r++)
                    a[r] = row[bi[b] + r];
#pragma unroll
                for (int jj = 0; jj < BC; jj++)
                    cj[jj] = row[bj[b] + jj];
#pragma unroll
                for (int r = 0; r < 2; r++)
#pragma unroll
                    for (int jj = 0; jj < BC; jj++) {
                        /* a conj(b) */
                        acc[b][r][jj].x = fma(a[r].x, cj[jj].x, fma(a[r].y, cj[jj].y, acc[b][r][jj].x));
                        acc[b][r][jj].y = fma(a[r].y, cj[jj].x, fma(-a[r].x, cj[jj].y, acc[b][r][jj].y));
                    }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < NB; b++) {
        if (bi[b] < 0)
            continue;
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int jj = 0; jj < BC; jj++) {
                const int i = bi[b] + r, j = bj[b] + jj;

                if (i < n && j < n && i <= j)
                    w.T[tc_pidx(n, i, j)] = acc[b][r][jj];
            }
    }
    __syncthreads();
}

/* T from the sums (tcoh.cl:611-636 in double, as tests/reference.py:124-142)
   and |T|. */
__device__ void ex_coherence(int n, int npu, const TcLinkConst &k, int looks, const ExWs &w)
{
    const int t = threadIdx.x;

    for (int i = t; i < n; i += EX_THREADS)
        w.nrm[i] = sqrt(w.T[tc_pidx(n, i, i)].x);
    __syncthreads();
    const double fl = (double)looks, ifl1 = looks > 1 ? 1.0 / (fl - 1.0) : 0.0;

    for (int q = t; q < npu; q += EX_THREADS) {
        const int i = w.tab[q] >> 8, j = w.tab[q] & 255;
        double2 v = make_double2(1.0, 0.0);

        if (i != j) {
            const double dd = w.nrm[i] * w.nrm[j];
            const double2 cs = w.T[q];

            v = make_double2(0.0, 0.0);
            if (dd > 0.0) {
                const double rdd = ex_rcp_any(dd);

                v = make_double2(cs.x * rdd, cs.y * rdd);
                if (k.bias && looks > 1) {
                    const double m2 = v.x * v.x + v.y * v.y;
                    const double m2c = (fl * m2 - 1.0) * ifl1;
                    const double f = (m2 > 0.0 && m2c > 0.0) ? sqrt(m2c * ex_rcp_any(m2)) : 0.0;

                    v.x *= f;
                    v.y *= f;
                }
            }
        }
        w.T[q] = v;
        w.G[q] = hypot(v.x, v.y);
    }
    __syncthreads();
}

/* Whether the non-zero coherences link all dates (tcoh.cl:494-513). */
__device__ bool ex_linked(int n, const ExWs &w)
{
    const int t = threadIdx.x;

    for (int i = t; i < n; i += EX_THREADS) {
        unsigned long long a = 0ull;

        for (int j = 0; j < n; j++)
            if (j != i && w.G[ex_sym(n, i, j)] != 0.0)
                a |= 1ull << j;
        w.adj[i] = a;
    }
    __syncthreads();
    if (t < 32) {
        const unsigned long long all = n == 64 ? ~0ull : (1ull << n) - 1ull;
        unsigned long long reached = 1ull, frontier = 1ull;

        for (int it = 0; it < n; it++) {
            unsigned long long mine = 0ull;

            if ((frontier >> t) & 1ull)
                mine |= w.adj[t];
            if (t + 32 < n && ((frontier >> (t + 32)) & 1ull))
                mine |= w.adj[t + 32];
            const unsigned lo = __reduce_or_sync(FULL, (unsigned)mine);
            const unsigned hi = __reduce_or_sync(FULL, (unsigned)(mine >> 32));
            const unsigned long long nw = (((unsigned long long)hi << 32) | lo) & ~reached;

            if (!nw)
                break;
            reached |= nw;
            frontier = nw;
        }
        if (t == 0)
            w.ints[1] = reached == all;
    }
    __syncthreads();
    return w.ints[1] != 0;
}

/* A^-1 in place of the packed symmetric A by the symmetric sweep
   (Gauss-Jordan elimination without pivoting in the form that keeps the
   matrix symmetric; Goodnight, The American Statistician 33, 1979):
   sweeping pivot k maps a_ij -> a_ij - a_ik a_kj / a_kk,
   a_ik, a_kj -> a_ik / a_kk, a_kk -> -1 / a_kk, and all pivots leave
   -A^-1, negated back at the end. It takes indefinite matrices. False when
   a pivot's magnitude is not above floor_ (A is then undefined).
   Each step copies the next pivot row as it updates it (into one of two
   buffers), so that one barrier a pivot suffices; against a form that
   scaled the pivot row into its own buffer behind a second barrier, this
   one is the faster at every size (30-date AD/EMI/-b exact tier 83.7 ->
   82.0 ms per 4096 x 4096 step). */
__device__ bool ex_sweep(int n, int npu, const ExWs &w, double *A, double floor_)
{
    const int t = threadIdx.x;
    /* the pivot row as it stands before its step, in one of two buffers
       (w.lu, free until the eigenvector): the step that updates row kp + 1
       also copies it to the other buffer, so that one barrier a pivot
       suffices */
    double *raw[2] = {w.lu, w.lu + 64};

    for (int j = t; j < n; j += EX_THREADS)
        raw[0][j] = A[ex_sym(n, 0, j)];
    __syncthreads();
    for (int kp = 0; kp < n; kp++) {
        const double *rk = raw[kp & 1];
        double *rn = raw[(kp + 1) & 1];
        const double d = rk[kp];

        if (!(fabs(d) > floor_)) {
            __syncthreads();
            return false;
        }
        const double id = ex_rcp_any(d);

        for (int q = t; q < npu; q += EX_THREADS) {
            const int i = w.tab[q] >> 8, j = w.tab[q] & 255;
            const double ri = rk[i] * id, rj = rk[j] * id;
            double a;

            if (i == kp && j == kp)
                a = -id;
            else if (i == kp)
                a = rj;
            else if (j == kp)
                a = ri;
            else
                a = fma(-ri * d, rj, A[q]);
            A[q] = a;
            if (i == kp + 1)
                rn[j] = a;
            else if (j == kp + 1)
                rn[i] = a;
        }
        __syncthreads();
    }
    for (int q = t; q < npu; q += EX_THREADS)
        A[q] = -A[q];
    __syncthreads();
    return true;
}

/* Whether the packed inverse is finite and moderate: n max|inv_ij| < 1e8,
   which keeps every eigenvalue of |T| above the pseudo-inverse floor 1e-9
   of tests/reference.py:151-156, where the pseudo-inverse is the inverse. */
__device__ bool ex_moderate(int n, int npu, const ExWs &w, const double *A)
{
    const int t = threadIdx.x;
    double mx = 0.0;

    for (int q = t; q < npu; q += EX_THREADS) {
        const double v = A[q];

        mx = v == v ? fmax(mx, fabs(v)) : INFINITY;
    }
    mx = wmaxd(mx);
    __syncthreads();
    if ((t & 31) == 0)
        w.red[t >> 5] = mx;
    __syncthreads();
    mx = fmax(fmax(w.red[0], w.red[1]), fmax(w.red[2], w.red[3]));
    __syncthreads();
    return mx <= 1.0e300 && n * mx < 1.0e8;
}

/* A^-1 in place of the full n x n A (row-major) by Gauss-Jordan
   elimination with partial pivoting (the row of the largest magnitude in
   the pivot column; the column permutation is undone at the end). It takes
   indefinite and ill-conditioned matrices; false when a pivot falls below
   1e-14 of the largest entry (numerically singular). */
__device__ bool ex_gauss_jordan(int n, const ExWs &w, double *A)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int *perm = (int *)w.adj;
    double amax = 0.0;

    for (int e = t; e < n * n; e += EX_THREADS)
        amax = fmax(amax, fabs(A[e]));
    amax = wmaxd(amax);
    if (lane == 0)
        w.red[warp] = amax;
    __syncthreads();
    amax = fmax(fmax(w.red[0], w.red[1]), fmax(w.red[2], w.red[3]));
    __syncthreads();
    for (int k = 0; k < n; k++) {
        /* pivot row: the largest |A[i][k]|, i >= k */
        double v = t >= k && t < n ? fabs(A[t * n + k]) : -1.0;
        int idx = t;

#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double ov = __shfl_xor_sync(FULL, v, o);
            const int oi = __shfl_xor_sync(FULL, idx, o);

            if (ov > v || (ov == v && oi < idx)) {
                v = ov;
                idx = oi;
            }
        }
        if (lane == 0) {
            w.red[warp] = v;
            w.ints[2 + warp] = idx;
        }
        __syncthreads();
        int p = w.ints[2];
        double best = w.red[0];

        for (int q = 1; q < EX_THREADS / 32; q++)
            if (w.red[q] > best) {
                best = w.red[q];
                p = w.ints[2 + q];
            }
        __syncthreads();
        if (!(best > 1.0e-14 * amax))
            return false;
        if (t == 0)
            perm[k] = p;
        /* swap rows p and k, then scale row k (its pivot becomes 1 / piv) */
        const double piv = A[p * n + k];

        __syncthreads();
        for (int j = t; j < n; j += EX_THREADS) {
            const double rk = A[k * n + j], rp = A[p * n + j];

            A[p * n + j] = rk;
            A[k * n + j] = (j == k ? 1.0 : rp) / piv;
        }
        __syncthreads();
        for (int i = t; i < n; i += EX_THREADS)
            w.rrow[i] = i == k ? 0.0 : A[i * n + k];
        __syncthreads();
        for (int i = warp; i < n; i += EX_THREADS / 32)
            if (i != k)
                for (int j = lane; j < n; j += 32)
                    A[i * n + j] = (j == k ? 0.0 : A[i * n + j]) - A[k * n + j] * w.rrow[i];
        __syncthreads();
    }
    /* undo the row swaps on the columns of the inverse, last swap first */
    for (int k = n - 1; k >= 0; k--) {
        const int p = perm[k];

        if (p != k)
            for (int i = t; i < n; i += EX_THREADS) {
                const double x = A[i * n + k];

                A[i * n + k] = A[i * n + p];
                A[i * n + p] = x;
            }
        __syncthreads();
    }
    return true;
}

/* |T|^-1 into w.G (which holds |T|), in tiers: the symmetric sweep with
   pivots above 1e-5; else Gauss-Jordan elimination with partial pivoting
   on the full |T| (in shared memory, the staged samples' region, up to 32
   dates; in the CTA's global scratch W above); else, or when the inverse is
   not moderate, the Jacobi eigen-pseudo-inverse with the absolute floor
   1e-9 (tests/reference.py:151-156) on warp 0. Returns status bits. */
__device__ unsigned ex_inverse(int n, int npu, int ld, const ExWs &w, double *W)
{
    const int t = threadIdx.x;

    if (ex_sweep(n, npu, w, w.G, 1.0e-5) && ex_moderate(n, npu, w, w.G))
        return 0;
    double *A = n <= 32 ? (double *)w.stage : W;

    for (int i = t >> 5; i < n; i += EX_THREADS / 32)
        for (int j = t & 31; j < n; j += 32) {
            const double2 v = ex_m(w.T, n, i, j);

            A[i * n + j] = i == j ? 1.0 : hypot(v.x, v.y);
        }
    __syncthreads();
    if (ex_gauss_jordan(n, w, A)) {
        for (int q = t; q < npu; q += EX_THREADS) {
            const int i = w.tab[q] >> 8, j = w.tab[q] & 255;

            w.G[q] = 0.5 * (A[i * n + j] + A[j * n + i]);
        }
        __syncthreads();
        if (ex_moderate(n, npu, w, w.G))
            return TC_STATUS_EMI_PIVOTED;
    }
    __syncthreads();
    unsigned st = TC_STATUS_EMI_PINV;

    if (t < 32) {
        double *V = W + n * ld, *lam = W + 2 * n * ld;

        for (int r = t; r < n; r += 32)
            for (int j = 0; j < n; j++) {
                const double2 v = ex_m(w.T, n, r, j);

                W[r * ld + j] = r == j ? 1.0 : hypot(v.x, v.y);
            }
        __syncwarp();
        st |= jacobi_pinv(n, ld, W, V, lam, t);
        for (int r = t; r < n; r += 32)
            for (int j = r; j < n; j++)
                w.G[tc_pidx(n, r, j)] = W[r * ld + j];
    }
    if (t == 0)
        w.ints[1] = (int)st;
    __syncthreads();
    return (unsigned)w.ints[1];
}

/* Row i = k + 1 + t / R of M22 v (the trailing block at step k, v in w.v),
   R threads per row, thread h = t % R taking the columns j = h mod R: M_ij
   = conj(P(j, i)) for j < i, at rb(j) + i - j with rb(j) = j (2n - j + 1) /
   2, then P(i, j) for j >= i, contiguous. Separate accumulators for the two
   products of each part keep the FMA chains one deep; the R threads' sums
   are combined by shuffles (every thread gets its row's). */
template <int R>
__device__ __forceinline__ void ex_matvec_rows(int n, int k, const ExWs &w, int t, int &i, int &h,
                                               double &sx, double &sy)
{
    i = k + 1 + t / R;
    h = t % R;
    sx = sy = 0.0;
    if (i < n) {
        int j = k + 1 + h;
        int idx = j * (2 * n - j + 1) / 2 + (i - j);
        double ax = 0.0, bx = 0.0, ay = 0.0, by = 0.0;

        for (; j < i; j += R) {
            const double2 m = w.T[idx], v = w.v[j];

            ax = fma(m.x, v.x, ax);
            bx = fma(m.y, v.y, bx);
            ay = fma(m.x, v.y, ay);
            by = fma(m.y, v.x, by);
            idx += R * (n - j) - R * (R + 1) / 2;
        }
        sx = ax + bx;
        sy = ay - by;
        ax = bx = ay = by = 0.0;
        for (idx = i * (2 * n - i + 1) / 2 + (j - i); j < n; j += R, idx += R) {
            const double2 m = w.T[idx], v = w.v[j];

            ax = fma(m.x, v.x, ax);
            bx = fma(m.y, v.y, bx);
            ay = fma(m.x, v.y, ay);
            by = fma(m.y, v.x, by);
        }
        sx += ax - bx;
        sy += ay + by;
    }
#pragma unroll
    for (int o = 1; o < R; o <<= 1) {
        sx += __shfl_xor_sync(FULL, sx, o);
        sy += __shfl_xor_sync(FULL, sy, o);
    }
}

/* Householder reduction of the packed Hermitian M (w.T) to the real
   tridiagonal (w.d, w.e), zhetd2 form; reflector k's vector is left in
   packed row k (entries k + 2 ..; its entry k + 1 is 1) and its scalar in
   w.tau[k]. Two forms: up to 32 dates five CTA barriers a step
   (ex_householder_cta); above, three (ex_householder_lean: every warp
   reduces the pivot column itself, and w = p + h v is formed where the
   rank-2 update reads it), which pays where the steps are many. */
__device__ void ex_householder_cta(int n, int npu, const ExWs &w)
{
    const int t = threadIdx.x;

    for (int k = 0; k < n - 1; k++) {
        /* column k below the diagonal: x_r = conj(M_k,r) */
        double xn2 = 0.0;

        if (t < n - k - 2) {
            const double2 a = w.T[tc_pidx(n, k, k + 2 + t)];

            xn2 = a.x * a.x + a.y * a.y;
        }
        /* two barriers separate this half of red from its last use */
        xn2 = ex_sum2p(xn2, 0.0, w.red).x;
        const double2 am = w.T[tc_pidx(n, k, k + 1)];
        const double ax = am.x, ay = -am.y; /* alpha = x_k+1 */
        double beta, tr = 0.0, ti = 0.0, sr = 0.0, si = 0.0;

        if (xn2 == 0.0 && ay == 0.0)
            beta = ax;
        else {
            beta = -copysign(sqrt(ax * ax + ay * ay + xn2), ax);
            const double rb = ex_rcp_any(beta);

            tr = (beta - ax) * rb;
            ti = -ay * rb;
            const double dr = ax - beta, di = ay, rden = ex_rcp_any(dr * dr + di * di);

            sr = dr * rden;
            si = -di * rden;
        }
        const bool reflect = tr != 0.0 || ti != 0.0;

        if (t < n) {
            double2 v = make_double2(0.0, 0.0);

            if (t == k + 1)
                v = make_double2(1.0, 0.0);
            else if (t > k + 1 && reflect) {
                const double2 a = w.T[tc_pidx(n, k, t)];
                const double xr = a.x, xi = -a.y;

                v = make_double2(xr * sr - xi * si, xr * si + xi * sr);
                w.T[tc_pidx(n, k, t)] = v;
            }
            w.v[t] = v;
        }
        if (t == 0) {
            w.d[k] = w.T[tc_pidx(n, k, k)].x;
            w.e[k] = beta;
            w.tau[k] = make_double2(tr, ti);
        }
        __syncthreads();
        if (!reflect)
            continue;
        /* p = M22 v over rows k+1 .. n-1, four threads per row */
        double sx, sy;
        int i, h;

        ex_matvec_rows<4>(n, k, w, t, i, h, sx, sy);
        const double2 wl = make_double2(tr * sx - ti * sy, tr * sy + ti * sx);
        double pr = 0.0, pi = 0.0;

        if (i < n && h == 0) {
            const double2 v = w.v[i];

            pr = wl.x * v.x + wl.y * v.y;
            pi = wl.x * v.y - wl.y * v.x;
        }
        const double2 pp = ex_sum2p(pr, pi, w.red + 8);
        const double hr = -0.5 * (tr * pp.x - ti * pp.y), hi = -0.5 * (tr * pp.y + ti * pp.x);

        if (i < n && h == 0) {
            const double2 v = w.v[i];

            w.w[i] = make_double2(wl.x + hr * v.x - hi * v.y, wl.y + hr * v.y + hi * v.x);
        }
        __syncthreads();
        /* M22 -= v w^H + w v^H over the trailing triangle (contiguous) */
        for (int q = tc_pidx(n, k + 1, k + 1) + t; q < npu; q += EX_THREADS) {
            const int r = w.tab[q] >> 8, j = w.tab[q] & 255;
            const double2 vr = w.v[r], wr = w.w[r], vj = w.v[j], wj = w.w[j];
            double2 a = w.T[q];

            a.x -= vr.x * wj.x + vr.y * wj.y + wr.x * vj.x + wr.y * vj.y;
            a.y -= vr.y * wj.x - vr.x * wj.y + wr.y * vj.x - wr.x * vj.y;
            w.T[q] = a;
        }
        __syncthreads();
    }
    if (t == 0)
        w.d[n - 1] = w.T[tc_pidx(n, n - 1, n - 1)].x;
    __syncthreads();
}

__device__ void ex_householder_lean(int n, int npu, const ExWs &w)
{
    const int t = threadIdx.x;

    for (int k = 0; k < n - 1; k++) {
        /* column k below the diagonal: x_r = conj(M_k,r); every warp
           reduces it itself (no CTA barrier) */
        const int lane = t & 31;
        double xn2 = 0.0;

        for (int r = lane; r < n - k - 2; r += 32) {
            const double2 a = w.T[tc_pidx(n, k, k + 2 + r)];

            xn2 = fma(a.x, a.x, fma(a.y, a.y, xn2));
        }
        xn2 = wsum<double>(xn2);
        const double2 am = w.T[tc_pidx(n, k, k + 1)];
        const double ax = am.x, ay = -am.y; /* alpha = x_k+1 */
        double beta, tr = 0.0, ti = 0.0, sr = 0.0, si = 0.0;

        if (xn2 == 0.0 && ay == 0.0)
            beta = ax;
        else {
            beta = -copysign(sqrt(ax * ax + ay * ay + xn2), ax);
            const double rb = ex_rcp_any(beta);

            tr = (beta - ax) * rb;
            ti = -ay * rb;
            const double dr = ax - beta, di = ay, rden = ex_rcp_any(dr * dr + di * di);

            sr = dr * rden;
            si = -di * rden;
        }
        const bool reflect = tr != 0.0 || ti != 0.0;
        /* v, into w.v now and into column k of T (which keeps the
           reflectors) after the barrier: other warps may still be reading
           the column */
        double2 vk = make_double2(0.0, 0.0);

        if (t < n) {
            if (t == k + 1)
                vk = make_double2(1.0, 0.0);
            else if (t > k + 1 && reflect) {
                const double2 a = w.T[tc_pidx(n, k, t)];
                const double xr = a.x, xi = -a.y;

                vk = make_double2(xr * sr - xi * si, xr * si + xi * sr);
            }
            w.v[t] = vk;
        }
        if (t == 0) {
            w.d[k] = w.T[tc_pidx(n, k, k)].x;
            w.e[k] = beta;
            w.tau[k] = make_double2(tr, ti);
        }
        __syncthreads();
        if (!reflect)
            continue;
        if (t > k + 1 && t < n)
            w.T[tc_pidx(n, k, t)] = vk;
        /* p = M22 v over rows k+1 .. n-1, two threads per row */
        double sx, sy;
        int i, h;

        ex_matvec_rows<2>(n, k, w, t, i, h, sx, sy);
        const double2 wl = make_double2(tr * sx - ti * sy, tr * sy + ti * sx);
        double pr = 0.0, pi = 0.0;

        if (i < n && h == 0) {
            const double2 v = w.v[i];

            pr = wl.x * v.x + wl.y * v.y;
            pi = wl.x * v.y - wl.y * v.x;
            /* w = wl + h v, the correction h known after the barrier */
            w.w[i] = wl;
        }
        pr = wsum<double>(pr);
        pi = wsum<double>(pi);
        if (lane == 0) {
            w.red[t >> 5] = pr;
            w.red[4 + (t >> 5)] = pi;
        }
        __syncthreads();
        const double ppx = w.red[0] + w.red[1] + w.red[2] + w.red[3];
        const double ppy = w.red[4] + w.red[5] + w.red[6] + w.red[7];
        const double hr = -0.5 * (tr * ppx - ti * ppy), hi = -0.5 * (tr * ppy + ti * ppx);

        /* M22 -= v w^H + w v^H over the trailing triangle (contiguous) */
        for (int q = tc_pidx(n, k + 1, k + 1) + t; q < npu; q += EX_THREADS) {
            const int r = w.tab[q] >> 8, j = w.tab[q] & 255;
            const double2 vr = w.v[r], vj = w.v[j], lr = w.w[r], lj = w.w[j];
            const double2 wr = make_double2(lr.x + hr * vr.x - hi * vr.y, lr.y + hr * vr.y + hi * vr.x);
            const double2 wj = make_double2(lj.x + hr * vj.x - hi * vj.y, lj.y + hr * vj.y + hi * vj.x);
            double2 a = w.T[q];

            a.x -= vr.x * wj.x + vr.y * wj.y + wr.x * vj.x + wr.y * vj.y;
            a.y -= vr.y * wj.x - vr.x * wj.y + wr.y * vj.x - wr.x * vj.y;
            w.T[q] = a;
        }
        __syncthreads();
    }
    if (t == 0)
        w.d[n - 1] = w.T[tc_pidx(n, n - 1, n - 1)].x;
    __syncthreads();
}

/* LEAN (above 32 dates) or not, chosen at compile time so that each kernel
   holds only the code it runs: the chains here are latency-bound and
   sensitive to instruction-cache misses. */
template <bool LEAN>
__device__ void ex_householder(int n, int npu, const ExWs &w)
{
    if constexpr (LEAN)
        ex_householder_lean(n, npu, w);
    else
        ex_householder_cta(n, npu, w);
}

/* Eigenvalue of rank `index` of (w.d, w.e) (0: the smallest, for EMI;
   n - 1: the largest, for EVD) by 128-way multisection on double Sturm
   counts, then its eigenvector by inverse iteration (thread 0), then
   z = Q y by the reflectors (warp 0): into w.z. Returns status bits. */
__device__ unsigned ex_eigvec(int n, int index, const ExWs &w)
{
    const int t = threadIdx.x;
    unsigned status = 0;
    double lo = INFINITY, hi = -INFINITY;

    if (t < n) {
        const double rad = (t > 0 ? fabs(w.e[t - 1]) : 0.0) + (t < n - 1 ? fabs(w.e[t]) : 0.0);

        lo = w.d[t] - rad;
        hi = w.d[t] + rad;
        if (t < n - 1)
            w.e2[t] = w.e[t] * w.e[t];
    }
    {
        double a = lo, b = hi;

#pragma unroll
        for (int o = 16; o; o >>= 1) {
            a = fmin(a, __shfl_xor_sync(FULL, a, o));
            b = fmax(b, __shfl_xor_sync(FULL, b, o));
        }
        __syncthreads();
        if ((t & 31) == 0) {
            w.red[t >> 5] = a;
            w.red[4 + (t >> 5)] = b;
        }
        __syncthreads();
        lo = fmin(fmin(w.red[0], w.red[1]), fmin(w.red[2], w.red[3]));
        hi = fmax(fmax(w.red[4], w.red[5]), fmax(w.red[6], w.red[7]));
        __syncthreads();
    }
    const double norm = fmax(fabs(lo), fabs(hi));

    lo -= 1.0e-12 * norm + 1e-300;
    hi += 1.0e-12 * norm + 1e-300;
    /* float Sturm counts first (on float copies in the LU's region), down to
       a few float ulps of the spectrum's scale; then, the interval widened
       by the float counts' possible error, double counts */
    float *df = (float *)w.lu, *e2f = df + 64;

    for (int r = t; r < n; r += EX_THREADS) {
        df[r] = (float)w.d[r];
        if (r < n - 1)
            e2f[r] = (float)w.e2[r];
    }
    __syncthreads();
    for (int fr = 0; fr < 4 && hi - lo > 1.0e-6 * norm; fr++) {
        const double xq = lo + (hi - lo) * ((double)(t + 1) * EX_INV_POINTS);
        const bool gt = sturmf(df, e2f, n, (float)xq, 1.0e-30f + 1.0e-14f * (float)norm) > index;
        const unsigned bal = __ballot_sync(FULL, gt);

        if ((t & 31) == 0)
            w.ints[2 + (t >> 5)] = bal ? (t & ~31) + __ffs(bal) - 1 : EX_THREADS;
        __syncthreads();
        const int f = min(min(w.ints[2], w.ints[3]), min(w.ints[4], w.ints[5]));
        const double nlo = f == 0 ? lo : lo + (hi - lo) * ((double)f * EX_INV_POINTS);
        const double nhi =
            f == EX_THREADS ? hi : lo + (hi - lo) * ((double)(f + 1) * EX_INV_POINTS);

        __syncthreads();
        lo = nlo;
        hi = nhi;
    }
    lo -= 4.0e-7 * norm;
    hi += 4.0e-7 * norm;
    const double pivmin = 1e-290 + 1e-28 * norm;
    int round = 0;

    for (; round < 12; round++) {
        if (hi - lo <= 2.0e-15 * norm)
            break;
        const double xq = lo + (hi - lo) * ((double)(t + 1) * EX_INV_POINTS);
        const bool gt = sturmd_minors(w.d, w.e2, n, xq, pivmin) > index;
        const unsigned bal = __ballot_sync(FULL, gt);

        if ((t & 31) == 0)
            w.ints[2 + (t >> 5)] = bal ? (t & ~31) + __ffs(bal) - 1 : EX_THREADS;
        __syncthreads();
        const int f = min(min(w.ints[2], w.ints[3]), min(w.ints[4], w.ints[5]));
        double nlo, nhi;

        if (f == EX_THREADS) {
            nlo = lo + (hi - lo) * ((double)EX_THREADS * EX_INV_POINTS);
            nhi = hi;
        }
        else {
            nhi = lo + (hi - lo) * ((double)(f + 1) * EX_INV_POINTS);
            nlo = f == 0 ? lo : lo + (hi - lo) * ((double)f * EX_INV_POINTS);
        }
        __syncthreads();
        if (!(nlo > lo || nhi < hi))
            break;
        lo = fmax(nlo, lo);
        hi = fmin(nhi, hi);
    }
    if (round == 12)
        status |= TC_STATUS_ITER_CAP;
    const double lambda = 0.5 * (lo + hi);

    /* Inverse iteration: LU of T - lambda I with partial pivoting, three
       solves from a vector of ones (the method of tcoh.cl:342-410). The
       recurrences carry their running values in registers; the shared
       arrays only hold what a later pass reads. */
    if (t == 0) {
        const double tiny = 1.0e-13 * (norm > 1e-300 ? norm : 1e-300);
        double *__restrict__ lu = w.lu;
        double *__restrict__ y = w.y;
        const double *__restrict__ dg = w.d;
        const double *__restrict__ eg = w.e;
        unsigned long long piv = 0ull;
        double dd = dg[0] - lambda, s1 = n > 1 ? eg[0] : 0.0;

        for (int kk = 0; kk < n - 1; kk++) {
            const double sub = eg[kk], nd = dg[kk + 1] - lambda;
            const double ns = kk + 1 < n - 1 ? eg[kk + 1] : 0.0;

            if (fabs(dd) >= fabs(sub)) {
                if (fabs(dd) < tiny)
                    dd = dd < 0.0 ? -tiny : tiny;
                const double rd = ex_rcp(dd), l = sub * rd;

                lu[4 * kk] = rd;
                lu[4 * kk + 1] = s1;
                lu[4 * kk + 2] = 0.0;
                lu[4 * kk + 3] = l;
                dd = nd - l * s1;
                s1 = ns;
            }
            else {
                const double rs = ex_rcp(sub), l = dd * rs;

                piv |= 1ull << kk;
                lu[4 * kk] = rs;
                lu[4 * kk + 1] = nd;
                lu[4 * kk + 2] = ns;
                lu[4 * kk + 3] = l;
                dd = s1 - l * nd;
                s1 = -l * ns;
            }
        }
        if (fabs(dd) < tiny)
            dd = dd < 0.0 ? -tiny : tiny;
        lu[4 * (n - 1)] = ex_rcp(dd);
        lu[4 * (n - 1) + 1] = 0.0;
        lu[4 * (n - 1) + 2] = 0.0;
        for (int kk = 0; kk < n; kk++)
            y[kk] = 1.0;
        for (int it = 0; it < 3; it++) {
            /* forward: the row interchanges and L, y[kk] final once the
               step leaves it */
            double cur = y[0];

            for (int kk = 0; kk < n - 1; kk++) {
                double a = cur, b = y[kk + 1];

                if ((piv >> kk) & 1ull) {
                    const double tmp = a;

                    a = b;
                    b = tmp;
                }
                y[kk] = a;
                cur = b - lu[4 * kk + 3] * a;
            }
            y[n - 1] = cur;
            /* backward: U, the next two solution entries in registers */
            double y1 = 0.0, y2 = 0.0, nrm = 0.0;

            for (int kk = n - 1; kk >= 0; kk--) {
                const double v = (y[kk] - lu[4 * kk + 1] * y1 - lu[4 * kk + 2] * y2) * lu[4 * kk];

                y[kk] = v;
                y2 = y1;
                y1 = v;
                nrm = fmax(nrm, fabs(v));
            }
            const double inv = 1.0 / nrm; /* may exceed the float range */

            for (int kk = 0; kk < n; kk++)
                y[kk] *= inv;
        }
    }
    __syncthreads();
    /* z = H_0 ... H_n-2 y (warp 0, rows lane and lane + 32), two
       reflectors at a time in application order (H_n-2 first): with
       a = v_0^H z, b = v_1^H z and g = v_1^H v_0 reduced over the warp at
       once, h_0 = tau_0 a, h_1 = tau_1 (b - g h_0), z -= v_0 h_0 + v_1 h_1,
       which is the one-by-one application rearranged. */
    if (t < 32) {
        double2 z[2];

#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = t + 32 * q;

            z[q] = make_double2(r < n ? w.y[r] : 0.0, 0.0);
        }
        for (int b0 = n - 2; b0 >= 0; b0 -= 2) {
            double2 vq[2][2], ta[2];

#pragma unroll
            for (int m = 0; m < 2; m++) {
                const int kk = b0 - m;

                ta[m] = kk >= 0 ? w.tau[kk] : make_double2(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int r = t + 32 * q;

                    vq[m][q] = make_double2(0.0, 0.0);
                    if (kk >= 0 && r == kk + 1)
                        vq[m][q] = make_double2(1.0, 0.0);
                    else if (kk >= 0 && r > kk + 1 && r < n)
                        vq[m][q] = w.T[tc_pidx(n, kk, r)];
                }
            }
            double rd[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

#pragma unroll
            for (int q = 0; q < 2; q++) {
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    rd[2 * m] += vq[m][q].x * z[q].x + vq[m][q].y * z[q].y;
                    rd[2 * m + 1] += vq[m][q].x * z[q].y - vq[m][q].y * z[q].x;
                }
                rd[4] += vq[1][q].x * vq[0][q].x + vq[1][q].y * vq[0][q].y;
                rd[5] += vq[1][q].x * vq[0][q].y - vq[1][q].y * vq[0][q].x;
            }
#pragma unroll
            for (int e = 0; e < 6; e++)
                rd[e] = wsum<double>(rd[e]);
            double2 h[2];

            h[0] = make_double2(ta[0].x * rd[0] - ta[0].y * rd[1], ta[0].x * rd[1] + ta[0].y * rd[0]);
            {
                const double sx = rd[2] - (rd[4] * h[0].x - rd[5] * h[0].y);
                const double sy = rd[3] - (rd[4] * h[0].y + rd[5] * h[0].x);

                h[1] = make_double2(ta[1].x * sx - ta[1].y * sy, ta[1].x * sy + ta[1].y * sx);
            }
#pragma unroll
            for (int m = 0; m < 2; m++)
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    z[q].x -= vq[m][q].x * h[m].x - vq[m][q].y * h[m].y;
                    z[q].y -= vq[m][q].x * h[m].y + vq[m][q].y * h[m].x;
                }
        }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = t + 32 * q;

            if (r < n)
                w.z[r] = z[q];
        }
    }
    __syncthreads();
    return status;
}

/* Unit phasors relative to the median date (tcoh.cl:700-724) into w.zs
   (warp 0), then gamma over the pairs (tcoh.cl:728-744), every thread. */
__device__ float ex_gamma(int n, int npu, const ExWs &w)
{
    const int t = threadIdx.x;

    if (t < 32) {
        double m[2];

#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = t + 32 * q;

            m[q] = r < n ? hypot(w.z[r].x, w.z[r].y) : 0.0;
        }
        double mx = fmax(m[0], m[1]);

        mx = wmaxd(mx);
        int ref = n / 2;

        if (hypot(w.z[ref].x, w.z[ref].y) <= 1.0e-3 * mx) {
            int last = -1;

#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int r = t + 32 * q;

                if (r < n && m[q] == mx)
                    last = max(last, r);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1)
                last = max(last, __shfl_xor_sync(FULL, last, o));
            ref = last;
        }
        const double2 zr = w.z[ref];
        const double refm = hypot(zr.x, zr.y);
        const double refr = zr.x / refm, refi = -zr.y / refm, floor_ = 1.0e-3 * mx;

#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = t + 32 * q;

            if (r < n) {
                const double2 z = w.z[r];
                const double re = z.x * refr - z.y * refi, im = z.x * refi + z.y * refr;
                const double mm = hypot(re, im);

                w.zs[r] = mm > floor_ ? make_float2((float)(re / mm), (float)(im / mm))
                                      : make_float2(1.f, 0.f);
            }
        }
    }
    __syncthreads();
    float sr = 0.f, si = 0.f;

    for (int q = t; q < npu; q += EX_THREADS) {
        const int i = w.tab[q] >> 8, j = w.tab[q] & 255;

        if (i == j)
            continue;
        const float2 tv = w.Tf[q];
        const float m2 = tv.x * tv.x + tv.y * tv.y;
        float ur = 1.f, ui = 0.f;

        if (m2 > 0.f) {
            const float r = rsqrtf(m2);

            ur = tv.x * r;
            ui = tv.y * r;
        }
        const float2 zi = w.zs[i], zj = w.zs[j];
        const float wr = zi.x * zj.x + zi.y * zj.y, wi = zi.x * zj.y - zi.y * zj.x;

        sr += ur * wr - ui * wi;
        si += ur * wi + ui * wr;
    }
    const double2 ssum = ex_sum2(sr, si, w.red);

    return (float)(hypot(ssum.x, ssum.y) / (0.5 * n * (n - 1)));
}

/* queue: null for every pixel of the chunk c (with its mask), else the
   queue's entries (TcExactQueue, any pixels of the strip; c unused). */
template <int NB, int BC>
__global__ void __launch_bounds__(EX_THREADS, ex_ctas(NB))
tc_link_exact_kernel(TcStrip s, TcChunk c, TcLinkConst k, ExLayout L,
                     const float2 *__restrict__ slc, const uint32_t *__restrict__ mask,
                     const int *__restrict__ count, int *queue, int qstride,
                     const unsigned short *__restrict__ upper_tab,
                     const unsigned short *__restrict__ pair_tab, double *__restrict__ scratch,
                     float *__restrict__ coh, float *__restrict__ pairs,
                     float *__restrict__ phases, unsigned char *__restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const ExWs w = ex_ws(smem, L);
    const int n = s.n, npu = L.npu, t = threadIdx.x, ld = L.ld;
    const long long plane = (long long)s.rows * s.cols;
    double *W = scratch + (size_t)blockIdx.x * (2 * n * ld + 64);

    for (int q = t; q < npu; q += EX_THREADS)
        w.tab[q] = upper_tab[q];
    if (t == 0) {
        const int rp = (n + 1) / 2, cg = (n + BC - 1) / BC;
        int b = 0;

        for (int ip = 0; ip < rp; ip++)
            for (int jg = (2 * ip) / BC; jg < cg; jg++)
                w.blk[b++] = (unsigned short)(ip << 8 | jg);
    }
    __syncthreads();
    const int total = queue ? queue[0] : c.npix;
    /* A chunk's pixels go to the CTAs in turn. Queued pixels vary more in
       cost (pivoted inverses, unlinked dates, several chunks' worth of
       flagged pixels of every kind): after its first, each CTA takes the
       next untaken entry from the queue's counter buf[1]. The barriers
       order thread 0's write of the index after every thread's read of the
       previous one. */
    auto next_item = [&](int it) -> int {
        if (!queue)
            return it + gridDim.x;
        __syncthreads();
        if (t == 0)
            w.ints[6] = gridDim.x + atomicAdd(queue + 1, 1);
        __syncthreads();
        return w.ints[6];
    };

    for (int it = blockIdx.x; it < total; it = next_item(it)) {
        const int *entry = queue ? queue + TC_QUEUE_HEAD + (long long)it * qstride : nullptr;
        int y, x;

        if (entry) {
            y = entry[0] / s.cols;
            x = entry[0] - y * s.cols;
        }
        else {
            tc_pixel_yx(c, it, y, x);
            if (y >= c.row0 + c.nrows || y >= s.rows || x >= s.cols)
                continue;
        }
        const long long out = (long long)y * s.cols + x;
        const int looks = count[out];

        if (looks < k.min_looks) {
            if (t == 0)
                coh[out] = NAN;
            for (int q = t; q < k.npairs; q += EX_THREADS)
                pairs[q * plane + out] = NAN;
            if (phases)
                for (int r = t; r < n; r += EX_THREADS)
                    phases[out * n + r] = NAN;
            if (status && t == 0)
                status[out] = 0;
            continue;
        }
        const int ncand =
            entry ? ex_candidates(s, (const uint32_t *)entry + 1, 1, w)
                  : ex_candidates(s, mask + it, c.npix, w);

        ex_gram<NB, BC>(s, slc, y, x, ncand, w, L);
        ex_coherence(n, npu, k, looks, w);
        for (int q = t; q < k.npairs; q += EX_THREADS) {
            const int i = pair_tab[q] >> 8, j = pair_tab[q] & 255;

            pairs[q * plane + out] = (float)w.G[tc_pidx(n, i, j)];
        }
        if (k.bias && !ex_linked(n, w)) {
            if (t == 0)
                coh[out] = NAN;
            if (phases)
                for (int r = t; r < n; r += EX_THREADS)
                    phases[out * n + r] = NAN;
            if (status && t == 0)
                status[out] = TC_STATUS_UNLINKED;
            __syncthreads();
            continue;
        }
        unsigned st = TC_STATUS_FP64;

        if (k.emi) {
            st |= ex_inverse(n, npu, ld, w, W);
            /* M = |T|^-1 o T in place of T; T in float in place of |T|^-1 */
            for (int q = t; q < npu; q += EX_THREADS) {
                const double g = w.G[q];
                const double2 v = w.T[q];

                w.T[q] = make_double2(g * v.x, g * v.y);
                w.Tf[q] = make_float2((float)v.x, (float)v.y);
            }
        }
        else
            /* EVD: T itself; T in float in place of |T| */
            for (int q = t; q < npu; q += EX_THREADS) {
                const double2 v = w.T[q];

                w.Tf[q] = make_float2((float)v.x, (float)v.y);
            }
        __syncthreads();
        ex_householder<(NB > 1)>(n, npu, w);
        st |= ex_eigvec(n, k.emi ? 0 : n - 1, w);
        const float gamma = ex_gamma(n, npu, w);

        if (t == 0)
            coh[out] = gamma;
        if (phases)
            for (int r = t; r < n; r += EX_THREADS) {
                const float2 u = w.zs[r];

                phases[out * n + r] = atan2f(u.y, u.x);
            }
        if (status && t == 0)
            status[out] = (unsigned char)st;
        __syncthreads();
    }
}

LinkLayout layout_for(int n)
{
    LinkLayout L;

    L.n = n;
    /* T's packed lower triangle, then the vectors */
    L.per_warp = up4(2 * tc_npu(n)) + VEC_FLOATS(n);
    return L;
}

} // namespace

static size_t exact_scratch_bytes(int n, int sms)
{
    /* per CTA: |T| and the Jacobi eigenvectors in full storage, and the
       eigenvalues, for the pseudo-inverse tier */
    return (size_t)sms * ex_ctas(ex_nb_for(n)) * (2 * n * (n | 1) + 64) * sizeof(double);
}

template <int NB, int BC>
static cudaError_t launch_exact_nb(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                   const float *slc, const uint32_t *mask, const int *count,
                                   const TcExactQueue *q, const unsigned short *upper_tab,
                                   const unsigned short *pair_tab, double *scratch, float *coh,
                                   float *pairs, float *phases, unsigned char *status, int sms,
                                   cudaStream_t st)
{
    const ExLayout L = ex_layout(s.n, s.area);
    const int ctas = sms * ex_ctas(NB);
    int blocks = ctas;

    if (!q && c.npix < ctas)
        blocks = c.npix;
    if (q && q->pending < ctas)
        blocks = (int)q->pending;
    cudaError_t e = cudaFuncSetAttribute(tc_link_exact_kernel<NB, BC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, L.bytes);

    if (e != cudaSuccess)
        return e;
    tc_link_exact_kernel<NB, BC><<<blocks, EX_THREADS, L.bytes, st>>>(
        s, c, k, L, (const float2 *)slc, mask, count, q ? q->buf : nullptr, q ? q->stride : 0,
        upper_tab, pair_tab, scratch, coh, pairs, phases, status);
    return cudaGetLastError();
}

static cudaError_t launch_exact(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                                const float *slc, const uint32_t *mask, const int *count,
                                const TcExactQueue *q, const unsigned short *upper_tab,
                                const unsigned short *pair_tab, double *scratch, float *coh,
                                float *pairs, float *phases, unsigned char *status, int sms,
                                cudaStream_t st)
{
    if (ex_nb_for(s.n) == 1 && ex_bc_for(s.n) == 2)
        return launch_exact_nb<1, 2>(s, c, k, slc, mask, count, q, upper_tab, pair_tab, scratch,
                                     coh, pairs, phases, status, sms, st);
    if (ex_nb_for(s.n) == 1)
        return launch_exact_nb<1, 4>(s, c, k, slc, mask, count, q, upper_tab, pair_tab, scratch,
                                     coh, pairs, phases, status, sms, st);
    return launch_exact_nb<EX_NB, 4>(s, c, k, slc, mask, count, q, upper_tab, pair_tab, scratch,
                                     coh, pairs, phases, status, sms, st);
}

bool tc_link_needs_gram(int n, int emi)
{
    return n <= 32 || !emi;
}

size_t tc_link_scratch_bytes(int n, int sms)
{
    /* the 32-date kernel and the exact tier run one after the other */
    const size_t a = tc_link_half_scratch_bytes(n, sms), b = exact_scratch_bytes(n, sms);

    return a > b ? a : b;
}

bool tc_link_queues(int n, const TcLinkConst &k)
{
    /* the float kernels hand pixels to the exact tier with EMI and with
       the bias correction; EMI above 32 dates is all exact */
    return (k.emi || k.bias) && !(n > 32 && k.emi);
}

size_t tc_exact_queue_bytes(int mask_words, long long capacity)
{
    return sizeof(int) * (TC_QUEUE_HEAD + (size_t)capacity * (1 + mask_words));
}

cudaError_t tc_flush_exact(const TcStrip &s, const TcLinkConst &k, TcExactQueue *q,
                           const float *slc, const int *count, const unsigned short *upper_tab,
                           const unsigned short *pair_tab, double *scratch, float *coh,
                           float *pairs, float *phases, unsigned char *status, int sms,
                           cudaStream_t st)
{
    cudaError_t e = cudaSuccess;

    if (q->pending > 0) {
        TcChunk none = {};

        if ((e = launch_exact(s, none, k, slc, nullptr, count, q, upper_tab, pair_tab, scratch,
                              coh, pairs, phases, status, sms, st)) == cudaSuccess)
            e = cudaMemsetAsync(q->buf, 0, sizeof(int) * TC_QUEUE_HEAD, st);
    }
    q->pending = 0;
    return e;
}

cudaError_t tc_launch_link(const TcStrip &s, const TcChunk &c, const TcLinkConst &k,
                           const float2 *gram, const float *slc, const uint32_t *mask,
                           const int *count, TcExactQueue *q,
                           const unsigned short *upper_tab, const unsigned short *pair_tab,
                           double *scratch, float *coh, float *pairs, float *phases,
                           unsigned char *status, int sms, cudaStream_t st)
{
    cudaError_t e;
    const bool queued = tc_link_queues(s.n, k);

    if (queued && (!q || !q->buf || q->stride != 1 + s.mask_words ||
                   q->pending + c.npix > q->capacity))
        return cudaErrorInvalidValue;
    int *qb = queued ? q->buf : nullptr;
    const int qs = queued ? q->stride : 0;

    if (s.n > 32 && k.emi)
        return launch_exact(s, c, k, slc, mask, count, nullptr, upper_tab, pair_tab, scratch, coh,
                            pairs, phases, status, sms, st);
    if (s.n <= 32)
        e = tc_launch_link_half(s, c, k, gram, mask, count, upper_tab, pair_tab, scratch, coh,
                                pairs, phases, status, qb, qs, sms, st);
    else {
        const LinkLayout L = layout_for(s.n);
        const size_t per_warp = (size_t)L.per_warp * sizeof(float);
        int wpb = (int)((227 * 1024) / per_warp);

        if (wpb > 12)
            wpb = 12;
        if (wpb < 1)
            return cudaErrorInvalidConfiguration;
        const size_t smem = per_warp * wpb;
        const int want = (c.npix + wpb - 1) / wpb;
        const int blocks = want < sms ? want : sms;

        e = cudaFuncSetAttribute(tc_link_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            tc_link_smem_kernel<<<blocks, wpb * 32, smem, st>>>(
                s, c, k, L, gram, count, upper_tab, pair_tab, scratch, coh, pairs, phases, status,
                mask, qb, qs);
        if (e == cudaSuccess)
            e = cudaGetLastError();
    }
    if (e == cudaSuccess && queued)
        q->pending += c.npix;
    return e;
}
