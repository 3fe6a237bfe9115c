/* Adjoint of the temporal coherence: from the per-pixel gradients of gamma
 * with respect to the coherence sums back to every sample's phase, and to
 * the height error and the phase screen.
 *
 * With the samples a_q = s_q exp(i theta_q) and the Hermitian gradient G_p
 * of pixel p (d gamma_p = Re sum_ij conj(G_p,ij) dC_p,ij, written by the
 * link kernel's backward stage), the gradient of L = sum_p gamma_p with
 * respect to theta_q,k is
 *
 *     dL/dtheta_q,k = 2 Im(conj(a_q,k) b_q,k),  b_q = (sum over the pixels p
 *                     that took q as an SHP of G_p) a_q
 *
 * the transpose of the masked Gram (tcoh.cl:567-602). One CTA per tile of
 * 128 output pixels, as the Gram kernels: the rows of the tile's G are
 * staged in shared memory one matrix row at a time, every thread takes a
 * candidate of the union of the tile's windows and sums the G of the tile
 * pixels that selected it, then adds 2 Im(conj(a) b) into the candidate's
 * dL/dtheta (atomically: a candidate lies in the windows of several tiles).
 *
 * dL/dpsi_q,k = dL/dtheta_q,k; dL/ddh_q = sum_k dL/dtheta_q,k dphi_k/dh at the
 * cell's height (the derivative of the quadratic in height of the grid's
 * coefficient form, TcGridCell; zero with a single height level).
 */
#include "tcoh_internal.h"

namespace {

constexpr int THREADS = 256;
constexpr int GS_LD = 33; /* float2 per pixel row of the staged G row */

__global__ void __launch_bounds__(THREADS)
tc_adjoint_scatter_kernel(TcStrip s, TcChunk c, int halo, const float2 *__restrict__ gbar,
                          const uint32_t *__restrict__ mask, const float2 *__restrict__ slc,
                          float *__restrict__ dtheta)
{
    extern __shared__ __align__(16) unsigned char sm[];
    float2 *gs = (float2 *)sm;                                  /* 128 x GS_LD */
    uint32_t *s_rows = (uint32_t *)(sm + TC_TILE_PIX * GS_LD * 8); /* wa x 128 */
    const int t = threadIdx.x, n = s.n, tile = blockIdx.x;
    const int ty = tile / c.tiles_x, tx = tile - ty * c.tiles_x;
    const int y0 = c.row0 + ty * TC_TILE_H, x0 = tx * TC_TILE_W;
    const int UW = TC_TILE_W + s.wr - 1, K = (TC_TILE_H + s.wa - 1) * UW;
    const uint32_t wr_mask = s.wr >= 32 ? 0xffffffffu : (1u << s.wr) - 1u;
    const int cols = s.cols;
    const size_t plane = (size_t)s.padded_rows * cols;

    for (int e = t; e < s.wa * TC_TILE_PIX; e += THREADS) {
        const int dy = e >> 7, m = e & 127;
        const int y = y0 + (m >> 3), x = x0 + (m & 7);
        uint32_t f = 0u;

        if (y < c.row0 + c.nrows && y < s.rows && x < s.cols) {
            const int b = dy * s.wr, w = b >> 5, o = b & 31;
            const long long p = (long long)tile * TC_TILE_PIX + m;
            const uint32_t lo = mask[(long long)w * c.npix + p];
            const uint32_t hi = o + s.wr > 32 ? mask[(long long)(w + 1) * c.npix + p] : 0u;

            f = (uint32_t)(((unsigned long long)hi << 32 | lo) >> o) & wr_mask;
        }
        s_rows[e] = f;
    }
    for (int base = 0; base < K; base += THREADS) {
        const int u = base + t;
        const int uy = u / UW, ux = u - uy * UW;
        const int py = y0 + uy, px = x0 + ux, col = px - halo;
        const bool cand = u < K && py < s.padded_rows && px < s.W && col >= 0 && col < cols;
        uint32_t bits[4] = {0u, 0u, 0u, 0u};
        float2 a[32], b[32];

        __syncthreads();
        if (cand)
            for (int m = 0; m < TC_TILE_PIX; m++) {
                const int dy = uy - (m >> 3), dx = ux - (m & 7);

                if (dy >= 0 && dy < s.wa && dx >= 0 && dx < s.wr &&
                    ((s_rows[dy * TC_TILE_PIX + m] >> dx) & 1u))
                    bits[m >> 5] |= 1u << (m & 31);
            }
        const bool any = (bits[0] | bits[1] | bits[2] | bits[3]) != 0u;
#pragma unroll
        for (int j = 0; j < 32; j++) {
            a[j] = cand && any && j < n ? slc[((size_t)py * s.W + px) * n + j]
                                        : make_float2(0.f, 0.f);
            b[j] = make_float2(0.f, 0.f);
        }
        for (int i = 0; i < n - 1; i++) {
            __syncthreads();
            for (int e = t; e < TC_TILE_PIX * n; e += THREADS) {
                const int m = e / n, j = e - m * n;

                if (j > i)
                    gs[m * GS_LD + j] =
                        gbar[(long long)tc_pidx(n, i, j) * c.npix + (long long)tile * TC_TILE_PIX + m];
            }
            __syncthreads();
            if (!any)
                continue;
            float2 h[32];

#pragma unroll
            for (int j = 0; j < 32; j++)
                h[j] = make_float2(0.f, 0.f);
#pragma unroll
            for (int w = 0; w < 4; w++) {
                uint32_t bw = bits[w];

                while (bw) {
                    const int m = w * 32 + __ffs(bw) - 1;
                    const float2 *row = gs + m * GS_LD;

                    bw &= bw - 1u;
#pragma unroll
                    for (int j = 0; j < 32; j++)
                        if (j > i && j < n) {
                            h[j].x += row[j].x;
                            h[j].y += row[j].y;
                        }
                }
            }
            /* G_ij a_j into b_i, conj(G_ij) a_i into b_j */
            float2 ai = make_float2(0.f, 0.f), bi = make_float2(0.f, 0.f);

#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j == i)
                    ai = a[j];
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j > i && j < n) {
                    bi.x += h[j].x * a[j].x - h[j].y * a[j].y;
                    bi.y += h[j].x * a[j].y + h[j].y * a[j].x;
                    b[j].x += h[j].x * ai.x + h[j].y * ai.y;
                    b[j].y += h[j].x * ai.y - h[j].y * ai.x;
                }
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j == i) {
                    b[j].x += bi.x;
                    b[j].y += bi.y;
                }
        }
        if (cand && any)
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k < n)
                    atomicAdd(dtheta + k * plane + (size_t)py * cols + col,
                              2.f * (a[k].x * b[k].y - a[k].y * b[k].x));
    }
}

/* dL/ddh from dL/dtheta (grad_psi) and the height derivative of the phase
   grid (coefficient form). */
__global__ void tc_adjoint_height_kernel(int n, int padded_rows, int cols, int row0,
                                         int region_rows, const double *__restrict__ elev,
                                         const double *__restrict__ dh, TcGeo g,
                                         const double *__restrict__ grid,
                                         const float *__restrict__ dtheta, float *__restrict__ gdh)
{
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;

    if (cell >= (long long)padded_rows * cols)
        return;
    const int r = (int)(cell / cols), col = (int)(cell - (long long)r * cols);
    const int row = row0 + r;
    float out = 0.f;

    if (grid && g.nheights == 3 && row >= 0 && row < region_rows) {
        const double h = (elev ? elev[cell] : g.h0) + (dh ? dh[cell] : 0.0);
        const TcGridCell gc = tc_grid_cell(g, grid, row, col, h);
        const size_t plane = (size_t)padded_rows * cols;
        double acc = 0.0;

        for (int k = 0; k < n; k++) {
            double d;

            gc.phase(k, &d);
            acc += d * dtheta[k * plane + cell];
        }
        out = (float)acc;
    }
    gdh[cell] = out;
}

} // namespace

cudaError_t tc_launch_adjoint_scatter(const TcStrip &s, const TcChunk &c, int halo,
                                      const float2 *gbar, const uint32_t *mask,
                                      const float *slc, float *dtheta, cudaStream_t st)
{
    const int bytes = TC_TILE_PIX * GS_LD * 8 + s.wa * TC_TILE_PIX * 4;
    cudaError_t e = cudaFuncSetAttribute(tc_adjoint_scatter_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);

    if (e != cudaSuccess)
        return e;
    tc_adjoint_scatter_kernel<<<c.npix / TC_TILE_PIX, THREADS, bytes, st>>>(
        s, c, halo, gbar, mask, (const float2 *)slc, dtheta);
    return cudaGetLastError();
}

cudaError_t tc_launch_adjoint_height(int n, int padded_rows, int cols, int row0, int region_rows,
                                     const double *elev, const double *dh, const TcGeo *g,
                                     const double *grid, const float *dtheta, float *gdh,
                                     cudaStream_t st)
{
    const long long cells = (long long)padded_rows * cols;
    const TcGeo none = {};

    tc_adjoint_height_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(
        n, padded_rows, cols, row0, region_rows, elev, dh, g ? *g : none, g ? grid : nullptr,
        dtheta, gdh);
    return cudaGetLastError();
}
