/* Masked coherence-matrix accumulation in plain FP32 on the CUDA cores:
 *
 *   C_p = sum over SHPs q of p:  s_q s_q^H        (tcoh.cl:567-602)
 *
 * One thread per output pixel (a CTA is one 16 x 8 tile); each thread walks
 * its window once per B x B block (I, J), J >= I, of the N x N
 * matrix and accumulates the block in registers, reading the candidates'
 * samples from the date-major planes so that the 32 lanes of a warp (8
 * consecutive columns of 4 rows) load contiguous 64-byte runs. Output is the
 * packed upper triangle, pixel-major: gram[p][tc_pidx(i, j)] (float2: re, im).
 */
#include "tcoh_internal.h"

template <int B>
__global__ void __launch_bounds__(TC_TILE_PIX)
tc_gram_fp32_kernel(TcStrip s, TcChunk c, const float2 *__restrict__ soa,
                    const uint32_t *__restrict__ mask, float2 *__restrict__ gram)
{
    const int p = blockIdx.x * TC_TILE_PIX + threadIdx.x;
    int y, x;

    tc_pixel_yx(c, p, y, x);
    if (y >= c.row0 + c.nrows || y >= s.rows || x >= s.cols)
        return;
    const int n = s.n, nb = (n + B - 1) / B;
    const long long base = (long long)y * s.W + x;

    for (int I = 0; I < nb; I++) {
        for (int J = I; J < nb; J++) {
            float2 acc[B][B];

#pragma unroll
            for (int a = 0; a < B; a++)
#pragma unroll
                for (int b = 0; b < B; b++)
                    acc[a][b] = make_float2(0.f, 0.f);
            int dy = 0, dx = 0;

            for (int w = 0; w < s.mask_words; w++) {
                uint32_t bits = mask[(long long)w * c.npix + p];
                const int nbits = min(32, s.area - 32 * w);

                for (int b = 0; b < nbits; b++) {
                    if (bits & 1u) {
                        const long long q = base + (long long)dy * s.W + dx;
                        float2 si[B], sj[B];

#pragma unroll
                        for (int a = 0; a < B; a++) {
                            si[a] = __ldg(soa + (long long)(I * B + a) * s.npad + q);
                            sj[a] = __ldg(soa + (long long)(J * B + a) * s.npad + q);
                        }
#pragma unroll
                        for (int a = 0; a < B; a++)
#pragma unroll
                            for (int b2 = 0; b2 < B; b2++) {
                                /* s_i conj(s_j), four FMAs */
                                acc[a][b2].x = fmaf(si[a].x, sj[b2].x, acc[a][b2].x);
                                acc[a][b2].x = fmaf(si[a].y, sj[b2].y, acc[a][b2].x);
                                acc[a][b2].y = fmaf(si[a].y, sj[b2].x, acc[a][b2].y);
                                acc[a][b2].y = fmaf(-si[a].x, sj[b2].y, acc[a][b2].y);
                            }
                    }
                    bits >>= 1;
                    if (++dx == s.wr) {
                        dx = 0;
                        dy++;
                    }
                }
            }
#pragma unroll
            for (int a = 0; a < B; a++)
#pragma unroll
                for (int b2 = 0; b2 < B; b2++) {
                    const int i = I * B + a, j = J * B + b2;

                    if (i < n && j < n && i <= j)
                        gram[tc_gram_at(tc_npu(n), p, tc_pidx(n, i, j))] =
                            i == j ? make_float2(acc[a][b2].x, 0.f) : acc[a][b2];
                }
        }
    }
}

cudaError_t tc_launch_gram_fp32(const TcStrip &s, const TcChunk &c, int block,
                                const float2 *soa, const uint32_t *mask, float2 *gram,
                                cudaStream_t st)
{
    const int blocks = c.npix / TC_TILE_PIX;

    switch (block) {
    case 4:
        tc_gram_fp32_kernel<4><<<blocks, TC_TILE_PIX, 0, st>>>(s, c, soa, mask, gram);
        break;
    case 5:
        tc_gram_fp32_kernel<5><<<blocks, TC_TILE_PIX, 0, st>>>(s, c, soa, mask, gram);
        break;
    case 6:
        tc_gram_fp32_kernel<6><<<blocks, TC_TILE_PIX, 0, st>>>(s, c, soa, mask, gram);
        break;
    default:
        tc_gram_fp32_kernel<8><<<blocks, TC_TILE_PIX, 0, st>>>(s, c, soa, mask, gram);
        break;
    }
    return cudaGetLastError();
}

/* Block size of the FP32 Gram for N dates: the largest of 8, 6, 5, 4 that
   pads N least. */
int tc_gram_block_for(int n)
{
    static const int cand[4] = {8, 6, 5, 4};
    int best = 4, best_pad = 1 << 30;

    for (int i = 0; i < 4; i++) {
        const int b = cand[i], pad = (n + b - 1) / b * b - n;

        if (pad < best_pad) {
            best_pad = pad;
            best = b;
        }
    }
    return best;
}
