// neat_igs.cu -- IndirectGridSample3D forward/backward in the reference's
// layout (src/modules/IndirectGridSample3D.cu:432-801): grid [N, C, Z, Y, X],
// one row per sample selected by index[s], trilinear with align_corners and
// index-clamped border.  Forward accumulates the eight corner terms per
// channel in the reference order as fused multiply-adds; backward adds
// w_corner * grad_out into grad_grid with float atomics (the unsorted-sample
// API offers no node ownership; the fused step sorts by node instead) and
// computes grad_uv per sample without atomics.
#include "neat_common.cuh"

namespace neat
{

__global__ void __launch_bounds__(128)
    k_igs_forward(const float* __restrict__ grid, int64_t N, int C, int Z, int Y, int X,
                  const int64_t* __restrict__ index, const float* __restrict__ uv, int64_t S, float* __restrict__ out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int64_t n = index[s];
    if (n < 0 || n >= N)
    {
        for (int c = 0; c < C; ++c) out[s * C + c] = 0.0f;
        return;
    }
    Corners k;
    igs_corners(uv[3 * s], uv[3 * s + 1], uv[3 * s + 2], Z, Y, X, k);
    int cell[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) cell[q] = corner_cell(k, q, Y, X);
    const int64_t G3 = (int64_t)Z * Y * X;
    const float* g   = grid + n * C * G3;  // channel c of row n: g + c G3
    float* o         = out + s * C;
    // two channels' 16 corner loads in flight per thread; plain (L1-cached)
    // loads: neighbouring samples of a ray reuse the corner lines
#pragma unroll 2
    for (int c = 0; c < C; ++c, g += G3)
    {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = g[cell[q]];
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) acc = fmaf(v[q], k.w[q], acc);
        o[c] = acc;
    }
}

__global__ void __launch_bounds__(128)
    k_igs_backward(const float* __restrict__ grid, int64_t N, int C, int Z, int Y, int X,
                   const int64_t* __restrict__ index, const float* __restrict__ uv, int64_t S,
                   const float* __restrict__ grad_out, float* __restrict__ grad_grid, float* __restrict__ grad_uv)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int64_t n = index[s];
    if (n < 0 || n >= N) return;
    Corners k;
    igs_corners(uv[3 * s], uv[3 * s + 1], uv[3 * s + 2], Z, Y, X, k);
    int cell[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) cell[q] = corner_cell(k, q, Y, X);
    const int64_t G3 = (int64_t)Z * Y * X;
    const float ix = k.ix, iy = k.iy, iz = k.iz;
    const float x0 = (float)k.x0, y0 = (float)k.y0, z0 = (float)k.z0;
    const float x1 = x0 + 1.0f, y1 = y0 + 1.0f, z1 = z0 + 1.0f;
    const float ax0 = __fsub_rn(x1, ix), ax1 = __fsub_rn(ix, x0);
    const float ay0 = __fsub_rn(y1, iy), ay1 = __fsub_rn(iy, y0);
    const float az0 = __fsub_rn(z1, iz), az1 = __fsub_rn(iz, z0);
    float gix = 0.0f, giy = 0.0f, giz = 0.0f;
    const float m1 = -1.0f;
    const float* g = grid + n * C * G3;  // channel c of row n: g + c G3
    float* gg      = grad_grid + n * C * G3;
    const float* gout = grad_out + s * C;
#pragma unroll 1
    for (int c = 0; c < C; ++c, g += G3, gg += G3)
    {
        const float go = gout[c];
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            atomicAdd(gg + cell[q], __fmul_rn(k.w[q], go));
            v[q] = __ldg(g + cell[q]);
        }
        if (grad_uv)
        {
            // IndirectGridSample3D.cu:738-770, every term one fma into the sum
            gix = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[0]), ay0), az0), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(v[1], ay0), az0), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[2]), ay1), az0), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(v[3], ay1), az0), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[4]), ay0), az1), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(v[5], ay0), az1), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[6]), ay1), az1), go, gix);
            gix = fmaf(__fmul_rn(__fmul_rn(v[7], ay1), az1), go, gix);

            giy = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[0]), ax0), az0), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[1]), ax1), az0), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(v[2], ax0), az0), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(v[3], ax1), az0), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[4]), ax0), az1), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[5]), ax1), az1), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(v[6], ax0), az1), go, giy);
            giy = fmaf(__fmul_rn(__fmul_rn(v[7], ax1), az1), go, giy);

            giz = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[0]), ax0), ay0), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[1]), ax1), ay0), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[2]), ax0), ay1), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(__fmul_rn(m1, v[3]), ax1), ay1), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(v[4], ax0), ay0), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(v[5], ax1), ay0), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(v[6], ax0), ay1), go, giz);
            giz = fmaf(__fmul_rn(__fmul_rn(v[7], ax1), ay1), go, giz);
        }
    }
    if (grad_uv)
    {
        grad_uv[3 * s + 0] += __fdiv_rn(__fmul_rn(gix, (float)(X - 1)), 2.0f);
        grad_uv[3 * s + 1] += __fdiv_rn(__fmul_rn(giy, (float)(Y - 1)), 2.0f);
        grad_uv[3 * s + 2] += __fdiv_rn(__fmul_rn(giz, (float)(Z - 1)), 2.0f);
    }
}

}  // namespace neat

using namespace neat;

static bool igs_args_ok(const float* grid, int64_t N, int C, int Z, int Y, int X, const int64_t* index,
                        const float* uv, int64_t S)
{
    if (N < 0 || C < 1 || Z < 1 || Y < 1 || X < 1 || S < 0) return false;
    if (S > 0 && (!grid || !index || !uv)) return false;
    return true;
}

extern "C" int neat_igs_forward(const float* grid, int64_t N, int C, int Z, int Y, int X, const int64_t* index,
                                const float* uv, int64_t num_samples, float* out, neat_stream_t stream)
{
    if (!igs_args_ok(grid, N, C, Z, Y, X, index, uv, num_samples)) return NEAT_ERR_BAD_INPUT;
    if (num_samples == 0) return NEAT_OK;
    if (!out) return NEAT_ERR_BAD_INPUT;
    k_igs_forward<<<(unsigned)((num_samples + 127) / 128), 128, 0, (cudaStream_t)stream>>>(grid, N, C, Z, Y, X, index,
                                                                                          uv, num_samples, out);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_igs_backward(const float* grid, int64_t N, int C, int Z, int Y, int X, const int64_t* index,
                                 const float* uv, int64_t num_samples, const float* grad_out, float* grad_grid,
                                 float* grad_uv, neat_stream_t stream)
{
    if (!igs_args_ok(grid, N, C, Z, Y, X, index, uv, num_samples)) return NEAT_ERR_BAD_INPUT;
    if (num_samples == 0) return NEAT_OK;
    if (!grad_out || !grad_grid) return NEAT_ERR_BAD_INPUT;
    k_igs_backward<<<(unsigned)((num_samples + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        grid, N, C, Z, Y, X, index, uv, num_samples, grad_out, grad_grid, grad_uv);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
