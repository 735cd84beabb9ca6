// neat_image.cu -- ComputeImage over an explicit SampleList
// (HierarchicalNeuralGeometry::ComputeImage, src/geometry/geometry.cpp:347-389,
// with GeometryExEx::SampleVolumeIndirect, src/geometry/geometry_ex_ex.cpp:161-180,
// and IntegrateSamplesXRay, src/geometry/geometry.cpp:393-424).
//
// Same tile engine as the fused step, fed from caller-owned sample arrays in
// the reference's layouts (grid [rows, C, G,G,G], int64 indices).  The image
// accumulation is index_add_ semantics (float atomics, as the reference).
#include "neat_internal.h"
#include "neat_tiles.cuh"

namespace neat
{

struct ImageTileArgs
{
    const float* grid;
    int64_t rows;
    int G;
    const float* decoder;
    float beta;
    const float* coords;
    const float* weight;
    const int64_t* ray_index;
    const int64_t* node_id;
    const int64_t* local_node_id;
    const float* node_min;
    const float* node_max;
    int64_t S;
    float* image;
    const float* grad_image;
    float* grad_grid;
    float* grad_decoder;
};

template <int C, bool BWD>
__global__ void __launch_bounds__(TN, 1) k_image_tiles(ImageTileArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    TileSmem<C, BWD>& sm = *reinterpret_cast<TileSmem<C, BWD>*>(smraw);
    const int t          = threadIdx.x;
    tile_load_decoder<C, BWD>(sm, a.decoder);
    DecGradAcc<C> g;
    g.zero();
    const int64_t ntiles = (a.S + TT - 1) / TT;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        bool valid = false;
        float wgt = 0.0f, lu = 0.0f, lv = 0.0f, lw = 0.0f;
        int64_t ray = 0, row = 0;
        if (t < TT)
        {
            const int64_t s = tile * TT + t;
            if (s < a.S)
            {
                row   = a.local_node_id[s];
                valid = row >= 0 && row < a.rows;
            }
            float x[C];
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = 0.0f;
            if (valid)
            {
                const int64_t nd = a.node_id[s];
                const float* mn  = a.node_min + 3 * nd;
                const float* mx  = a.node_max + 3 * nd;
                lu               = local_coord(a.coords[3 * s + 0], mn[0], mx[0]);
                lv               = local_coord(a.coords[3 * s + 1], mn[1], mx[1]);
                lw               = local_coord(a.coords[3 * s + 2], mn[2], mx[2]);
                Corners k;
                igs_corners(lu, lv, lw, a.G, a.G, a.G, k);
                gather_cf<C>(a.grid, row, a.G, k, x);
                wgt = a.weight[s];
                ray = a.ray_index[s];
            }
#pragma unroll
            for (int c = 0; c < C; ++c) sm.XT[c * TT + t] = x[c];
        }
        __syncthreads();
        tile_layer1<C, BWD>(sm);
        __syncthreads();
        float z2[4][HPW];
        tile_gemm_fwd<C, BWD>(sm, z2);
        tile_ypart<C, BWD>(sm, z2);
        __syncthreads();
        if (t < TT)
        {
            const float y = tile_y(sm, t);
            if (!BWD)
            {
                if (valid) atomicAdd(a.image + ray, softplusf_(y, a.beta) * wgt);
            }
            else
            {
                const float dv = valid ? a.grad_image[ray] : 0.0f;
                const float dy = dv * wgt * softplus_grad(y, a.beta);
                sm.val[t]      = dy;
                g.db3 += dy;
            }
        }
        __syncthreads();
        if constexpr (BWD)
        {
            float dx[C];
            tile_backward<C>(sm, z2, g, dx);
            if (t < TT && valid)
            {
                Corners k;
                igs_corners(lu, lv, lw, a.G, a.G, a.G, k);
                scatter_cf<C>(a.grad_grid, row, a.G, k, dx);
            }
            __syncthreads();
        }
    }
    if constexpr (BWD) dec_grad_flush<C>(g, a.grad_decoder, true, sm.ypart);
}

template <int C, bool BWD>
static cudaError_t launch_image(const ImageTileArgs& a, cudaStream_t st)
{
    const size_t smem = sizeof(TileSmem<C, BWD>);
    static int grid   = 0;
    if (grid == 0)
    {
        cudaFuncSetAttribute(k_image_tiles<C, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        grid = resident_ctas((const void*)k_image_tiles<C, BWD>, TN, smem, 0) * sm_count();
    }
    const int64_t ntiles = (a.S + TT - 1) / TT;
    const int g          = (int)std::min<int64_t>(grid, std::max<int64_t>(ntiles, 1));
    k_image_tiles<C, BWD><<<g, TN, smem, st>>>(a);
    return cudaGetLastError();
}

static cudaError_t launch_image_any(int C, bool bwd, const ImageTileArgs& a, cudaStream_t st)
{
    switch (C)
    {
        case 4: return bwd ? launch_image<4, true>(a, st) : launch_image<4, false>(a, st);
        case 8: return bwd ? launch_image<8, true>(a, st) : launch_image<8, false>(a, st);
        case 16: return bwd ? launch_image<16, true>(a, st) : launch_image<16, false>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace neat

using namespace neat;

static int image_common(const float* grid, int64_t num_rows, int C, int G, const float* decoder,
                        const float* coords, const float* weight, const int64_t* ray_index, const int64_t* node_id,
                        const int64_t* local_node_id, const float* node_min, const float* node_max,
                        int64_t num_samples)
{
    if (C != 4 && C != 8 && C != 16) return NEAT_ERR_UNSUPPORTED;
    if (num_rows < 0 || G < 2 || num_samples < 0) return NEAT_ERR_BAD_INPUT;
    if (num_samples > 0 && (!grid || !decoder || !coords || !weight || !ray_index || !node_id || !local_node_id ||
                            !node_min || !node_max))
        return NEAT_ERR_BAD_INPUT;
    return NEAT_OK;
}

extern "C" int neat_compute_image_forward(const float* grid, int64_t num_rows, int C, int G, const float* decoder,
                                          float softplus_beta, const float* coords, const float* weight,
                                          const int64_t* ray_index, const int64_t* node_id,
                                          const int64_t* local_node_id, const float* node_min, const float* node_max,
                                          int64_t num_samples, float* image, neat_stream_t stream)
{
    int e = image_common(grid, num_rows, C, G, decoder, coords, weight, ray_index, node_id, local_node_id, node_min,
                         node_max, num_samples);
    if (e != NEAT_OK) return e;
    if (num_samples == 0) return NEAT_OK;
    if (!image) return NEAT_ERR_BAD_INPUT;
    ImageTileArgs a{grid,     num_rows, G,        decoder, softplus_beta, coords,  weight,  ray_index, node_id,
                    local_node_id, node_min, node_max, num_samples, image,   nullptr, nullptr, nullptr};
    return launch_image_any(C, false, a, (cudaStream_t)stream) == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_compute_image_backward(const float* grid, int64_t num_rows, int C, int G, const float* decoder,
                                           float softplus_beta, const float* coords, const float* weight,
                                           const int64_t* ray_index, const int64_t* node_id,
                                           const int64_t* local_node_id, const float* node_min,
                                           const float* node_max, int64_t num_samples, const float* grad_image,
                                           float* grad_grid, float* grad_decoder, neat_stream_t stream)
{
    int e = image_common(grid, num_rows, C, G, decoder, coords, weight, ray_index, node_id, local_node_id, node_min,
                         node_max, num_samples);
    if (e != NEAT_OK) return e;
    if (num_samples == 0) return NEAT_OK;
    if (!grad_image || !grad_grid || !grad_decoder) return NEAT_ERR_BAD_INPUT;
    ImageTileArgs a{grid,     num_rows, G,          decoder,   softplus_beta, coords, weight, ray_index,
                    node_id,  local_node_id, node_min, node_max, num_samples, nullptr, grad_image, grad_grid,
                    grad_decoder};
    return launch_image_any(C, true, a, (cudaStream_t)stream) == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
