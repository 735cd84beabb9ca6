// neat_volume.cu -- uniformly sampled volume of the trained density field
// (HierarchicalNeuralGeometry::UniformSampledVolume, src/geometry/geometry.cpp:166-248).
//
// Voxel v = x + nx (y + ny z) sits at the voxel-corner position
//   p_d = (c_d / (n_d - 1)) * 2 - 1          (VolumeSamples, src/structure/HyperTree.cu:546-580)
// and is evaluated in the active node found by the top-down descent of
// ActiveNodeIdForGlobalPosition (HyperTree.cu:598-637): stop at an active
// node; otherwise step into the first child (child order 0..7) whose closed
// box contains p; a leaf that is not active, or no containing child, gives
// "outside" (value 0, node 0, valid 0, as UniformSampledVolume leaves those
// entries of its zero-initialised outputs untouched).
//
// The field value is the decoder of the fused step (IGS -> FCBlock ->
// softplus) on 128-voxel tiles, SIMT FP32 (this is an export, not the hot path).
#include "neat_internal.h"
#include "neat_tiles.cuh"

namespace neat
{

struct VolumeArgs
{
    const NodeEntry* table;
    int max_depth;
    const float* node_min;
    const float* node_max;
    const float* grid;
    int channel_last;
    int G;
    const float* decoder;
    float beta;
    int nx, ny, nz;
    int64_t V;
    float* out;
    int64_t* out_node;
    float* out_valid;
};

__device__ __forceinline__ bool box_contains(const float* mn, const float* mx, float x, float y, float z)
{
    return !(mn[0] > x || mx[0] < x || mn[1] > y || mx[1] < y || mn[2] > z || mx[2] < z);
}

// Active node of a position, or -1.
__device__ __forceinline__ int64_t active_node_for(const VolumeArgs& a, float x, float y, float z)
{
    const int64_t first_leaf = tree_nodes(a.max_depth - 1);
    int64_t n                = 0;
    for (int level = 0; level <= a.max_depth; ++level)
    {
        if (a.table[n].active) return n;
        if (n >= first_leaf) return -1;
        int64_t next = -1;
        for (int cid = 0; cid < 8; ++cid)
        {
            const int64_t c = 8 * n + 1 + cid;
            if (box_contains(a.node_min + 3 * c, a.node_max + 3 * c, x, y, z))
            {
                next = c;
                break;
            }
        }
        if (next < 0) return -1;
        n = next;
    }
    return -1;
}

template <int C>
__global__ void __launch_bounds__(TN, 1) k_volume_tiles(VolumeArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    TileSmem<C, false>& sm = *reinterpret_cast<TileSmem<C, false>*>(smraw);
    const int t            = threadIdx.x;
    tile_load_decoder<C, false>(sm, a.decoder);
    const int64_t ntiles = (a.V + TT - 1) / TT;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        bool valid   = false;
        int64_t node = -1, v = tile * TT + t;
        if (t < TT)
        {
            float x[C];
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = 0.0f;
            if (v < a.V)
            {
                const int cx  = (int)(v % a.nx);
                const int cy  = (int)((v / a.nx) % a.ny);
                const int cz  = (int)(v / ((int64_t)a.nx * a.ny));
                const float px = __fsub_rn(__fmul_rn(__fdiv_rn((float)cx, (float)(a.nx - 1)), 2.0f), 1.0f);
                const float py = __fsub_rn(__fmul_rn(__fdiv_rn((float)cy, (float)(a.ny - 1)), 2.0f), 1.0f);
                const float pz = __fsub_rn(__fmul_rn(__fdiv_rn((float)cz, (float)(a.nz - 1)), 2.0f), 1.0f);
                node           = active_node_for(a, px, py, pz);
                valid          = node >= 0;
                if (valid)
                {
                    const float* mn = a.node_min + 3 * node;
                    const float* mx = a.node_max + 3 * node;
                    Corners k;
                    igs_corners(local_coord(px, mn[0], mx[0]), local_coord(py, mn[1], mx[1]),
                                local_coord(pz, mn[2], mx[2]), a.G, a.G, a.G, k);
                    const int64_t row = a.table[node].local;
                    if (a.channel_last)
                        gather_cl<C>(a.grid, row, a.G, k, x);
                    else
                        gather_cf<C>(a.grid, row, a.G, k, x);
                }
            }
#pragma unroll
            for (int c = 0; c < C; ++c) sm.XT[c * TT + t] = x[c];
        }
        __syncthreads();
        tile_layer1<C, false>(sm);
        __syncthreads();
        float z2[4][HPW];
        tile_gemm_fwd<C, false>(sm, z2);
        tile_ypart<C, false>(sm, z2);
        __syncthreads();
        if (t < TT && v < a.V)
        {
            const float y = tile_y(sm, t);
            a.out[v]      = valid ? softplusf_(y, a.beta) : 0.0f;
            if (a.out_node) a.out_node[v] = valid ? node : 0;
            if (a.out_valid) a.out_valid[v] = valid ? 1.0f : 0.0f;
        }
        __syncthreads();
    }
}

template <int C>
static cudaError_t launch_volume(const VolumeArgs& a, cudaStream_t st)
{
    const size_t smem = sizeof(TileSmem<C, false>);
    static int grid   = 0;
    if (grid == 0)
    {
        cudaFuncSetAttribute(k_volume_tiles<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        grid = resident_ctas((const void*)k_volume_tiles<C>, TN, smem, 0) * sm_count();
    }
    const int64_t ntiles = (a.V + TT - 1) / TT;
    const int g          = (int)std::min<int64_t>(grid, std::max<int64_t>(ntiles, 1));
    k_volume_tiles<C><<<g, TN, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace neat

using namespace neat;

extern "C" int neat_sample_volume(const void* tree_table, int max_depth, const float* node_min, const float* node_max,
                                  const float* grid, int channel_last, int C, int G, const float* decoder,
                                  float softplus_beta, int nx, int ny, int nz, float* out, int64_t* out_node,
                                  float* out_valid, neat_stream_t stream)
{
    if (C != 4 && C != 8 && C != 16) return NEAT_ERR_UNSUPPORTED;
    if (max_depth < 1 || max_depth > kMaxDepth || G < 2 || nx < 2 || ny < 2 || nz < 2) return NEAT_ERR_BAD_INPUT;
    if (!tree_table || !node_min || !node_max || !grid || !decoder || !out) return NEAT_ERR_BAD_INPUT;
    if (channel_last && ((uintptr_t)grid & 15)) return NEAT_ERR_BAD_INPUT;
    VolumeArgs a;
    a.table        = (const NodeEntry*)tree_table;
    a.max_depth    = max_depth;
    a.node_min     = node_min;
    a.node_max     = node_max;
    a.grid         = grid;
    a.channel_last = channel_last;
    a.G            = G;
    a.decoder      = decoder;
    a.beta         = softplus_beta;
    a.nx           = nx;
    a.ny           = ny;
    a.nz           = nz;
    a.V            = (int64_t)nx * ny * nz;
    a.out          = out;
    a.out_node     = out_node;
    a.out_valid    = out_valid;
    cudaError_t e  = cudaSuccess;
    switch (C)
    {
        case 4: e = launch_volume<4>(a, (cudaStream_t)stream); break;
        case 8: e = launch_volume<8>(a, (cudaStream_t)stream); break;
        default: e = launch_volume<16>(a, (cudaStream_t)stream); break;
    }
    return e == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
