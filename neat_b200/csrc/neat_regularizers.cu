// neat_regularizers.cu -- the volume regularisers of GeometryExEx
// (src/geometry/geometry_ex_ex.cpp:86-156): total variation of the node grids
// and the edge loss between neighbouring nodes' features.  Both add their
// gradient into the grid-gradient buffer of the fused step (channel-last), so
// a caller runs them on the step's stream right before neat_train_step, whose
// Adam then applies the sum.
#include <algorithm>

#include "neat_internal.h"
#include "neat_tiles.cuh"

namespace neat
{

// ---------------------------------------------------------------------------
// TV (TVLoss::forward, src/geometry/geometry_ex_ex.h:18-58, no weight):
//   loss = w * C * sum_d mean_a mean_{c, cells along d} |g[.., i+1, ..] - g[.., i, ..]|
// over the three grid axes; every node and axis has C (G-1) G^2 differences.
// ---------------------------------------------------------------------------
__global__ void k_tv(const float* __restrict__ grid, int64_t A, int C, int G, float w, float* __restrict__ grad,
                     float* __restrict__ loss_part)
{
    __shared__ float red[256];
    const int64_t G3 = (int64_t)G * G * G, n = A * G3 * C;
    // d(loss)/d(diff) = w * C / (A * C (G-1) G^2) * sign
    const float scale = w / ((float)A * (float)(G - 1) * (float)G * (float)G);
    float acc         = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t cell = i / C;
        const int64_t loc  = cell % G3;
        const int x = (int)(loc % G), y = (int)((loc / G) % G), z = (int)(loc / ((int64_t)G * G));
        const float v = grid[i];
        const int64_t stride[3] = {(int64_t)C, (int64_t)G * C, (int64_t)G * G * C};
        const int pos[3]        = {x, y, z};
        float gsum              = 0.0f;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
        {
            if (pos[ax] + 1 < G)
            {
                const float d = grid[i + stride[ax]] - v;  // this cell -> next along the axis
                acc += fabsf(d);
                gsum -= d > 0.0f ? scale : (d < 0.0f ? -scale : 0.0f);
            }
            if (pos[ax] > 0)
            {
                const float d = v - grid[i - stride[ax]];
                gsum += d > 0.0f ? scale : (d < 0.0f ? -scale : 0.0f);
            }
        }
        if (grad) grad[i] += gsum;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0] * scale;
}

__global__ void k_sum_into(const float* __restrict__ part, int n, float* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += part[i];
    *out += s;
}

// ---------------------------------------------------------------------------
// Edge loss (VolumeRegularizer, geometry_ex_ex.cpp:101-131, with
// NodeNeighborSamples, src/structure/HyperTree.cu:830-928): on every face of
// every active node a G x G lattice of points p = local * size + min
// (local: the face coordinate 0 or 1, the others i / (G-1)); the active node
// that contains p + eps * outward normal (ActiveNodeIdForGlobalPosition) and
// is not the node itself forms a pair.  error = mean_c |f_node(p) - f_other(p)|
// * r with r uniform in [0,1) per pair (Philox keyed on (node, face, point,
// step) here; torch::rand_like in the reference); loss = w * C * mean_pairs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool contains(const float* mn, const float* mx, const float p[3])
{
    return !(mn[0] > p[0] || mx[0] < p[0] || mn[1] > p[1] || mx[1] < p[1] || mn[2] > p[2] || mx[2] < p[2]);
}

__device__ __forceinline__ int64_t active_node_at(const NodeEntry* table, int max_depth, const float* node_min,
                                                  const float* node_max, const float p[3])
{
    const int64_t first_leaf = tree_nodes(max_depth - 1);
    int64_t n                = 0;
    for (int level = 0; level <= max_depth; ++level)
    {
        if (table[n].active) return n;
        if (n >= first_leaf) return -1;
        int64_t next = -1;
        for (int cid = 0; cid < 8; ++cid)
        {
            const int64_t c = 8 * n + 1 + cid;
            if (contains(node_min + 3 * c, node_max + 3 * c, p))
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

struct EdgeArgs
{
    const NodeEntry* table;
    int max_depth;
    const float* node_min;
    const float* node_max;
    const int64_t* active_ids;
    int64_t A;
    const float* grid;
    int G;
    float eps, w;
    uint64_t seed;
    uint32_t step;
    int* count;
    float* grad;
    float* loss_part;
};

// The pair of lattice point (node a, face f, point k): other node or -1, and the point.
__device__ __forceinline__ int64_t edge_pair(const EdgeArgs& e, int64_t a, int f, int k, float p[3], int64_t& node)
{
    node            = e.active_ids[a];
    const int side  = f >> 1, front = f & 1;
    const int sa    = (side + 1) % 3, sb = (side + 2) % 3;
    const float* mn = e.node_min + 3 * node;
    const float* mx = e.node_max + 3 * node;
    float local[3];
    local[side] = front ? 1.0f : 0.0f;
    local[sa]   = __fdiv_rn((float)(k % e.G), (float)(e.G - 1));
    local[sb]   = __fdiv_rn((float)(k / e.G), (float)(e.G - 1));
    float q[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        p[c] = __fadd_rn(__fmul_rn(local[c], __fsub_rn(mx[c], mn[c])), mn[c]);
        q[c] = p[c];
    }
    q[side] = __fadd_rn(q[side], front ? e.eps : -e.eps);
    const int64_t other = active_node_at(e.table, e.max_depth, e.node_min, e.node_max, q);
    return (other != -1 && other != node) ? other : -1;
}

__global__ void k_edge_count(EdgeArgs e)
{
    const int64_t per = 6ll * e.G * e.G;
    int cnt           = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e.A * per; i += (int64_t)gridDim.x * blockDim.x)
    {
        float p[3];
        int64_t node;
        if (edge_pair(e, i / per, (int)((i % per) / ((int64_t)e.G * e.G)), (int)(i % ((int64_t)e.G * e.G)), p, node) >=
            0)
            ++cnt;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(e.count, cnt);
}

template <int C>
__global__ void k_edge(EdgeArgs e)
{
    __shared__ float red[256];
    const int64_t per = 6ll * e.G * e.G;
    const int npairs  = *e.count;
    float acc         = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e.A * per && npairs > 0;
         i += (int64_t)gridDim.x * blockDim.x)
    {
        float p[3];
        int64_t node;
        const int64_t a = i / per;
        const int f = (int)((i % per) / ((int64_t)e.G * e.G)), k = (int)(i % ((int64_t)e.G * e.G));
        const int64_t other = edge_pair(e, a, f, k, p, node);
        if (other < 0) continue;
        const int64_t nd[2] = {node, other};
        float feat[2][C];
        Corners kc[2];
        int64_t row[2];
#pragma unroll
        for (int s = 0; s < 2; ++s)
        {
            const float* mn = e.node_min + 3 * nd[s];
            const float* mx = e.node_max + 3 * nd[s];
            igs_corners(local_coord(p[0], mn[0], mx[0]), local_coord(p[1], mn[1], mx[1]),
                        local_coord(p[2], mn[2], mx[2]), e.G, e.G, e.G, kc[s]);
            row[s] = e.table[nd[s]].local;
            gather_cl<C>(e.grid, row[s], e.G, kc[s], feat[s]);
        }
        const float r = uniform01(e.seed, (uint32_t)a, (uint32_t)(f * e.G * e.G + k), e.step, 0x45444745u);
        float err     = 0.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) err += fabsf(feat[0][c] - feat[1][c]);
        acc += err * r;  // * (1/C) * C
        if (e.grad)
        {
            // d loss / d feat_node[c] = w * r * sign / npairs, the other side opposite
            const float g = e.w * r / (float)npairs;
            float dx[C];
#pragma unroll
            for (int c = 0; c < C; ++c)
            {
                const float d = feat[0][c] - feat[1][c];
                dx[c]         = d > 0.0f ? g : (d < 0.0f ? -g : 0.0f);
            }
            scatter_cl<C>(e.grad, row[0], e.G, kc[0], dx);
#pragma unroll
            for (int c = 0; c < C; ++c) dx[c] = -dx[c];
            scatter_cl<C>(e.grad, row[1], e.G, kc[1], dx);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) e.loss_part[blockIdx.x] = npairs > 0 ? red[0] * e.w / (float)npairs : 0.0f;
}

}  // namespace neat

using namespace neat;

extern "C" size_t neat_regularizer_workspace_bytes(void) { return (size_t)(4 * 148 * 4 + 64) * 4; }

extern "C" int neat_tv_loss(const float* grid, int64_t A, int C, int G, float weight, float* loss, float* grid_grad,
                            void* workspace, neat_stream_t stream)
{
    if (!grid || !loss || !workspace || A < 1 || C < 1 || G < 2) return NEAT_ERR_BAD_INPUT;
    cudaStream_t st = (cudaStream_t)stream;
    const int nb    = std::min(4 * sm_count(), 4 * 148);
    float* part     = (float*)workspace;
    k_tv<<<nb, 256, 0, st>>>(grid, A, C, G, weight, grid_grad, part);
    k_sum_into<<<1, 32, 0, st>>>(part, nb, loss);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_edge_loss(const void* tree_table, int max_depth, const float* node_min, const float* node_max,
                              const int64_t* active_ids, int64_t A, const float* grid, int C, int G, float epsilon,
                              float weight, uint64_t seed, uint32_t step, float* loss, float* grid_grad,
                              void* workspace, neat_stream_t stream)
{
    if (!tree_table || !node_min || !node_max || !active_ids || !grid || !loss || !workspace || A < 1 || G < 2 ||
        max_depth < 1 || max_depth > kMaxDepth)
        return NEAT_ERR_BAD_INPUT;
    if (C != 4 && C != 8 && C != 16) return NEAT_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    const int nb    = std::min(4 * sm_count(), 4 * 148);
    float* part     = (float*)workspace;
    int* count      = (int*)(part + 4 * 148);
    EdgeArgs e{(const NodeEntry*)tree_table, max_depth, node_min, node_max, active_ids, A, grid, G, epsilon, weight,
               seed, step, count, grid_grad, part};
    if (cudaMemsetAsync(count, 0, sizeof(int), st) != cudaSuccess) return NEAT_ERR_CUDA;
    k_edge_count<<<nb, 256, 0, st>>>(e);
    switch (C)
    {
        case 4: k_edge<4><<<nb, 256, 0, st>>>(e); break;
        case 8: k_edge<8><<<nb, 256, 0, st>>>(e); break;
        default: k_edge<16><<<nb, 256, 0, st>>>(e); break;
    }
    k_sum_into<<<1, 32, 0, st>>>(part, nb, loss);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
