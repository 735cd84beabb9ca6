// neat_structure.cu -- GPU side of the octree structure updates:
//   ComputeMaxDensity (samples/reconstruct.cpp:254-286) with PointInAnyImage
//   (src/data/SceneBase.cu:13-45), and InterpolateInactiveNodes
//   (src/geometry/geometry_ex_ex.cpp:182-209).  The structure decisions
//   themselves (culling, the MIP) stay on the host.
//
// Node lattice of both (UniformGlobalSamples, src/structure/HyperTree.cu:781-815):
// cell (x, y, z) of a G^3 lattice at local (x, y, z) / (G-1) in [0,1], global
// position local * size + min (two roundings), cells x fastest.
#include <algorithm>

#include "neat_internal.h"
#include "neat_tiles.cuh"

namespace neat
{

__device__ __forceinline__ void lattice_point(int64_t cell, int G, const float* mn, const float* mx, float p[3])
{
    const int r[3] = {(int)(cell % G), (int)((cell / G) % G), (int)(cell / ((int64_t)G * G))};
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const float l = __fdiv_rn((float)r[d], (float)(G - 1));
        p[d]          = __fadd_rn(__fmul_rn(l, __fsub_rn(mx[d], mn[d])), mn[d]);
    }
}

// PointInAnyImage: the point projects, rounded to the nearest pixel, into some
// image: view = R^T (p - t) from the camera-to-world pose (quaternion x,y,z,w),
// pixel = (fx x/z + cx, fy y/z + cy) (skew 0), in f64.
__device__ __forceinline__ bool point_in_any_image(const float p[3], int n_img, int w, int h, const double* intr,
                                                   const double* rot, const double* trans)
{
    const double fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    for (int i = 0; i < n_img; ++i)
    {
        const double qx = rot[4 * i], qy = rot[4 * i + 1], qz = rot[4 * i + 2], qw = rot[4 * i + 3];
        const double vx = (double)p[0] - trans[3 * i], vy = (double)p[1] - trans[3 * i + 1],
                     vz = (double)p[2] - trans[3 * i + 2];
        // rotate by the conjugate: v' = v + 2 w' (u' x v) + 2 u' x (u' x v), u' = -u
        const double ux = -qx, uy = -qy, uz = -qz;
        const double tx = 2.0 * (uy * vz - uz * vy), ty = 2.0 * (uz * vx - ux * vz), tz = 2.0 * (ux * vy - uy * vx);
        const double x = vx + qw * tx + (uy * tz - uz * ty);
        const double y = vy + qw * ty + (uz * tx - ux * tz);
        const double z = vz + qw * tz + (ux * ty - uy * tx);
        const double px = round(fx * x / z + cx), py = round(fy * y / z + cy);
        if (px >= 0.0 && px < (double)w && py >= 0.0 && py < (double)h) return true;
    }
    return false;
}

// Max over the node lattice of the decoded density (times the in-image mask).
template <int C>
__global__ void __launch_bounds__(256) k_node_max_density(const int64_t* __restrict__ active_ids, int64_t A,
                                                          const float* __restrict__ node_min,
                                                          const float* __restrict__ node_max,
                                                          const float* __restrict__ grid, int G,
                                                          const float* __restrict__ dec, float beta, int n_img, int w,
                                                          int h, const double* intr, const double* rot,
                                                          const double* trans, float* __restrict__ out_max)
{
    using O = DecOff<C>;
    __shared__ float sW1[HH * C], sb1[HH], sW2[HH * HH], sb2[HH], sw3[HH];
    __shared__ float red[256];
    const int t = threadIdx.x;
    for (int i = t; i < HH * C; i += 256) sW1[i] = dec[O::W1 + i];
    for (int i = t; i < HH * HH; i += 256) sW2[i] = dec[O::W2 + i];
    if (t < HH)
    {
        sb1[t] = dec[O::b1 + t];
        sb2[t] = dec[O::b2 + t];
        sw3[t] = dec[O::W3 + t];
    }
    const float b3 = dec[O::b3];
    __syncthreads();
    const int64_t cells = (int64_t)G * G * G;
    for (int64_t a = blockIdx.x; a < A; a += gridDim.x)
    {
        const int64_t node = active_ids[a];
        const float* mn    = node_min + 3 * node;
        const float* mx    = node_max + 3 * node;
        float best         = 0.0f;
        for (int64_t cell = t; cell < cells; cell += 256)
        {
            float p[3];
            lattice_point(cell, G, mn, mx, p);
            if (n_img > 0 && !point_in_any_image(p, n_img, w, h, intr, rot, trans)) continue;  // density * 0
            Corners kc;
            igs_corners(local_coord(p[0], mn[0], mx[0]), local_coord(p[1], mn[1], mx[1]),
                        local_coord(p[2], mn[2], mx[2]), G, G, G, kc);
            float x[C];
            gather_cl<C>(grid, a, G, kc, x);
            float h1[HH];
#pragma unroll
            for (int j = 0; j < HH; ++j)
            {
                float z = sb1[j];
#pragma unroll
                for (int c = 0; c < C; ++c) z = fmaf(sW1[j * C + c], x[c], z);
                h1[j] = siluf_(z);
            }
            float y = b3;
#pragma unroll 4
            for (int k = 0; k < HH; ++k)
            {
                float z = sb2[k];
#pragma unroll
                for (int j = 0; j < HH; ++j) z = fmaf(sW2[k * HH + j], h1[j], z);
                y = fmaf(sw3[k], siluf_(z), y);
            }
            best = fmaxf(best, softplusf_(y, beta));
        }
        red[t] = best;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1)
        {
            if (t < o) red[t] = fmaxf(red[t], red[t + o]);
            __syncthreads();
        }
        if (t == 0) out_max[a] = red[0];
        __syncthreads();
    }
}

// InterpolateInactiveNodes: every lattice point of every new active node takes
// the old grid's features there (old node by the top-down descent; outside
// every old active node the first old active node, as NodeIdForPositionGPU
// returns, with its clamped border).
template <int C>
__global__ void k_interpolate_grid(const int64_t* __restrict__ new_ids, int64_t newA, const float* __restrict__ node_min,
                                   const float* __restrict__ node_max, const NodeEntry* __restrict__ old_table,
                                   int max_depth, int64_t old_first, const float* __restrict__ old_grid, int G,
                                   float* __restrict__ new_grid)
{
    const int64_t cells = (int64_t)G * G * G;
    const int64_t first_leaf = tree_nodes(max_depth - 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < newA * cells;
         i += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t a = i / cells, cell = i % cells;
        const int64_t node = new_ids[a];
        float p[3];
        lattice_point(cell, G, node_min + 3 * node, node_max + 3 * node, p);
        // ActiveNodeIdForGlobalPosition in the old tree
        int64_t n = 0, found = -1;
        for (int level = 0; level <= max_depth; ++level)
        {
            if (old_table[n].active)
            {
                found = n;
                break;
            }
            if (n >= first_leaf) break;
            int64_t next = -1;
            for (int cid = 0; cid < 8; ++cid)
            {
                const int64_t c = 8 * n + 1 + cid;
                const float* mn = node_min + 3 * c;
                const float* mx = node_max + 3 * c;
                if (!(mn[0] > p[0] || mx[0] < p[0] || mn[1] > p[1] || mx[1] < p[1] || mn[2] > p[2] || mx[2] < p[2]))
                {
                    next = c;
                    break;
                }
            }
            if (next < 0) break;
            n = next;
        }
        const int64_t on = found >= 0 ? found : old_first;
        const float* mn  = node_min + 3 * on;
        const float* mx  = node_max + 3 * on;
        Corners kc;
        igs_corners(local_coord(p[0], mn[0], mx[0]), local_coord(p[1], mn[1], mx[1]), local_coord(p[2], mn[2], mx[2]),
                    G, G, G, kc);
        float x[C];
        gather_cl<C>(old_grid, old_table[on].local, G, kc, x);
        float* dst = new_grid + i * C;
#pragma unroll
        for (int c = 0; c < C; ++c) dst[c] = x[c];
    }
}

}  // namespace neat

using namespace neat;

extern "C" int neat_node_max_density(const int64_t* active_ids, int64_t num_active, const float* node_min,
                                     const float* node_max, const float* grid, int C, int G, const float* decoder,
                                     float softplus_beta, int num_images, int w, int h, const double* intrinsics,
                                     const double* rotation, const double* translation, float* out_max,
                                     neat_stream_t stream)
{
    if (!active_ids || !node_min || !node_max || !grid || !decoder || !out_max || num_active < 1 || G < 2)
        return NEAT_ERR_BAD_INPUT;
    if (num_images > 0 && (!intrinsics || !rotation || !translation || w < 1 || h < 1)) return NEAT_ERR_BAD_INPUT;
    if ((uintptr_t)grid & 15) return NEAT_ERR_BAD_INPUT;
    const int nb    = (int)std::min<int64_t>(num_active, (int64_t)sm_count() * 8);
    cudaStream_t st = (cudaStream_t)stream;
    switch (C)
    {
        case 4:
            k_node_max_density<4><<<nb, 256, 0, st>>>(active_ids, num_active, node_min, node_max, grid, G, decoder,
                                                       softplus_beta, num_images, w, h, intrinsics, rotation,
                                                       translation, out_max);
            break;
        case 8:
            k_node_max_density<8><<<nb, 256, 0, st>>>(active_ids, num_active, node_min, node_max, grid, G, decoder,
                                                       softplus_beta, num_images, w, h, intrinsics, rotation,
                                                       translation, out_max);
            break;
        case 16:
            k_node_max_density<16><<<nb, 256, 0, st>>>(active_ids, num_active, node_min, node_max, grid, G, decoder,
                                                        softplus_beta, num_images, w, h, intrinsics, rotation,
                                                        translation, out_max);
            break;
        default: return NEAT_ERR_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_interpolate_grid(const int64_t* new_active_ids, int64_t new_num_active, const float* node_min,
                                     const float* node_max, const void* old_tree_table, int max_depth,
                                     int64_t old_first_active, const float* old_grid, int C, int G, float* new_grid,
                                     neat_stream_t stream)
{
    if (!new_active_ids || !node_min || !node_max || !old_tree_table || !old_grid || !new_grid ||
        new_num_active < 1 || G < 2 || max_depth < 1 || max_depth > kMaxDepth || old_first_active < 0)
        return NEAT_ERR_BAD_INPUT;
    if (((uintptr_t)old_grid | (uintptr_t)new_grid) & 15) return NEAT_ERR_BAD_INPUT;
    const int64_t n = new_num_active * (int64_t)G * G * G;
    const int nb    = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16);
    cudaStream_t st = (cudaStream_t)stream;
    const NodeEntry* tab = (const NodeEntry*)old_tree_table;
    switch (C)
    {
        case 4:
            k_interpolate_grid<4><<<nb, 256, 0, st>>>(new_active_ids, new_num_active, node_min, node_max, tab,
                                                       max_depth, old_first_active, old_grid, G, new_grid);
            break;
        case 8:
            k_interpolate_grid<8><<<nb, 256, 0, st>>>(new_active_ids, new_num_active, node_min, node_max, tab,
                                                       max_depth, old_first_active, old_grid, G, new_grid);
            break;
        case 16:
            k_interpolate_grid<16><<<nb, 256, 0, st>>>(new_active_ids, new_num_active, node_min, node_max, tab,
                                                        max_depth, old_first_active, old_grid, G, new_grid);
            break;
        default: return NEAT_ERR_UNSUPPORTED;
    }
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
