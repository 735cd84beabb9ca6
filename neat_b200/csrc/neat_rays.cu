// neat_rays.cu -- camera rays, ray-octree intersection and stratified
// sampling (GetRays, IntersectBoxRayPrecise, ComputeRaySamples /
// CreateSamplesForRays of darglein/NeAT), B200 edition.
//
// One warp per ray.  The warp first evaluates the slab parameter of every
// dyadic plane the tree can have, T[a][k] = (plane_k - o_a) / d_a (3 * 17
// divisions at depth 4, instead of 6 per node), then tests all active nodes
// 32 at a time with table lookups, compacts the hits with a ballot into
// shared memory and rank-sorts them by (tmin, node_id).  Segments and
// samples are written in that canonical order; the reference's order comes
// from a shared-memory atomic (src/structure/HyperTree.cu:281) and is not
// reproducible, its content (hit set, tmin/tmax, sample counts) is matched
// bit for bit.
#include <cstdio>

#include "neat_common.cuh"
#include "neat_internal.h"
#include "neat_scan.cuh"

namespace neat
{

constexpr int RAY_WARPS = 4;  // rays per 128-thread block
constexpr int MAX_PLANES = (1 << kMaxDepth) + 1;

struct WarpHits
{
    float T[3 * MAX_PLANES];
    float tmin[kMaxHits];
    float tmax[kMaxHits];
    int a[kMaxHits];     // active (local) id
    int node[kMaxHits];  // global node id
    int n[kMaxHits];     // samples of the segment
    int ord[kMaxHits];   // sorted position -> hit index
    int pre[kMaxHits];   // exclusive prefix of n in sorted order
};

// Hits of one ray against all active nodes; returns the raw count (may
// exceed kMaxHits, in which case only the first kMaxHits are stored).
__device__ int warp_find_hits(const NodeEntry* __restrict__ table, int A, int D, int M, const float o[3],
                              const float d[3], WarpHits& ws, int lane)
{
    const int P = (1 << D) + 1;
    for (int i = lane; i < 3 * P; i += 32)
    {
        const int ax = i / P, k = i - ax * P;
        const float dv = d[ax];
        ws.T[i]        = (dv != 0.0f) ? __fdiv_rn(__fsub_rn(plane_coord(k, D), o[ax]), dv) : 0.0f;
    }
    __syncwarp();
    int count = 0;
    for (int base = 0; base < A; base += 32)
    {
        const int a = base + lane;
        bool hit    = false;
        float t0 = 0.0f, t1 = 0.0f;
        int n = 0, node = 0;
        if (a < A)
        {
            const NodeEntry e = table[a];
            const bool h      = slab_test(e, ws.T, P, D, o, d, t0, t1);
            const float dt    = __fsub_rn(t1, t0);
            // HyperTree.cu:274-277: skip when tmax - tmin < 1e-5 (float diff, double compare)
            if (h && !((double)dt < 1e-5))
            {
                hit  = true;
                n    = iceil_pos(__fmul_rn(__fdiv_rn(dt, e.diag), (float)M));
                node = e.node_id;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit)
        {
            const int pos = count + __popc(m & ((1u << lane) - 1u));
            if (pos < kMaxHits)
            {
                ws.tmin[pos] = t0;
                ws.tmax[pos] = t1;
                ws.a[pos]    = a;
                ws.node[pos] = node;
                ws.n[pos]    = n;
            }
        }
        count += __popc(m);
    }
    __syncwarp();
    return count;
}

// Rank sort by (tmin, node id) and exclusive prefix of sample counts in that
// order.  Returns the ray's total sample count.
__device__ int warp_sort_prefix(WarpHits& ws, int k, int lane)
{
    for (int i = lane; i < k; i += 32)
    {
        const float ti = ws.tmin[i];
        const int ni   = ws.node[i];
        int rank       = 0;
        for (int j = 0; j < k; ++j)
        {
            const float tj = ws.tmin[j];
            rank += (tj < ti) || (tj == ti && ws.node[j] < ni);
        }
        ws.ord[rank] = i;
    }
    __syncwarp();
    int carry = 0;
    for (int base = 0; base < k; base += 32)
    {
        const int p = base + lane;
        const int v = (p < k) ? ws.n[ws.ord[p]] : 0;
        int x       = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (p < k) ws.pre[p] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    __syncwarp();
    return carry;
}

// ---------------------------------------------------------------------------
// Node table
// ---------------------------------------------------------------------------
__global__ void k_tree_prepare(const float* __restrict__ nmin, const float* __restrict__ nmax,
                               const int64_t* __restrict__ active_ids, int A, int D, NodeEntry* __restrict__ table,
                               int* status)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A) return;
    const int64_t id = active_ids[a];
    NodeEntry e;
    e.node_id = (int32_t)id;
    e.pad[0] = e.pad[1] = 0;
    const float scale   = (float)(1 << (D - 1));
    bool ok             = true;
    float ext[3];
    for (int ax = 0; ax < 3; ++ax)
    {
        const float lo = nmin[3 * id + ax], hi = nmax[3 * id + ax];
        ext[ax]        = __fsub_rn(hi, lo);
        for (int side = 0; side < 2; ++side)
        {
            const float c  = side ? hi : lo;
            const float kf = __fmul_rn(__fadd_rn(c, 1.0f), scale);
            int k          = (int)kf;
            const bool good = (kf == (float)k) && k >= 0 && k <= (1 << D) && plane_coord(k, D) == c;
            ok              = ok && good;
            e.k[2 * ax + side] = (uint8_t)(good ? k : 0);
        }
    }
    e.diag = node_diag(ext[0], ext[1], ext[2]);
    if (!ok) raise_status(status, NEAT_ERR_NON_DYADIC);
    table[a] = e;
}

// ---------------------------------------------------------------------------
// Rays
// ---------------------------------------------------------------------------
__global__ void k_make_rays(const float* __restrict__ uv, const int32_t* __restrict__ image_id,
                            const int32_t* __restrict__ camera_id, int64_t R, int w, int h,
                            const double* __restrict__ intr, const double* __restrict__ rot,
                            const double* __restrict__ trans, float* __restrict__ origin,
                            float* __restrict__ direction)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int img = image_id[r];
    const int cam = camera_id ? camera_id[r] : 0;
    float o[3], d[3];
    make_ray(uv[2 * r], uv[2 * r + 1], w, h, intr + 5 * cam, rot + 4 * img, trans + 3 * img, o, d);
    for (int c = 0; c < 3; ++c)
    {
        origin[3 * r + c]    = o[c];
        direction[3 * r + c] = d[c];
    }
}

// ---------------------------------------------------------------------------
// CreateSamplesForRays: count pass and write pass
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * RAY_WARPS) k_samples_count(const float* __restrict__ origin,
                                                                  const float* __restrict__ direction, int64_t R,
                                                                  const NodeEntry* __restrict__ table, int A, int D,
                                                                  int M, int* __restrict__ ray_nsamp,
                                                                  int64_t* out_count, int* status)
{
    __shared__ WarpHits sh[RAY_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * RAY_WARPS + warp;
    if (r >= R) return;
    float o[3], d[3];
    for (int c = 0; c < 3; ++c)
    {
        o[c] = origin[3 * r + c];
        d[c] = direction[3 * r + c];
    }
    WarpHits& ws = sh[warp];
    int k        = warp_find_hits(table, A, D, M, o, d, ws, lane);
    if (k > kMaxHits)
    {
        if (lane == 0) raise_status(status, NEAT_ERR_TOO_MANY_HITS);
        k = kMaxHits;
    }
    int s = 0;
    for (int i = lane; i < k; i += 32) s += ws.n[i];
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o2);
    if (lane == 0)
    {
        ray_nsamp[r] = s;
        atomicMax((unsigned long long*)&out_count[1], (unsigned long long)s);
    }
}

__global__ void __launch_bounds__(32 * RAY_WARPS)
    k_samples_write(const float* __restrict__ origin, const float* __restrict__ direction, int64_t R,
                    const NodeEntry* __restrict__ table, int A, int D, int M, int jitter, uint64_t seed,
                    uint32_t step, const int64_t* __restrict__ samp_off, int64_t capacity, float* __restrict__ coords,
                    float* __restrict__ ray_t, float* __restrict__ weight, int64_t* __restrict__ ray_index,
                    int64_t* __restrict__ local_index, int64_t* __restrict__ node_id, int* status)
{
    __shared__ WarpHits sh[RAY_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * RAY_WARPS + warp;
    if (r >= R) return;
    float o[3], d[3];
    for (int c = 0; c < 3; ++c)
    {
        o[c] = origin[3 * r + c];
        d[c] = direction[3 * r + c];
    }
    WarpHits& ws = sh[warp];
    int k        = warp_find_hits(table, A, D, M, o, d, ws, lane);
    if (k > kMaxHits) k = kMaxHits;
    warp_sort_prefix(ws, k, lane);
    const int64_t base = samp_off[r];
    bool overflow      = false;
    for (int p = 0; p < k; ++p)
    {
        const int i = ws.ord[p];
        const int n = ws.n[i];
        const float t0 = ws.tmin[i], t1 = ws.tmax[i];
        const int lb    = ws.pre[p];
        const int64_t nd = ws.node[i];
        for (int j = lane; j < n; j += 32)
        {
            const int64_t s = base + lb + j;
            if (s >= capacity)
            {
                overflow = true;
                continue;
            }
            float t, wgt;
            seg_sample(t0, t1, n, j, jitter != 0, seed, step, (int)r, lb, t, wgt);
            ray_t[s]  = t;
            weight[s] = wgt;
            for (int c = 0; c < 3; ++c) coords[3 * s + c] = __fadd_rn(o[c], __fmul_rn(d[c], t));
            ray_index[s]   = r;
            local_index[s] = lb + j;
            node_id[s]     = nd;
        }
    }
    if (overflow) raise_status(status, NEAT_ERR_CAPACITY);
}

// ---------------------------------------------------------------------------
// Fused step: pass 1 (rays + counts) and pass 2 (segment lists)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * RAY_WARPS)
    k_step_rays_count(const float* __restrict__ uv, const int32_t* __restrict__ image_id, int64_t R, int w, int h,
                      const double* __restrict__ intr, const double* __restrict__ rot,
                      const double* __restrict__ trans, const NodeEntry* __restrict__ table, int A, int D, int M,
                      float* __restrict__ origin, float* __restrict__ direction, int* __restrict__ ray_nseg,
                      int* __restrict__ node_nseg, int64_t* counters, int* status)
{
    __shared__ WarpHits sh[RAY_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * RAY_WARPS + warp;
    if (r >= R) return;
    const int img = image_id[r];
    float o[3], d[3];
    make_ray(uv[2 * r], uv[2 * r + 1], w, h, intr, rot + 4 * img, trans + 3 * img, o, d);
    if (lane < 3)
    {
        origin[3 * r + lane]    = o[lane];
        direction[3 * r + lane] = d[lane];
    }
    WarpHits& ws = sh[warp];
    int k        = warp_find_hits(table, A, D, M, o, d, ws, lane);
    if (k > kMaxHits)
    {
        if (lane == 0) raise_status(status, NEAT_ERR_TOO_MANY_HITS);
        k = kMaxHits;
    }
    for (int i = lane; i < k; i += 32) atomicAdd(&node_nseg[ws.a[i]], 1);
    if (lane == 0)
    {
        ray_nseg[r] = k;
        atomicMax((unsigned long long*)&counters[2], (unsigned long long)k);
    }
}

__global__ void __launch_bounds__(32 * RAY_WARPS)
    k_step_rays_write(const float* __restrict__ origin, const float* __restrict__ direction, int64_t R,
                      const NodeEntry* __restrict__ table, int A, int D, int M, const int* __restrict__ ray_seg_off,
                      const int* __restrict__ node_seg_off, int* __restrict__ node_cursor, SegRec* __restrict__ segs,
                      int* __restrict__ seg_n, const int64_t* nseg_eff, int64_t cap, int* status)
{
    __shared__ WarpHits sh[RAY_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * RAY_WARPS + warp;
    if (r >= R) return;
    if (*nseg_eff == 0) return;  // nothing to place (no hits, or capacity overflow)
    float o[3], d[3];
    for (int c = 0; c < 3; ++c)
    {
        o[c] = origin[3 * r + c];
        d[c] = direction[3 * r + c];
    }
    WarpHits& ws = sh[warp];
    int k        = warp_find_hits(table, A, D, M, o, d, ws, lane);
    if (k > kMaxHits) k = kMaxHits;
    warp_sort_prefix(ws, k, lane);
    const int rbase = ray_seg_off[r];
    for (int p = lane; p < k; p += 32)
    {
        const int i  = ws.ord[p];
        const int a  = ws.a[i];
        const int rm = rbase + p;
        const int nm = node_seg_off[a] + atomicAdd(&node_cursor[a], 1);
        if (rm >= cap || nm >= cap)
        {
            raise_status(status, NEAT_ERR_CAPACITY);
            continue;
        }
        SegRec s;
        s.ray        = (int32_t)r;
        s.local_base = ws.pre[p];
        s.tmin       = ws.tmin[i];
        s.tmax       = ws.tmax[i];
        s.n          = ws.n[i];
        s.rm         = rm;
        s.row        = a;
        s.node       = ws.node[i];
        segs[nm]     = s;
        seg_n[nm]    = s.n;
    }
}

cudaError_t launch_step_rays_count(const float* uv, const int32_t* image_id, int64_t R, int w, int h,
                                   const double* intr, const double* rot, const double* trans, const void* table,
                                   int A, int D, int M, float* origin, float* direction, int* ray_nseg,
                                   int* node_nseg, int64_t* counters, int* status, cudaStream_t st)
{
    if (R <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((R + RAY_WARPS - 1) / RAY_WARPS);
    k_step_rays_count<<<grid, 32 * RAY_WARPS, 0, st>>>(uv, image_id, R, w, h, intr, rot, trans,
                                                       (const NodeEntry*)table, A, D, M, origin, direction, ray_nseg,
                                                       node_nseg, counters, status);
    return cudaGetLastError();
}

cudaError_t launch_step_rays_write(const float* origin, const float* direction, int64_t R, const void* table, int A,
                                   int D, int M, const int* ray_seg_off, const int* node_seg_off, int* node_cursor,
                                   SegRec* segs, int* seg_n, const int64_t* nseg_eff, int64_t cap, int* status,
                                   cudaStream_t st)
{
    if (R <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((R + RAY_WARPS - 1) / RAY_WARPS);
    k_step_rays_write<<<grid, 32 * RAY_WARPS, 0, st>>>(origin, direction, R, (const NodeEntry*)table, A, D, M,
                                                       ray_seg_off, node_seg_off, node_cursor, segs, seg_n, nseg_eff,
                                                       cap, status);
    return cudaGetLastError();
}

}  // namespace neat

using namespace neat;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" size_t neat_tree_table_bytes(int num_active) { return (size_t)(num_active > 0 ? num_active : 0) * 16; }

extern "C" int neat_tree_prepare(const float* node_min, const float* node_max, const int64_t* active_ids,
                                 int num_active, int max_depth, void* table, int* status, neat_stream_t stream)
{
    if (num_active < 0 || max_depth < 1 || max_depth > kMaxDepth || !node_min || !node_max ||
        (num_active > 0 && (!active_ids || !table)))
        return NEAT_ERR_BAD_INPUT;
    if (num_active == 0) return NEAT_OK;
    k_tree_prepare<<<(num_active + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        node_min, node_max, active_ids, num_active, max_depth, (NodeEntry*)table, status);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_make_rays(const float* uv, const int32_t* image_id, const int32_t* camera_id, int64_t num_rays,
                              int w, int h, const double* intrinsics, const double* rotation,
                              const double* translation, float* origin, float* direction, neat_stream_t stream)
{
    if (num_rays < 0 || w < 2 || h < 2) return NEAT_ERR_BAD_INPUT;
    if (num_rays == 0) return NEAT_OK;
    if (!uv || !image_id || !intrinsics || !rotation || !translation || !origin || !direction)
        return NEAT_ERR_BAD_INPUT;
    const unsigned grid = (unsigned)((num_rays + 255) / 256);
    k_make_rays<<<grid, 256, 0, (cudaStream_t)stream>>>(uv, image_id, camera_id, num_rays, w, h, intrinsics, rotation,
                                                        translation, origin, direction);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" size_t neat_samples_workspace_bytes(int64_t num_rays)
{
    const int64_t R = num_rays > 0 ? num_rays : 0;
    size_t b        = 0;
    b += ((size_t)R * 4 + 255) / 256 * 256;                              // ray_nsamp
    b += ((size_t)(R + 1) * 8 + 255) / 256 * 256;                        // samp_off
    b += ((size_t)scan_scratch_elems(R) * 8 + 255) / 256 * 256;          // scan scratch
    return b;
}

extern "C" int neat_create_samples(const void* table, int num_active, int max_depth, const float* origin,
                                   const float* direction, int64_t num_rays, int max_samples_per_node, int jitter,
                                   uint64_t seed, uint32_t step, int64_t capacity, float* coords, float* ray_t,
                                   float* weight, int64_t* ray_index, int64_t* local_index_in_ray, int64_t* node_id,
                                   int64_t* out_count, int* status, void* workspace, neat_stream_t stream)
{
    if (num_rays < 0 || num_active < 0 || max_depth < 1 || max_depth > kMaxDepth || max_samples_per_node < 1 ||
        capacity < 0 || !out_count)
        return NEAT_ERR_BAD_INPUT;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(out_count, 0, 2 * sizeof(int64_t), st) != cudaSuccess) return NEAT_ERR_CUDA;
    if (num_rays == 0) return NEAT_OK;
    if (!table && num_active > 0) return NEAT_ERR_BAD_INPUT;
    if (!origin || !direction || !workspace) return NEAT_ERR_BAD_INPUT;
    if (capacity > 0 && (!coords || !ray_t || !weight || !ray_index || !local_index_in_ray || !node_id))
        return NEAT_ERR_BAD_INPUT;
    char* ws        = (char*)workspace;
    int* ray_nsamp  = (int*)ws;
    ws += ((size_t)num_rays * 4 + 255) / 256 * 256;
    int64_t* samp_off = (int64_t*)ws;
    ws += ((size_t)(num_rays + 1) * 8 + 255) / 256 * 256;
    int64_t* scratch = (int64_t*)ws;
    const unsigned grid = (unsigned)((num_rays + RAY_WARPS - 1) / RAY_WARPS);
    k_samples_count<<<grid, 32 * RAY_WARPS, 0, st>>>(origin, direction, num_rays, (const NodeEntry*)table, num_active,
                                                     max_depth, max_samples_per_node, ray_nsamp, out_count, status);
    if (scan_exclusive<int64_t>(ray_nsamp, nullptr, num_rays, samp_off, scratch, out_count, st) != cudaSuccess)
        return NEAT_ERR_CUDA;
    k_samples_write<<<grid, 32 * RAY_WARPS, 0, st>>>(origin, direction, num_rays, (const NodeEntry*)table, num_active,
                                                     max_depth, max_samples_per_node, jitter, seed, step, samp_off,
                                                     capacity, coords, ray_t, weight, ray_index, local_index_in_ray,
                                                     node_id, status);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Sampling without a caller workspace.
//
// Some callers cannot allocate device memory while they run (a host framework
// that owns the GPU's memory pool, a latency-bound loop that cannot afford the
// device-wide synchronisation of cudaMalloc, a binding that only passes input
// and output arrays).  For them the per-ray counts, offsets and scan partials
// of the sampler live in this file-scope array, sized for
// NEAT_NOALLOC_MAX_RAYS rays.  Every GPU that loads the library keeps it until
// the process exits.  All calls on a device share it: the kernels overwrite
// every entry they read before reading it, so nothing needs clearing between
// calls, but calls that overlap on the GPU race on it.
// ---------------------------------------------------------------------------
#include <mutex>

namespace neat
{
constexpr int64_t kNoAllocRays = NEAT_NOALLOC_MAX_RAYS;
constexpr size_t kNoAllocNsampBytes = ((size_t)kNoAllocRays * 4 + 255) / 256 * 256;
constexpr size_t kNoAllocOffBytes   = ((size_t)(kNoAllocRays + 1) * 8 + 255) / 256 * 256;
constexpr size_t kNoAllocScanBytes  = ((size_t)((kNoAllocRays + SCAN_TILE - 1) / SCAN_TILE + 1) * 8 + 255) / 256 * 256;
constexpr size_t kNoAllocBytes      = kNoAllocNsampBytes + kNoAllocOffBytes + kNoAllocScanBytes;
}  // namespace neat

static __device__ __align__(256) unsigned char g_noalloc_scratch[neat::kNoAllocBytes];

namespace
{
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the host-side name is only a stand-in, never a device pointer).
int noalloc_scratch(char** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return NEAT_ERR_CUDA;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return NEAT_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev])
    {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return NEAT_ERR_CUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = (char*)g_noalloc_ptr[dev];
    return NEAT_OK;
}
}  // namespace

extern "C" int neat_create_samples_noalloc(const void* table, int num_active, int max_depth, const float* origin,
                                           const float* direction, int64_t num_rays, int max_samples_per_node,
                                           int jitter, uint64_t seed, uint32_t step, int64_t capacity, float* coords,
                                           float* ray_t, float* weight, int64_t* ray_index,
                                           int64_t* local_index_in_ray, int64_t* node_id, int64_t* out_count,
                                           int* status, neat_stream_t stream)
{
    if (num_rays < 0 || num_active < 0 || max_depth < 1 || max_depth > kMaxDepth || max_samples_per_node < 1 ||
        capacity < 0 || !out_count)
        return NEAT_ERR_BAD_INPUT;
    if (num_rays > kNoAllocRays) return NEAT_ERR_CAPACITY;  // beyond the static scratch: nothing launched
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(out_count, 0, 2 * sizeof(int64_t), st) != cudaSuccess) return NEAT_ERR_CUDA;
    if (num_rays == 0) return NEAT_OK;
    if (!table && num_active > 0) return NEAT_ERR_BAD_INPUT;
    if (!origin || !direction) return NEAT_ERR_BAD_INPUT;
    if (capacity > 0 && (!coords || !ray_t || !weight || !ray_index || !local_index_in_ray || !node_id))
        return NEAT_ERR_BAD_INPUT;
    char* ws = nullptr;
    const int e = noalloc_scratch(&ws);
    if (e != NEAT_OK) return e;
    int* ray_nsamp    = (int*)ws;
    int64_t* samp_off = (int64_t*)(ws + kNoAllocNsampBytes);
    int64_t* scratch  = (int64_t*)(ws + kNoAllocNsampBytes + kNoAllocOffBytes);
    const unsigned grid = (unsigned)((num_rays + RAY_WARPS - 1) / RAY_WARPS);
    k_samples_count<<<grid, 32 * RAY_WARPS, 0, st>>>(origin, direction, num_rays, (const NodeEntry*)table, num_active,
                                                     max_depth, max_samples_per_node, ray_nsamp, out_count, status);
    if (scan_exclusive<int64_t>(ray_nsamp, nullptr, num_rays, samp_off, scratch, out_count, st) != cudaSuccess)
        return NEAT_ERR_CUDA;
    k_samples_write<<<grid, 32 * RAY_WARPS, 0, st>>>(origin, direction, num_rays, (const NodeEntry*)table, num_active,
                                                     max_depth, max_samples_per_node, jitter, seed, step, samp_off,
                                                     capacity, coords, ray_t, weight, ray_index, local_index_in_ray,
                                                     node_id, status);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
