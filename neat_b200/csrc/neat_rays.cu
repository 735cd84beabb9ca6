// neat_rays.cu -- camera rays, ray-octree intersection and stratified
// sampling (GetRays, IntersectBoxRayPrecise, ComputeRaySamples /
// CreateSamplesForRays of darglein/NeAT), B200 edition.
//
// One warp per ray.  The warp first evaluates the slab parameter of every
// dyadic plane the tree can have, T[a][k] = (plane_k - o_a) / d_a (3 * 17
// divisions at depth 4, instead of 6 per node box), then walks the octree
// top-down, one level per iteration: the 8 children of every frontier node
// are slab-tested 32 at a time, active children that are hit become segments
// and hit children with active descendants form the next frontier.  The
// reference tests every active node (HyperTree.cu:258-292); the walk finds
// the same set because the float slab interval of a child lies inside its
// parent's (fl((p - o) / d) is monotone in p), so a missed parent has only
// missed children.  Hits are rank-sorted by (tmin, node_id).  Segments and
// samples are written in that canonical order; the reference's order comes
// from a shared-memory atomic (src/structure/HyperTree.cu:281) and is not
// reproducible, its content (hit set, tmin/tmax, sample counts) is matched
// bit for bit.
#include <algorithm>
#include <cstdio>

#include "neat_common.cuh"
#include "neat_internal.h"
#include "neat_scan.cuh"

namespace neat
{

constexpr int RAY_WARPS = 4;  // rays per 128-thread block

constexpr int MAX_FRONT = 256;  // a line meets at most 3 * 2^d - 2 nodes of level d (d <= 6 here)

// Per-warp scratch of one ray: HC hits, FC frontier nodes, planes of depth <= DM.
template <int HC, int FC, int DM>
struct WarpHitsT
{
    static constexpr int kHits  = HC;
    static constexpr int kFront = FC;
    static constexpr int kDepth = DM;
    float T[3 * ((1 << DM) + 1)];
    float tmin[HC];
    float tmax[HC];
    int a[HC];     // active (local) id
    int node[HC];  // global node id
    int n[HC];     // samples of the segment
    int ord[HC];   // sorted position -> hit index
    int pre[HC];   // exclusive prefix of n in sorted order
    int front[2][FC];
};
// Any tree the library takes (the reference's 256-hit limit, depth 7).
using WarpHits = WarpHitsT<kMaxHits, MAX_FRONT, kMaxDepth>;
// The fused step with at most 64 hits kept per ray and depth <= 5: a line
// meets at most 3 * 2^4 - 2 = 46 nodes of level 4, so 64 frontier entries
// hold every internal level; 2.7 KB per warp instead of 10.7 KB.
using WarpHitsStep = WarpHitsT<64, 64, 5>;
// Depth 5 with room for every hit a line can have (3 * 2^5 - 2 = 94): the
// step's per-ray capacity of a depth-5 tree; 3.6 KB per warp.
using WarpHitsStep96 = WarpHitsT<96, 64, 5>;

// Hits of one ray: active nodes whose slab test passes and whose segment is
// at least 1e-5 long (HyperTree.cu:274-277).  Returns the raw count (only
// the first kMaxHits are stored); sets *overflow if a frontier overflowed.
template <class WH>
__device__ int warp_traverse_hits(const NodeEntry* __restrict__ tab, int D, int M, const float o[3], const float d[3],
                                  WH& ws, int lane, bool& overflow)
{
    constexpr int kMaxHits  = WH::kHits;
    constexpr int MAX_FRONT = WH::kFront;
    const int P = (1 << D) + 1;
    for (int i = lane; i < 3 * P; i += 32)
    {
        const int ax = i / P, k = i - ax * P;
        const float dv = d[ax];
        ws.T[i]        = (dv != 0.0f) ? plane_t(k, D, o[ax], dv) : 0.0f;
    }
    __syncwarp();
    int count = 0, fsz = 0, cur = 0;
    overflow  = false;
    // level 0: the root
    {
        bool act = false, below = false;
        float t0 = 0.0f, t1 = 0.0f;
        if (lane == 0)
        {
            const NodeEntry e = tab[0];
            const bool h      = slab_test(e, ws.T, P, D, o, d, t0, t1);
            act               = h && e.active && !(__fsub_rn(t1, t0) <= 1e-5f);  // (double)dt < 1e-5
            below             = h && e.below;
            if (act)
            {
                ws.tmin[0] = t0;
                ws.tmax[0] = t1;
                ws.a[0]    = e.local;
                ws.node[0] = 0;
                ws.n[0]    = iceil_pos(__fmul_rn(__fdiv_rn(__fsub_rn(t1, t0), e.diag), (float)M));
            }
            if (below) ws.front[0][0] = 0;
        }
        count = __shfl_sync(0xffffffffu, act ? 1 : 0, 0);
        fsz   = __shfl_sync(0xffffffffu, below ? 1 : 0, 0);
        __syncwarp();
    }
    while (fsz > 0)
    {
        const int total = fsz * 8;
        int nfsz        = 0;
        for (int base = 0; base < total; base += 32)
        {
            const int i = base + lane;
            bool act = false, below = false;
            float t0 = 0.0f, t1 = 0.0f;
            int node = 0, local = 0, n = 0;
            if (i < total)
            {
                node              = 8 * ws.front[cur][i >> 3] + 1 + (i & 7);
                const NodeEntry e = tab[node];
                const bool h      = slab_test(e, ws.T, P, D, o, d, t0, t1);
                const float dt    = __fsub_rn(t1, t0);
                act               = h && e.active && !(dt <= 1e-5f);  // (double)dt < 1e-5: 1e-5f is the float below
                below             = h && e.below;
                if (act)
                {
                    local = e.local;
                    n     = iceil_pos(__fmul_rn(__fdiv_rn(dt, e.diag), (float)M));
                }
            }
            const unsigned ma = __ballot_sync(0xffffffffu, act);
            const unsigned mb = __ballot_sync(0xffffffffu, below);
            const unsigned lt = (1u << lane) - 1u;
            if (act)
            {
                const int pos = count + __popc(ma & lt);
                if (pos < kMaxHits)
                {
                    ws.tmin[pos] = t0;
                    ws.tmax[pos] = t1;
                    ws.a[pos]    = local;
                    ws.node[pos] = node;
                    ws.n[pos]    = n;
                }
            }
            if (below)
            {
                const int pos = nfsz + __popc(mb & lt);
                if (pos < MAX_FRONT)
                    ws.front[cur ^ 1][pos] = node;
                else
                    overflow = true;
            }
            count += __popc(ma);
            nfsz += __popc(mb);
        }
        __syncwarp();
        fsz = nfsz < MAX_FRONT ? nfsz : MAX_FRONT;
        cur ^= 1;
    }
    overflow = __any_sync(0xffffffffu, overflow);
    return count;
}

// Rank sort by (tmin, node id) and exclusive prefix of sample counts in that
// order.  Returns the ray's total sample count.
template <class WH>
__device__ int warp_sort_prefix(WH& ws, int k, int lane)
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
// Node table pass 1: every node of the complete tree (plane indices, diagonal).
__global__ void k_tree_nodes(const float* __restrict__ nmin, const float* __restrict__ nmax, int64_t N, int D,
                             NodeEntry* __restrict__ table, uint32_t* __restrict__ below, int* status)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= N) return;
    NodeEntry e;
    e.local           = -1;
    e.active          = 0;
    e.below           = 0;
    const float scale = (float)(1 << (D - 1));
    bool ok           = true;
    float ext[3];
    for (int ax = 0; ax < 3; ++ax)
    {
        const float lo = nmin[3 * id + ax], hi = nmax[3 * id + ax];
        ext[ax]        = __fsub_rn(hi, lo);
        for (int side = 0; side < 2; ++side)
        {
            const float c   = side ? hi : lo;
            const float kf  = __fmul_rn(__fadd_rn(c, 1.0f), scale);
            const int k     = (int)kf;
            const bool good = (kf == (float)k) && k >= 0 && k <= (1 << D) && plane_coord(k, D) == c;
            ok              = ok && good;
            e.k[2 * ax + side] = (uint8_t)(good ? k : 0);
        }
    }
    e.diag    = node_diag(ext[0], ext[1], ext[2]);
    table[id] = e;
    below[id] = 0;
    if (!ok) raise_status(status, NEAT_ERR_NON_DYADIC);
}

// Pass 2: active nodes get their grid row; their ancestors are marked.
__global__ void k_tree_active(const int64_t* __restrict__ active_ids, int A, int64_t N, NodeEntry* __restrict__ table,
                              uint32_t* __restrict__ below, int* status)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A) return;
    const int64_t id = active_ids[a];
    if (id < 0 || id >= N)
    {
        raise_status(status, NEAT_ERR_BAD_INPUT);
        return;
    }
    table[id].local  = a;
    table[id].active = 1;
    for (int64_t p = id; p > 0;)
    {
        p = (p - 1) >> 3;
        atomicOr(&below[p], 1u);
    }
}

// Pass 3: copy the descendant marks into the entries.
__global__ void k_tree_below(int64_t N, NodeEntry* __restrict__ table, const uint32_t* __restrict__ below)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= N) return;
    table[id].below = below[id] ? 1 : 0;
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
    bool ovf     = false;
    int k        = warp_traverse_hits(table, D, M, o, d, ws, lane, ovf);
    if (k > kMaxHits || ovf)
    {
        if (lane == 0) raise_status(status, NEAT_ERR_TOO_MANY_HITS);
        k = min(k, kMaxHits);
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
    bool ovf     = false;
    int k        = warp_traverse_hits(table, D, M, o, d, ws, lane, ovf);
    k            = min(k, kMaxHits);
    warp_sort_prefix(ws, k, lane);
    const int64_t base = samp_off[r];
    bool overflow      = false;
    for (int p = 0; p < k; ++p)
    {
        const int i      = ws.ord[p];
        const int n      = ws.n[i];
        const float t0   = ws.tmin[i], t1 = ws.tmax[i];
        const int lb     = ws.pre[p];
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
// Fused step: one traversal per ray (canonical hit list kept per ray), then
// the lists are placed node-major.
// ---------------------------------------------------------------------------
// The rays come from k_make_rays, one thread per ray, launched just before:
// the f64 camera model (five divisions and a square root) would otherwise run
// on all 32 lanes of the ray's warp alike.
template <class WH>
__global__ void __launch_bounds__(32 * RAY_WARPS)
    k_step_rays(int64_t R, const NodeEntry* __restrict__ table, int D, int M, int cap_ray,
                const float* __restrict__ origin, const float* __restrict__ direction, SegRec* __restrict__ ray_hits,
                int* __restrict__ ray_nseg, int* __restrict__ node_nseg, int64_t* counters, int* status)
{
    constexpr int kMaxHits = WH::kHits;
    __shared__ WH sh[RAY_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * RAY_WARPS + warp;
    if (r >= R) return;
    float o[3], d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        o[c] = origin[3 * r + c];
        d[c] = direction[3 * r + c];
    }
    WH& ws   = sh[warp];
    bool ovf = false;
    int k    = warp_traverse_hits(table, D, M, o, d, ws, lane, ovf);
    if (k > kMaxHits || ovf)
    {
        // the reference keeps 256 hits; beyond this scratch's capacity the
        // step's own per-ray capacity (<= the scratch) is exceeded as well
        if (lane == 0) raise_status(status, (k > kMaxHits && kMaxHits < NEAT_MAX_HITS_PER_RAY && !ovf)
                                                ? NEAT_ERR_CAPACITY
                                                : NEAT_ERR_TOO_MANY_HITS);
        k = min(k, kMaxHits);
    }
    if (k > cap_ray)
    {
        if (lane == 0) raise_status(status, NEAT_ERR_CAPACITY);
        k = cap_ray;
    }
    warp_sort_prefix(ws, k, lane);
    SegRec* out = ray_hits + r * (int64_t)cap_ray;
    for (int p = lane; p < k; p += 32)
    {
        const int i = ws.ord[p];
        SegRec sg;
        sg.ray        = (int32_t)r;
        sg.local_base = ws.pre[p];
        sg.tmin       = ws.tmin[i];
        sg.tmax       = ws.tmax[i];
        sg.n          = ws.n[i];
        sg.row        = ws.a[i];
        // rank in its node's bucket (the count's own increment); the placement
        // puts the segment there and makes rm its ray-major index
        sg.rm         = atomicAdd(&node_nseg[sg.row], 1);
        sg.step       = __fdiv_rn(__fsub_rn(sg.tmax, sg.tmin), (float)sg.n);
        const NodeEntry e = table[ws.node[i]];
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
            sg.o[c]  = o[c];
            sg.d[c]  = d[c];
            sg.mn[c] = plane_coord(e.k[2 * c], D);  // exact: the box lies on the plane grid
            sg.mx[c] = plane_coord(e.k[2 * c + 1], D);
        }
        out[p] = sg;
    }
    if (lane == 0)
    {
        ray_nseg[r] = k;
        // the step's largest hit count: every ray's atomic on one address would
        // serialise at its L2 slice, so read first (a stale value only lets an
        // atomic through; the maximum is monotone) and reduce only when k may
        // raise it
        if ((unsigned long long)k > *(volatile unsigned long long*)&counters[2])
            atomicMax((unsigned long long*)&counters[2], (unsigned long long)k);
    }
}

// Place every ray's segments into its nodes' buckets: one thread per segment
// (ray-major index rm < counters[0]), 256 consecutive segments per block; the
// slot in the bucket is the rank the walk drew when it counted the segment.  The
// ray of a segment is the last r with ray_seg_off[r] <= rm: the block finds
// its first ray by a 256-ary search in global memory (each round every thread
// tests the lower end of one of 256 sub-ranges and __syncthreads_count picks
// the last sub-range that starts at or before the block's first segment: three
// rounds for 2^18 rays instead of 18 dependent loads), stages the next 257 ray
// offsets in shared memory and each thread searches there (rays that miss the
// volume own no segment, so a window can end before the block's last segment;
// such a thread searches global memory from the window's end).
constexpr int PLACE_T = 256;

__device__ __forceinline__ int64_t last_le(const int* __restrict__ off, int64_t lo, int64_t hi, int64_t v)
{
    // off[lo] <= v < off[hi]
    while (hi - lo > 1)
    {
        const int64_t mid = (lo + hi) >> 1;
        if (off[mid] <= v)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(PLACE_T)
    k_step_place(const SegRec* __restrict__ ray_hits, const int* __restrict__ ray_seg_off, int64_t R, int cap_ray,
                 const int* __restrict__ node_seg_off, SegRec* __restrict__ segs,
                 int* __restrict__ seg_n, int64_t* counters, int64_t cap, double* __restrict__ partial, int* status)
{
    __shared__ int soff[PLACE_T + 1];
    // more segments than the capacity: nothing is placed, the step processes
    // nothing (counters[0] = 0 for the kernels after this one)
    const int64_t n0   = counters[0];
    const int64_t nseg = n0 > cap ? 0 : n0;
    if (n0 > cap && blockIdx.x == 0 && threadIdx.x == 0)
    {
        raise_status(status, NEAT_ERR_CAPACITY);
        counters[0] = 0;
    }
    for (int64_t base = (int64_t)blockIdx.x * PLACE_T; base < nseg; base += (int64_t)gridDim.x * PLACE_T)
    {
        // ray_seg_off[lo] <= base < ray_seg_off[hi] (ray_seg_off[R] = total > base);
        // block-uniform bounds, the offsets are nondecreasing
        int64_t lo = 0, hi = R;
        while (hi - lo > 1)
        {
            const int64_t step = (hi - lo + PLACE_T - 1) / PLACE_T;
            const int64_t c    = lo + (int64_t)threadIdx.x * step;
            const int n        = __syncthreads_count(c < hi && ray_seg_off[c] <= base);  // >= 1: c = lo holds
            lo                 = lo + (int64_t)(n - 1) * step;
            hi                 = min(lo + step, hi);
        }
        const int64_t r0 = lo;
        for (int j = threadIdx.x; j <= PLACE_T; j += PLACE_T)
            soff[j] = (r0 + j <= R) ? ray_seg_off[r0 + j] : 0x7fffffff;
        __syncthreads();
        const int64_t rm = base + threadIdx.x;
        if (rm < nseg)
        {
            partial[rm] = 0.0;  // the segment's projection partial, summed by the forward tiles
            int64_t ray;
            if (rm < soff[PLACE_T])
            {
                int lo = 0, hi = PLACE_T;  // soff[lo] <= rm < soff[hi]
                while (hi - lo > 1)
                {
                    const int mid = (lo + hi) >> 1;
                    if (soff[mid] <= rm)
                        lo = mid;
                    else
                        hi = mid;
                }
                ray = r0 + lo;
            }
            else
            {
                ray = last_le(ray_seg_off, r0 + PLACE_T, R, rm);
            }
            const int p  = (int)(rm - ray_seg_off[ray]);
            SegRec sg    = ray_hits[ray * cap_ray + p];
            const int nm = node_seg_off[sg.row] + sg.rm;  // the rank the walk drew in the node's bucket
            if (rm < cap && nm < cap)  // always: the totals were checked against cap
            {
                sg.rm     = (int32_t)rm;
                segs[nm]  = sg;
                seg_n[nm] = sg.n;
            }
        }
        __syncthreads();  // soff is rewritten by the next round
    }
}

// ---------------------------------------------------------------------------
// Hits by a 3-D DDA over the finest cells (a tree of depth <= 5 whose active
// nodes are disjoint; cell_node maps each finest cell to its active node, or
// -1).  One thread per ray steps from cell to cell along the line inside the
// root box, in the order of the plane crossings (the slab parameters of the
// table the walk uses: plane_t); when the cell's node changes, the node's own
// slab test (slab_test_k, unchanged) gives its interval and the 1e-5 rule
// decides.  A node whose interval has positive length holds cells of
// positive length along the ray, so the DDA visits it; cells crossed at one
// point only (the ray through an edge or a corner) are stepped over, and a
// node touched only there fails the 1e-5 rule anyway.  Boxes are convex and
// disjoint, so each hit is visited once and in increasing tmin: the canonical
// (tmin, node id) order, with the same records as k_step_rays.
// ---------------------------------------------------------------------------
// The step uses it at depth 5, where it is faster than the walk (segment build
// 0.83 -> 0.75 ms at 2^19 rays); at depth 4 the walk is (0.36 against 0.37 ms).
constexpr int DDA_THREADS = 128;

__global__ void __launch_bounds__(DDA_THREADS)
    k_step_rays_dda(int64_t R, const NodeEntry* __restrict__ table, const int32_t* __restrict__ cell_node, int D,
                    int M, int cap_ray, const float* __restrict__ origin, const float* __restrict__ direction,
                    SegRec* __restrict__ ray_hits, int* __restrict__ ray_nseg, int* __restrict__ node_nseg,
                    int64_t* counters, int* status)
{
    const int64_t r = (int64_t)blockIdx.x * DDA_THREADS + threadIdx.x;
    if (r >= R) return;
    float o[3], d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        o[c] = origin[3 * r + c];
        d[c] = direction[3 * r + c];
    }
    const int N       = 1 << D;
    const int n_nodes = (int)tree_nodes(D);
    auto Tf           = [&](int a, int k) { return plane_t(k, D, o[a], d[a]); };
    bool bad          = false;
    SegRec* out = ray_hits + r * (int64_t)cap_ray;
    int k = 0, prefix = 0;
    bool over = false;
    // the segment of node `node` (visited in tmin order), if it is a hit
    auto emit = [&](int node) {
        const NodeEntry e = table[node];
        float t0, t1;
        const bool h   = slab_test_k(e.k, Tf, D, o, d, t0, t1);
        const float dt = __fsub_rn(t1, t0);
        if (!(h && e.active && !(dt <= 1e-5f))) return;  // (double)dt < 1e-5
        const int n = iceil_pos(__fmul_rn(__fdiv_rn(dt, e.diag), (float)M));
        if (k < cap_ray)
        {
            SegRec sg;
            sg.ray        = (int32_t)r;
            sg.local_base = prefix;
            sg.tmin       = t0;
            sg.tmax       = t1;
            sg.n          = n;
            sg.row        = e.local;
            sg.rm         = atomicAdd(&node_nseg[e.local], 1);
            sg.step       = __fdiv_rn(dt, (float)n);
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                sg.o[c]  = o[c];
                sg.d[c]  = d[c];
                sg.mn[c] = plane_coord(e.k[2 * c], D);
                sg.mx[c] = plane_coord(e.k[2 * c + 1], D);
            }
            out[k] = sg;
        }
        else
            over = true;
        prefix += n;
        ++k;
    };
    const uint8_t root[6] = {0, (uint8_t)N, 0, (uint8_t)N, 0, (uint8_t)N};
    float ta, tb;
    if (slab_test_k(root, Tf, D, o, d, ta, tb))
    {
        // the cell holding the line just after ta on each axis, and the slab
        // parameter where the line leaves it along that axis
        int ci[3];
        float nx[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
        {
            if (d[a] == 0.0f)
            {
                int lo = 0, hi = N;  // plane_coord(lo) <= o < plane_coord(hi)
                while (hi - lo > 1)
                {
                    const int mid = (lo + hi) >> 1;
                    if (plane_coord(mid, D) <= o[a])
                        lo = mid;
                    else
                        hi = mid;
                }
                ci[a] = lo;
                nx[a] = INFINITY;
            }
            else if (d[a] > 0.0f)
            {
                int lo = 0, hi = N;  // the last plane k < N with T(k) <= ta (T increases with k)
                while (hi - lo > 1)
                {
                    const int mid = (lo + hi) >> 1;
                    if (Tf(a, mid) <= ta)
                        lo = mid;
                    else
                        hi = mid;
                }
                ci[a] = lo;
                nx[a] = Tf(a, lo + 1);
            }
            else
            {
                int lo = 0, hi = N;  // the first plane k > 0 with T(k) <= ta (T decreases with k)
                while (hi - lo > 1)
                {
                    const int mid = (lo + hi) >> 1;
                    if (Tf(a, mid) <= ta)
                        hi = mid;
                    else
                        lo = mid;
                }
                ci[a] = hi - 1;
                nx[a] = Tf(a, hi - 1);
            }
        }
        int cur = -1;
        for (int steps = 0; steps < 3 * N + 3; ++steps)
        {
            int node = __ldg(cell_node + ((int64_t)ci[2] * N + ci[1]) * N + ci[0]);
            if (node < -1 || node >= n_nodes)
            {
                bad  = true;  // not a node of this tree: the map does not belong to it
                node = -1;
            }
            if (node != cur)
            {
                if (cur >= 0) emit(cur);
                cur = node;
            }
            const float tn = fminf(nx[0], fminf(nx[1], nx[2]));
            if (!(tn < tb)) break;
            bool out_of_box = false;
#pragma unroll
            for (int a = 0; a < 3; ++a)
            {
                if (nx[a] == tn)
                {
                    if (d[a] > 0.0f)
                    {
                        ++ci[a];
                        out_of_box = out_of_box || ci[a] >= N;
                        if (ci[a] < N) nx[a] = Tf(a, ci[a] + 1);
                    }
                    else
                    {
                        --ci[a];
                        out_of_box = out_of_box || ci[a] < 0;
                        if (ci[a] >= 0) nx[a] = Tf(a, ci[a]);
                    }
                }
            }
            if (out_of_box) break;
        }
        if (cur >= 0) emit(cur);
    }
    if (over) raise_status(status, NEAT_ERR_CAPACITY);
    if (bad) raise_status(status, NEAT_ERR_BAD_INPUT);
    if (k > NEAT_MAX_HITS_PER_RAY) raise_status(status, NEAT_ERR_TOO_MANY_HITS);
    k = min(k, cap_ray);
    ray_nseg[r] = k;
    if ((unsigned long long)k > *(volatile unsigned long long*)&counters[2])
        atomicMax((unsigned long long*)&counters[2], (unsigned long long)k);
}

cudaError_t launch_step_rays(const float* uv, const int32_t* image_id, int64_t R, int w, int h, const double* intr,
                             const double* rot, const double* trans, const void* table, int D, int M, int cap_ray,
                             float* origin, float* direction, SegRec* ray_hits, int* ray_nseg, int* node_nseg,
                             int64_t* counters, int* status, cudaStream_t st, const int32_t* cell_node)
{
    if (R <= 0) return cudaSuccess;
    k_make_rays<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(uv, image_id, nullptr, R, w, h, intr, rot, trans, origin,
                                                            direction);
    if (cell_node && D == 5)
    {
        k_step_rays_dda<<<(unsigned)((R + DDA_THREADS - 1) / DDA_THREADS), DDA_THREADS, 0, st>>>(
            R, (const NodeEntry*)table, cell_node, D, M, cap_ray, origin, direction, ray_hits, ray_nseg, node_nseg,
            counters, status);
        return cudaGetLastError();
    }
    const unsigned grid = (unsigned)((R + RAY_WARPS - 1) / RAY_WARPS);
    const NodeEntry* tab = (const NodeEntry*)table;
    if (cap_ray <= WarpHitsStep::kHits && D <= WarpHitsStep::kDepth)
        k_step_rays<WarpHitsStep><<<grid, 32 * RAY_WARPS, 0, st>>>(R, tab, D, M, cap_ray, origin, direction, ray_hits,
                                                                   ray_nseg, node_nseg, counters, status);
    else if (cap_ray <= WarpHitsStep96::kHits && D <= WarpHitsStep96::kDepth)
        k_step_rays<WarpHitsStep96><<<grid, 32 * RAY_WARPS, 0, st>>>(R, tab, D, M, cap_ray, origin, direction,
                                                                     ray_hits, ray_nseg, node_nseg, counters, status);
    else
        k_step_rays<WarpHits><<<grid, 32 * RAY_WARPS, 0, st>>>(R, tab, D, M, cap_ray, origin, direction, ray_hits,
                                                               ray_nseg, node_nseg, counters, status);
    return cudaGetLastError();
}

cudaError_t launch_step_place(const SegRec* ray_hits, const int* ray_nseg, const int* ray_seg_off, int64_t R,
                              int cap_ray, const int* node_seg_off, SegRec* segs, int* seg_n,
                              int64_t* counters, int64_t cap, double* partial, int* status, cudaStream_t st)
{
    if (R <= 0) return cudaSuccess;
    (void)ray_nseg;
    const int64_t est = std::min<int64_t>(cap, R * 8);
    const unsigned nb =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((est + PLACE_T - 1) / PLACE_T, (int64_t)sm_count() * 16));
    k_step_place<<<nb, PLACE_T, 0, st>>>(ray_hits, ray_seg_off, R, cap_ray, node_seg_off, segs, seg_n,
                                         counters, cap, partial, status);
    return cudaGetLastError();
}

}  // namespace neat

using namespace neat;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" size_t neat_tree_table_bytes(int max_depth)
{
    if (max_depth < 1 || max_depth > kMaxDepth) return 0;
    const int64_t N = tree_nodes(max_depth);
    return (size_t)N * sizeof(NodeEntry) + ((size_t)N * 4 + 255) / 256 * 256;
}

extern "C" int neat_tree_prepare(const float* node_min, const float* node_max, const int64_t* active_ids,
                                 int num_active, int max_depth, void* table, int* status, neat_stream_t stream)
{
    if (num_active < 0 || max_depth < 1 || max_depth > kMaxDepth || !node_min || !node_max || !table ||
        (num_active > 0 && !active_ids))
        return NEAT_ERR_BAD_INPUT;
    const int64_t N     = tree_nodes(max_depth);
    NodeEntry* entries  = (NodeEntry*)table;
    uint32_t* below     = (uint32_t*)((char*)table + (size_t)N * sizeof(NodeEntry));
    cudaStream_t st     = (cudaStream_t)stream;
    const unsigned gN   = (unsigned)((N + 255) / 256);
    k_tree_nodes<<<gN, 256, 0, st>>>(node_min, node_max, N, max_depth, entries, below, status);
    if (num_active > 0)
        k_tree_active<<<(num_active + 255) / 256, 256, 0, st>>>(active_ids, num_active, N, entries, below, status);
    k_tree_below<<<gN, 256, 0, st>>>(N, entries, below);
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
// Device address of g_noalloc_scratch in the current device's context (the
// host-side name is only a stand-in, never a device pointer).  Looked up on
// every call rather than cached per device ordinal: after a context is torn
// down and created again the module is loaded anew and the array may move.
// Once the module is loaded the lookup is a table read.
int noalloc_scratch(char** out)
{
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return NEAT_ERR_CUDA;
    *out = (char*)p;
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
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(out_count, 0, 2 * sizeof(int64_t), st) != cudaSuccess) return NEAT_ERR_CUDA;
    if (num_rays > kNoAllocRays) return NEAT_ERR_CAPACITY;  // beyond the static scratch: no kernel launched
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
