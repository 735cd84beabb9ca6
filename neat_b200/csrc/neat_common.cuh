// neat_common.cuh -- device helpers shared by the NeAT B200 kernels.
//
// Arithmetic that decides ray-node hits and sample counts is written with
// explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn,
// __dmul_rn ...) so that nvcc never contracts it into FMAs: the results are
// bit-identical to the source-order evaluation of the reference expressions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/neat_b200.h"

namespace neat
{

constexpr uint32_t kJitterStream = 0x4a495454u;  // 4th Philox counter word of the jitter stream
constexpr uint32_t kBatchStream  = 0x42415443u;  // synthetic ray batches
constexpr int kMaxHits           = NEAT_MAX_HITS_PER_RAY;
constexpr int kMaxDepth          = 7;  // plane indices fit in uint8 (2^7 + 1 planes per axis)

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11).  Counter-based: a value depends only
// on (seed, counter), never on launch geometry or scheduling.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r)
    {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c  = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ float uniform01(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3)
{
    uint4 o = philox4x32_10(make_uint4(c0, c1, c2, c3), (uint32_t)seed, (uint32_t)(seed >> 32));
    return (float)(o.x >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ void raise_status(int* status, int flag)
{
    if (status) atomicOr(status, flag);
}

// ---------------------------------------------------------------------------
// Node table entry, one per node of the complete octree (breadth-first ids:
// children of n are 8n+1 .. 8n+8): plane indices of the node's faces on the
// dyadic grid of depth D (plane k at -1 + k * 2^(1-D)), its diagonal, its
// grid row when active, and whether an active node lies below it.
// ---------------------------------------------------------------------------
struct __align__(16) NodeEntry
{
    int32_t local;   // active (local) id = grid row, or -1
    uint8_t k[6];    // x0, x1, y0, y1, z0, z1
    uint8_t active;  // 1: the node is active
    uint8_t below;   // 1: some descendant is active (traversal continues)
    float diag;
};

__host__ __device__ constexpr int64_t tree_nodes(int D)
{
    int64_t n = 0, p = 1;
    for (int i = 0; i <= D; ++i, p *= 8) n += p;
    return n;
}
static_assert(sizeof(NodeEntry) == 16, "NodeEntry must be 16 bytes");

__device__ __forceinline__ float plane_coord(int k, int D)
{
    // exact: k * 2^(1-D) is a dyadic rational with < 24 significant bits.
    // 2^(1-D) is built from its exponent field (128 - D; D <= 7 here), the
    // value 2 / 2^D has exactly, without a division.
    return __fadd_rn(__fmul_rn((float)k, __uint_as_float((uint32_t)(128 - D) << 23)), -1.0f);
}

// (box_max - box_min).norm() in float, evaluated a0 + (a1 + a2) (Eigen's
// fixed-size reduction), src/structure/HyperTree.cu:286.
__device__ __forceinline__ float node_diag(float dx, float dy, float dz)
{
    float s = __fadd_rn(__fmul_rn(dx, dx), __fadd_rn(__fmul_rn(dy, dy), __fmul_rn(dz, dz)));
    return __fsqrt_rn(s);
}

__device__ __forceinline__ int iceil_pos(float x)
{
    int i = (int)x;  // truncation toward zero, x > 0
    return i + ((float)i < x ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Ray generation, f64: SceneBase::GetRays (src/data/SceneBase.cpp:171-193),
// UVToPixel (src/modules/CameraPose.h:20-36), Unproject (CameraPose.cu:262-274),
// RotatePointGPUk (CameraPose.cu:20-33) with Eigen's quaternion rotation
//   uv = 2 (q.vec x p);  r = (p + w uv) + q.vec x uv.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void make_ray(float u, float v, int w, int h, const double* intr, const double* q,
                                         const double* t, float o[3], float d[3])
{
    float px = __fmul_rn(u, (float)(w - 1));
    float py = __fmul_rn(v, (float)(h - 1));
    double x = __ddiv_rn(__dsub_rn((double)px, intr[2]), intr[0]);
    double y = __ddiv_rn(__dsub_rn((double)py, intr[3]), intr[1]);
    double z = 1.0;
    double n = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    x = __ddiv_rn(x, n);
    y = __ddiv_rn(y, n);
    z = __ddiv_rn(z, n);
    double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
    double ux = __dsub_rn(__dmul_rn(qy, z), __dmul_rn(qz, y));
    double uy = __dsub_rn(__dmul_rn(qz, x), __dmul_rn(qx, z));
    double uz = __dsub_rn(__dmul_rn(qx, y), __dmul_rn(qy, x));
    ux = __dadd_rn(ux, ux);
    uy = __dadd_rn(uy, uy);
    uz = __dadd_rn(uz, uz);
    double cx = __dsub_rn(__dmul_rn(qy, uz), __dmul_rn(qz, uy));
    double cy = __dsub_rn(__dmul_rn(qz, ux), __dmul_rn(qx, uz));
    double cz = __dsub_rn(__dmul_rn(qx, uy), __dmul_rn(qy, ux));
    d[0] = (float)__dadd_rn(__dadd_rn(x, __dmul_rn(qw, ux)), cx);
    d[1] = (float)__dadd_rn(__dadd_rn(y, __dmul_rn(qw, uy)), cy);
    d[2] = (float)__dadd_rn(__dadd_rn(z, __dmul_rn(qw, uz)), cz);
    o[0] = (float)t[0];
    o[1] = (float)t[1];
    o[2] = (float)t[2];
}

// ---------------------------------------------------------------------------
// IntersectBoxRayPrecise (src/structure/HyperTree.h:41-83) on a node whose
// faces lie on the dyadic plane grid.  T[a*P + k] = (plane_k - o_a) / d_a in
// float for non-parallel axes.  The reference runs near/far in double from
// the bounds -236436436.0 and 43637575.0, neither a float; here they run in
// float from -inf / +inf with the same strict compares (so ties, +0 against
// -0 included, resolve alike), and the bounds enter at the end through their
// float neighbours:
//   (float)max(-236436436.0, near)   = max(near, -236436432.0f), also the
//     value the double compares see (no float lies strictly between);
//   min(43637575.0, far) in compares = min(far, 43637572.0f) (the float below),
//   (float)min(43637575.0, far)      = min(far, 43637576.0f) (the float above).
// Equal to the double form bit for bit (hit, tmin, tmax) over 2e8 random and
// boundary cases, signed zeros and infinities included.  The reference's
// early per-axis rejection gives the same answer as testing once at the end
// because near only grows and far only shrinks.  Returns hit, tmin, tmax
// (float, as the reference's tuple).
// ---------------------------------------------------------------------------
// The slab test of the box with plane indices k[0..5] (x0, x1, y0, y1, z0, z1);
// Tf(a, k) gives the slab parameter (plane_k - o_a) / d_a of axis a (read
// only where d_a != 0).
template <class TF>
__device__ __forceinline__ bool slab_test_k(const uint8_t* k, TF&& Tf, int D, const float o[3], const float d[3],
                                            float& tmin, float& tmax)
{
    float tn = -INFINITY, tf = INFINITY;
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        int k0 = k[2 * a], k1 = k[2 * a + 1];
        if (d[a] == 0.0f)
        {
            float mn = plane_coord(k0, D), mx = plane_coord(k1, D);
            ok = ok && !((o[a] < mn) || (o[a] >= mx));
        }
        else
        {
            float T1 = Tf(a, k0), T2 = Tf(a, k1);
            if (T1 > T2)
            {
                float tmp = T1;
                T1        = T2;
                T2        = tmp;
            }
            if (T1 > tn) tn = T1;
            if (T2 < tf) tf = T2;
        }
    }
    tn             = fmaxf(tn, -236436432.0f);
    const float fc = fminf(tf, 43637572.0f);
    ok             = ok && !(tn > fc) && !(fc < 0.0f);
    tmin           = ok ? tn : 0.0f;
    tmax           = ok ? fminf(tf, 43637576.0f) : 0.0f;
    return ok;
}

// The slab test of a node with the slab parameters of every plane in T
// ([3][P], P = 2^D + 1).
__device__ __forceinline__ bool slab_test(const NodeEntry& e, const float* T, int P, int D, const float o[3],
                                          const float d[3], float& tmin, float& tmax)
{
    return slab_test_k(
        e.k, [&](int a, int k) { return T[a * P + k]; }, D, o, d, tmin, tmax);
}

// The slab parameter of plane k of axis a: the value a [3][P] table holds.
__device__ __forceinline__ float plane_t(int k, int D, float oa, float da)
{
    return __fdiv_rn(__fsub_rn(plane_coord(k, D), oa), da);
}

// Stratified sample position j of a segment, HyperTree.cu:341-358, rounded as
// the reference's CUDA build computes it: nvcc contracts `tmin + j * step` into
// one fused multiply-add (checked bit for bit against the reference kernel
// compiled for sm_100a), and `t1 * (1 - a) + t2 * a` into
// fma(t1, 1 - a, t2 * a), the first product fused.  With a = 0.5 both products
// of the blend are exact, so the blend is the correctly rounded sum either way.
__device__ __forceinline__ float seg_t(float tmin, float step, int j, float a)
{
    float t1 = __fmaf_rn((float)j, step, tmin);
    float t2 = __fmaf_rn((float)(j + 1), step, tmin);
    return __fmaf_rn(t1, __fsub_rn(1.0f, a), __fmul_rn(t2, a));
}

__device__ __forceinline__ float jitter_a(bool jitter, uint64_t seed, uint32_t step, int ray, int local_index)
{
    return jitter ? uniform01(seed, (uint32_t)ray, (uint32_t)local_index, step, kJitterStream) : 0.5f;
}

// t_j and the midpoint-interval weight of sample j (HyperTree.cu:372-389).
__device__ __forceinline__ void seg_sample(float tmin, float tmax, int n, int j, bool jitter, uint64_t seed,
                                           uint32_t step, int ray, int local_base, float& t, float& w)
{
    float stp = __fdiv_rn(__fsub_rn(tmax, tmin), (float)n);
    t         = seg_t(tmin, stp, j, jitter_a(jitter, seed, step, ray, local_base + j));
    float lo, hi;
    if (j == 0)
        lo = tmin;
    else
        lo = __fmul_rn(__fadd_rn(seg_t(tmin, stp, j - 1, jitter_a(jitter, seed, step, ray, local_base + j - 1)), t),
                       0.5f);
    if (j == n - 1)
        hi = tmax;
    else
        hi = __fmul_rn(__fadd_rn(seg_t(tmin, stp, j + 1, jitter_a(jitter, seed, step, ray, local_base + j + 1)), t),
                       0.5f);
    w = __fsub_rn(hi, lo);
}

// local = (g - min) / (max - min) * 2 - 1, every op rounded (HyperTree.cu:177-192).
// Octree boxes have power-of-two sizes; dividing by 2^e is then the same
// correctly rounded value as multiplying by 2^-e, which is what is computed.
__device__ __forceinline__ float local_coord(float g, float mn, float mx)
{
    const float size = __fsub_rn(mx, mn);
    const float num  = __fsub_rn(g, mn);
    const uint32_t b = __float_as_uint(size);
    const uint32_t e = (b >> 23) & 0xFFu;
    float v;
    if ((b & 0x807FFFFFu) == 0u && e > 1u && e < 253u)
        v = __fmul_rn(num, __uint_as_float((254u - e) << 23));
    else
        v = __fdiv_rn(num, size);
    return __fsub_rn(__fmul_rn(v, 2.0f), 1.0f);
}

// ---------------------------------------------------------------------------
// IndirectGridSample3D corner setup (src/modules/IndirectGridSample3D.cu:449-540):
// unnormalise with align_corners, weights from unclamped corners, indices
// clamped to the grid (border by index clamp).  Corner q: x-bit q&1,
// y-bit (q>>1)&1, z-bit (q>>2)&1 -> tnw tne tsw tse bnw bne bsw bse.
// ---------------------------------------------------------------------------
struct Corners
{
    float ix, iy, iz;  // scaled coordinates
    int x0, y0, z0;    // unclamped tnw corner
    int cx0, cx1, cy0, cy1, cz0, cz1;
    float w[8];
};

__device__ __forceinline__ int clampi(int v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); }

__device__ __forceinline__ void igs_corners(float u, float v, float s, int Z, int Y, int X, Corners& k)
{
    float ix = __fmul_rn(__fmul_rn(__fadd_rn(u, 1.0f), 0.5f), (float)(X - 1));
    float iy = __fmul_rn(__fmul_rn(__fadd_rn(v, 1.0f), 0.5f), (float)(Y - 1));
    float iz = __fmul_rn(__fmul_rn(__fadd_rn(s, 1.0f), 0.5f), (float)(Z - 1));
    int x0 = (int)floorf(ix), y0 = (int)floorf(iy), z0 = (int)floorf(iz);
    float fx0 = (float)x0, fy0 = (float)y0, fz0 = (float)z0;
    float fx1 = (float)(x0 + 1), fy1 = (float)(y0 + 1), fz1 = (float)(z0 + 1);
    float ax0 = __fsub_rn(fx1, ix), ax1 = __fsub_rn(ix, fx0);
    float ay0 = __fsub_rn(fy1, iy), ay1 = __fsub_rn(iy, fy0);
    float az0 = __fsub_rn(fz1, iz), az1 = __fsub_rn(iz, fz0);
    k.w[0] = __fmul_rn(__fmul_rn(ax0, ay0), az0);
    k.w[1] = __fmul_rn(__fmul_rn(ax1, ay0), az0);
    k.w[2] = __fmul_rn(__fmul_rn(ax0, ay1), az0);
    k.w[3] = __fmul_rn(__fmul_rn(ax1, ay1), az0);
    k.w[4] = __fmul_rn(__fmul_rn(ax0, ay0), az1);
    k.w[5] = __fmul_rn(__fmul_rn(ax1, ay0), az1);
    k.w[6] = __fmul_rn(__fmul_rn(ax0, ay1), az1);
    k.w[7] = __fmul_rn(__fmul_rn(ax1, ay1), az1);
    k.ix = ix; k.iy = iy; k.iz = iz;
    k.x0 = x0; k.y0 = y0; k.z0 = z0;
    k.cx0 = clampi(x0, X); k.cx1 = clampi(x0 + 1, X);
    k.cy0 = clampi(y0, Y); k.cy1 = clampi(y0 + 1, Y);
    k.cz0 = clampi(z0, Z); k.cz1 = clampi(z0 + 1, Z);
}

__device__ __forceinline__ int corner_cell(const Corners& k, int q, int Y, int X)
{
    int z = (q & 4) ? k.cz1 : k.cz0;
    int y = (q & 2) ? k.cy1 : k.cy0;
    int x = (q & 1) ? k.cx1 : k.cx0;
    return (z * Y + y) * X + x;
}

// Block-wide exclusive-scan helpers live in neat_scan.cuh.

}  // namespace neat
