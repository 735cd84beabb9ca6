// neat_tiles.cuh -- sample-tile engine: grid lookup + decoder MLP + softplus
// and its hand-written backward, for 128 samples per tile on 256 threads.
//
// Forward per sample (GeometryExEx::SampleVolumeIndirect + DecodeFeatures,
// src/geometry/geometry_ex_ex.cpp:161-180, src/geometry/geometry.cpp:102-163):
//   x   = IGS(grid[row], local)                        [C]
//   h1  = silu(W1 x + b1), h2 = silu(W2 h1 + b2)      [64]
//   y   = w3 . h2 + b3;  density = softplus(y, beta)  (threshold 20)
//   val = density * weight                            (IntegrateSamplesXRay)
// Backward per sample, given dval = dL/dval:
//   dy = dval * weight * softplus'(y); dz2 = dy w3 * silu'(z2);
//   dW2 += dz2 h1^T; dh1 = W2^T dz2; dz1 = dh1 * silu'(z1); dW1 += dz1 x^T;
//   dx = W1^T dz1  -> scattered into the feature grid with the trilinear
//   corner weights (IndirectGridSample3D backward, .cu:584-801).
//
// The 64x64 layer runs as a register-tiled FP32 SIMT GEMM out of shared
// memory (each thread: 4 samples x 8 hidden units; operand reads are either
// conflict-free columns or warp broadcasts).  No TF32: the plain path keeps
// full FP32 products and accumulation.
#pragma once

#include "neat_common.cuh"

namespace neat
{

constexpr int TT  = 128;      // samples per tile
constexpr int TN  = 256;      // threads per CTA
constexpr int TW  = TN / 32;  // warps per CTA
constexpr int HH  = NEAT_HIDDEN;
constexpr int HPW = HH / TW;  // hidden units per warp in the GEMMs (8)
constexpr int LDS = HH + 4;   // padded row stride of [sample][hidden] tiles
static_assert(HPW == 8, "tile mapping assumes 8 hidden units per warp");

// Packed decoder parameter offsets (torch nn.Linear [out][in] weights).
template <int C>
struct DecOff
{
    static constexpr int W1 = 0;
    static constexpr int b1 = W1 + HH * C;
    static constexpr int W2 = b1 + HH;
    static constexpr int b2 = W2 + HH * HH;
    static constexpr int W3 = b2 + HH;
    static constexpr int b3 = W3 + HH;
    static constexpr int total = b3 + 1;
};

template <int C, bool BWD>
struct TileSmem
{
    float W1[HH * C];   // [h][c]
    float W2[HH * HH];  // [h_out][k_in]
    float W2T[HH * HH]; // [k_in][h_out]
    float b1[HH];
    float b2[HH];
    float w3[HH];
    float b3[4];
    float XT[C * TT];   // features [c][s]
    float H1T[HH * TT]; // [k][s]
    float ypart[TW * TT];
    float val[TT];      // per-slot value: contribution (fwd) / dL/dy (bwd)
    int mark[TT];
    int slot_seg[TT];
    float H1S[BWD ? TT * LDS : 4];  // [s][k]; reused for dz1 [s][k]
    float dZ2T[BWD ? HH * TT : 4];  // [h][s]; reused for dx partials
    float dZ2S[BWD ? TT * LDS : 4]; // [s][h]
};

__device__ __forceinline__ float sigmoidf_(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }
__device__ __forceinline__ float siluf_(float z) { return z * sigmoidf_(z); }
__device__ __forceinline__ float silu_grad(float z)
{
    float s = sigmoidf_(z);
    return s * (1.0f + z * (1.0f - s));
}
// torch softplus(x, beta, threshold=20)
__device__ __forceinline__ float softplusf_(float y, float beta)
{
    float bx = y * beta;
    return (bx > 20.0f) ? y : log1pf(__expf(bx)) / beta;
}
__device__ __forceinline__ float softplus_grad(float y, float beta)
{
    float bx = y * beta;
    if (bx > 20.0f) return 1.0f;
    float z = __expf(bx);
    return z / (z + 1.0f);
}

template <int C, bool BWD>
__device__ __forceinline__ void tile_load_decoder(TileSmem<C, BWD>& sm, const float* __restrict__ dec)
{
    using O = DecOff<C>;
    for (int i = threadIdx.x; i < HH * C; i += TN) sm.W1[i] = dec[O::W1 + i];
    for (int i = threadIdx.x; i < HH * HH; i += TN)
    {
        float v                       = dec[O::W2 + i];
        sm.W2[i]                      = v;
        sm.W2T[(i % HH) * HH + i / HH] = v;
    }
    for (int i = threadIdx.x; i < HH; i += TN)
    {
        sm.b1[i] = dec[O::b1 + i];
        sm.b2[i] = dec[O::b2 + i];
        sm.w3[i] = dec[O::W3 + i];
    }
    if (threadIdx.x == 0) sm.b3[0] = dec[O::b3];
}

// Layer 1 for all slots: thread t -> slot t&127, hidden half t>>7.
template <int C, bool BWD>
__device__ __forceinline__ void tile_layer1(TileSmem<C, BWD>& sm)
{
    const int s = threadIdx.x & (TT - 1);
    const int k0 = (threadIdx.x >> 7) * (HH / 2);
    float x[C];
#pragma unroll
    for (int c = 0; c < C; ++c) x[c] = sm.XT[c * TT + s];
#pragma unroll 4
    for (int kk = 0; kk < HH / 2; ++kk)
    {
        const int k = k0 + kk;
        float z     = sm.b1[k];
#pragma unroll
        for (int c = 0; c < C; ++c) z = fmaf(x[c], sm.W1[k * C + c], z);
        float h           = siluf_(z);
        sm.H1T[k * TT + s] = h;
        if (BWD) sm.H1S[s * LDS + k] = h;
    }
}

// z2[m][i] for samples l+32m, hidden 8w+i.
template <int C, bool BWD>
__device__ __forceinline__ void tile_gemm_fwd(TileSmem<C, BWD>& sm, float acc[4][HPW])
{
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < HPW; ++i)
    {
        float b = sm.b2[w * HPW + i];
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m][i] = b;
    }
#pragma unroll 4
    for (int k = 0; k < HH; ++k)
    {
        float a[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) a[m] = sm.H1T[k * TT + l + 32 * m];
        const float4 b0 = *reinterpret_cast<const float4*>(&sm.W2T[k * HH + w * HPW]);
        const float4 b1 = *reinterpret_cast<const float4*>(&sm.W2T[k * HH + w * HPW + 4]);
        const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int i = 0; i < HPW; ++i) acc[m][i] = fmaf(a[m], b[i], acc[m][i]);
    }
}

// y partial sums of this warp's hidden units -> sm.ypart[w][s]
template <int C, bool BWD>
__device__ __forceinline__ void tile_ypart(TileSmem<C, BWD>& sm, const float z2[4][HPW])
{
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
        float p = 0.0f;
#pragma unroll
        for (int i = 0; i < HPW; ++i) p = fmaf(siluf_(z2[m][i]), sm.w3[w * HPW + i], p);
        sm.ypart[w * TT + l + 32 * m] = p;
    }
}

template <int C, bool BWD>
__device__ __forceinline__ float tile_y(const TileSmem<C, BWD>& sm, int s)
{
    float y = sm.b3[0];
#pragma unroll
    for (int w = 0; w < TW; ++w) y += sm.ypart[w * TT + s];
    return y;
}

// Per-thread persistent decoder-gradient accumulators.
template <int C>
struct DecGradAcc
{
    float dW2[HPW][2];  // h = 8w+i, k = 2l+j
    float db2[HPW];     // h = 8w+i (partial over this lane's samples)
    float dW3[HPW];
    float dW1[C / 4 > 0 ? C / 4 : 1];  // k = t>>2, c = (t&3)*(C/4) + c'
    float db1;          // k = t>>2 (threads with t&3 == 0)
    float db3;          // slot threads
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int i = 0; i < HPW; ++i)
        {
            dW2[i][0] = dW2[i][1] = 0.0f;
            db2[i] = dW3[i] = 0.0f;
        }
#pragma unroll
        for (int c = 0; c < (C / 4 > 0 ? C / 4 : 1); ++c) dW1[c] = 0.0f;
        db1 = db3 = 0.0f;
    }
};

// Backward of the tile after sm.val[s] holds dL/dy for each slot (0 for
// padding slots).  z2 are the layer-2 pre-activations from tile_gemm_fwd.
// Leaves dL/dx for slot s in dx_out (threads < 128) and accumulates decoder
// gradients in acc.
template <int C>
__device__ __forceinline__ void tile_backward(TileSmem<C, true>& sm, const float z2[4][HPW], DecGradAcc<C>& g,
                                              float dx_out[C])
{
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    // dz2 = dy * w3 * silu'(z2); dW3 += h2 * dy; db2 += dz2
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
        const int s    = l + 32 * m;
        const float dy = sm.val[s];
        float d[HPW];
#pragma unroll
        for (int i = 0; i < HPW; ++i)
        {
            const int h = w * HPW + i;
            const float z = z2[m][i];
            d[i]          = dy * sm.w3[h] * silu_grad(z);
            g.dW3[i]      = fmaf(siluf_(z), dy, g.dW3[i]);
            g.db2[i] += d[i];
            sm.dZ2T[h * TT + s] = d[i];
        }
        *reinterpret_cast<float4*>(&sm.dZ2S[s * LDS + w * HPW])     = make_float4(d[0], d[1], d[2], d[3]);
        *reinterpret_cast<float4*>(&sm.dZ2S[s * LDS + w * HPW + 4]) = make_float4(d[4], d[5], d[6], d[7]);
    }
    __syncthreads();
    // dW2[h][k] += sum_s dz2[s][h] * h1[s][k]
#pragma unroll 4
    for (int s = 0; s < TT; ++s)
    {
        const float4 a0 = *reinterpret_cast<const float4*>(&sm.dZ2S[s * LDS + w * HPW]);
        const float4 a1 = *reinterpret_cast<const float4*>(&sm.dZ2S[s * LDS + w * HPW + 4]);
        const float2 b  = *reinterpret_cast<const float2*>(&sm.H1S[s * LDS + 2 * l]);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int i = 0; i < HPW; ++i)
        {
            g.dW2[i][0] = fmaf(a[i], b.x, g.dW2[i][0]);
            g.dW2[i][1] = fmaf(a[i], b.y, g.dW2[i][1]);
        }
    }
    // dh1[s][k] = sum_h dz2[s][h] W2[h][k]   (k = 8w+i, s = l+32m)
    float acc[4][HPW];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int i = 0; i < HPW; ++i) acc[m][i] = 0.0f;
#pragma unroll 4
    for (int h = 0; h < HH; ++h)
    {
        float a[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) a[m] = sm.dZ2T[h * TT + l + 32 * m];
        const float4 b0 = *reinterpret_cast<const float4*>(&sm.W2[h * HH + w * HPW]);
        const float4 b1 = *reinterpret_cast<const float4*>(&sm.W2[h * HH + w * HPW + 4]);
        const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int i = 0; i < HPW; ++i) acc[m][i] = fmaf(a[m], b[i], acc[m][i]);
    }
    __syncthreads();  // H1S, dZ2T, dZ2S free from here
    // dz1 = dh1 * silu'(z1), z1 recomputed from x; stored [s][k] in H1S
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
        const int s = l + 32 * m;
        float d[HPW];
#pragma unroll
        for (int i = 0; i < HPW; ++i)
        {
            const int k = w * HPW + i;
            float z     = sm.b1[k];
#pragma unroll
            for (int c = 0; c < C; ++c) z = fmaf(sm.XT[c * TT + s], sm.W1[k * C + c], z);
            d[i] = acc[m][i] * silu_grad(z);
        }
        *reinterpret_cast<float4*>(&sm.H1S[s * LDS + w * HPW])     = make_float4(d[0], d[1], d[2], d[3]);
        *reinterpret_cast<float4*>(&sm.H1S[s * LDS + w * HPW + 4]) = make_float4(d[4], d[5], d[6], d[7]);
    }
    __syncthreads();
    // dW1[k][c] += sum_s dz1[s][k] x[s][c]; db1[k] += sum_s dz1[s][k]
    {
        constexpr int CQ = (C / 4 > 0 ? C / 4 : 1);
        const int k = t >> 2, c0 = (t & 3) * CQ;
        if (c0 < C)
        {
            for (int s = 0; s < TT; ++s)
            {
                const float gz = sm.H1S[s * LDS + k];
#pragma unroll
                for (int c = 0; c < CQ; ++c) g.dW1[c] = fmaf(gz, sm.XT[(c0 + c) * TT + s], g.dW1[c]);
                if ((t & 3) == 0) g.db1 += gz;
            }
        }
    }
    // dx partial over a hidden half: thread t -> slot t&127, half t>>7
    {
        const int s = t & (TT - 1), k0 = (t >> 7) * (HH / 2);
        float p[C];
#pragma unroll
        for (int c = 0; c < C; ++c) p[c] = 0.0f;
#pragma unroll 4
        for (int kk = 0; kk < HH / 2; ++kk)
        {
            const float gz = sm.H1S[s * LDS + k0 + kk];
#pragma unroll
            for (int c = 0; c < C; ++c) p[c] = fmaf(gz, sm.W1[(k0 + kk) * C + c], p[c]);
        }
        float* dxp = sm.dZ2T;  // [half][s][c]
#pragma unroll
        for (int c = 0; c < C; ++c) dxp[((t >> 7) * TT + s) * C + c] = p[c];
    }
    __syncthreads();
    if (t < TT)
    {
        const float* dxp = sm.dZ2T;
#pragma unroll
        for (int c = 0; c < C; ++c) dx_out[c] = dxp[t * C + c] + dxp[(TT + t) * C + c];
    }
}

// Write this CTA's decoder-gradient partial (deterministic layout) or add it
// atomically into dst (atomic != 0).  scratch: >= TN floats of shared memory.
template <int C>
__device__ __forceinline__ void dec_grad_flush(const DecGradAcc<C>& g, float* __restrict__ dst, bool atomic,
                                               float* scratch)
{
    using O = DecOff<C>;
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    auto put = [&](int idx, float v) {
        if (atomic)
            atomicAdd(dst + idx, v);
        else
            dst[idx] = v;
    };
#pragma unroll
    for (int i = 0; i < HPW; ++i)
    {
        const int h = w * HPW + i;
        put(O::W2 + h * HH + 2 * l, g.dW2[i][0]);
        put(O::W2 + h * HH + 2 * l + 1, g.dW2[i][1]);
        float b = g.db2[i], v = g.dW3[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            b += __shfl_xor_sync(0xffffffffu, b, o);
            v += __shfl_xor_sync(0xffffffffu, v, o);
        }
        if (l == 0)
        {
            put(O::b2 + h, b);
            put(O::W3 + h, v);
        }
    }
    constexpr int CQ = (C / 4 > 0 ? C / 4 : 1);
    {
        const int k = t >> 2, c0 = (t & 3) * CQ;
        if (c0 < C)
        {
#pragma unroll
            for (int c = 0; c < CQ; ++c) put(O::W1 + k * C + c0 + c, g.dW1[c]);
            if ((t & 3) == 0) put(O::b1 + k, g.db1);
        }
    }
    // db3: block reduction of slot partials
    scratch[t] = (t < TT) ? g.db3 : 0.0f;
    __syncthreads();
    if (t == 0)
    {
        float s = 0.0f;
        for (int i = 0; i < TT; ++i) s += scratch[i];
        put(O::b3, s);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Feature gather (forward) and scatter (backward) for the two grid layouts.
// ---------------------------------------------------------------------------
// Channel-last [rows][G^3][C]: one corner is C contiguous floats.
template <int C>
__device__ __forceinline__ void gather_cl(const float* __restrict__ grid, int64_t row, int G, const Corners& k,
                                          float x[C])
{
    const int64_t base = row * (int64_t)G * G * G;
    if constexpr (C % 4 == 0)
    {
        // one round of 8 loads (one per corner) per 4 channels; each channel
        // still accumulates its corners in order 0..7
        const float* pq[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) pq[q] = grid + (base + corner_cell(k, q, G, G)) * C;
#pragma unroll
        for (int c4 = 0; c4 < C / 4; ++c4)
        {
            float4 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = __ldg(reinterpret_cast<const float4*>(pq[q]) + c4);
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                a0 = fmaf(v[q].x, k.w[q], a0);
                a1 = fmaf(v[q].y, k.w[q], a1);
                a2 = fmaf(v[q].z, k.w[q], a2);
                a3 = fmaf(v[q].w, k.w[q], a3);
            }
            x[4 * c4]     = a0;
            x[4 * c4 + 1] = a1;
            x[4 * c4 + 2] = a2;
            x[4 * c4 + 3] = a3;
        }
    }
    else
    {
#pragma unroll
        for (int c = 0; c < C; ++c) x[c] = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            const float* p = grid + (base + corner_cell(k, q, G, G)) * C;
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = fmaf(__ldg(p + c), k.w[q], x[c]);
        }
    }
}

// BF16 channel-last copy of the grid: one corner is C bf16 (C = 8: one
// 16-byte load); widened to f32, FP32 accumulation.
template <int C>
__device__ __forceinline__ void gather_cl_bf16(const uint16_t* __restrict__ grid, int64_t row, int G, const Corners& k,
                                               float x[C])
{
    const int64_t base = row * (int64_t)G * G * G;
#pragma unroll
    for (int c = 0; c < C; ++c) x[c] = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
    {
        const uint16_t* p = grid + (base + corner_cell(k, q, G, G)) * C;
        const float wq    = k.w[q];
        if constexpr (C % 8 == 0)
        {
#pragma unroll
            for (int c8 = 0; c8 < C / 8; ++c8)
            {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(p) + c8);
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int i = 0; i < 4; ++i)
                {
                    x[8 * c8 + 2 * i]     = fmaf(__uint_as_float(w[i] << 16), wq, x[8 * c8 + 2 * i]);
                    x[8 * c8 + 2 * i + 1] = fmaf(__uint_as_float(w[i] & 0xFFFF0000u), wq, x[8 * c8 + 2 * i + 1]);
                }
            }
        }
        else
        {
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = fmaf(__uint_as_float((uint32_t)__ldg(p + c) << 16), wq, x[c]);
        }
    }
}

__device__ __forceinline__ void red_add_v4(float* addr, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

template <int C>
__device__ __forceinline__ void scatter_cl(float* __restrict__ grad, int64_t row, int G, const Corners& k,
                                           const float dx[C])
{
    const int64_t base = row * (int64_t)G * G * G;
#pragma unroll
    for (int q = 0; q < 8; ++q)
    {
        float* p       = grad + (base + corner_cell(k, q, G, G)) * C;
        const float wq = k.w[q];
        if constexpr (C % 4 == 0)
        {
#pragma unroll
            for (int c4 = 0; c4 < C / 4; ++c4)
                red_add_v4(p + 4 * c4, wq * dx[4 * c4], wq * dx[4 * c4 + 1], wq * dx[4 * c4 + 2], wq * dx[4 * c4 + 3]);
        }
        else
        {
#pragma unroll
            for (int c = 0; c < C; ++c) atomicAdd(p + c, wq * dx[c]);
        }
    }
}

// Corners Q0 .. Q0+NQ-1 only (a sample's scatter split over threads or over
// phases; compile-time corners keep the corner arrays in registers).
template <int C, int Q0, int NQ>
__device__ __forceinline__ void scatter_cl_part(float* __restrict__ grad, int64_t row, int G, const Corners& k,
                                                const float dx[C])
{
    const int64_t base = row * (int64_t)G * G * G;
#pragma unroll
    for (int q = Q0; q < Q0 + NQ; ++q)
    {
        float* p       = grad + (base + corner_cell(k, q, G, G)) * C;
        const float wq = k.w[q];
        if constexpr (C % 4 == 0)
        {
#pragma unroll
            for (int c4 = 0; c4 < C / 4; ++c4)
                red_add_v4(p + 4 * c4, wq * dx[4 * c4], wq * dx[4 * c4 + 1], wq * dx[4 * c4 + 2], wq * dx[4 * c4 + 3]);
        }
        else
        {
#pragma unroll
            for (int c = 0; c < C; ++c) atomicAdd(p + c, wq * dx[c]);
        }
    }
}

// Corners 4*half .. 4*half+3 only (two threads share one sample's scatter).
template <int C>
__device__ __forceinline__ void scatter_cl_half(float* __restrict__ grad, int64_t row, int G, const Corners& k,
                                                const float dx[C], int half)
{
    const int64_t base = row * (int64_t)G * G * G;
#pragma unroll
    for (int qq = 0; qq < 4; ++qq)
    {
        const int q    = 4 * half + qq;
        float* p       = grad + (base + corner_cell(k, q, G, G)) * C;
        const float wq = k.w[q];
        if constexpr (C % 4 == 0)
        {
#pragma unroll
            for (int c4 = 0; c4 < C / 4; ++c4)
                red_add_v4(p + 4 * c4, wq * dx[4 * c4], wq * dx[4 * c4 + 1], wq * dx[4 * c4 + 2], wq * dx[4 * c4 + 3]);
        }
        else
        {
#pragma unroll
            for (int c = 0; c < C; ++c) atomicAdd(p + c, wq * dx[c]);
        }
    }
}

// Reference layout [rows][C][G^3].
template <int C>
__device__ __forceinline__ void gather_cf(const float* __restrict__ grid, int64_t row, int G, const Corners& k,
                                          float x[C])
{
    const int64_t G3 = (int64_t)G * G * G;
    int cell[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) cell[q] = corner_cell(k, q, G, G);
#pragma unroll
    for (int c = 0; c < C; ++c)
    {
        const float* p = grid + (row * C + c) * G3;
        float a        = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) a = fmaf(__ldg(p + cell[q]), k.w[q], a);
        x[c] = a;
    }
}

template <int C>
__device__ __forceinline__ void scatter_cf(float* __restrict__ grad, int64_t row, int G, const Corners& k,
                                           const float dx[C])
{
    const int64_t G3 = (int64_t)G * G * G;
#pragma unroll
    for (int c = 0; c < C; ++c)
    {
        float* p = grad + (row * C + c) * G3;
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(p + corner_cell(k, q, G, G), k.w[q] * dx[c]);
    }
}

}  // namespace neat
