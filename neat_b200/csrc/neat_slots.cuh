// neat_slots.cuh -- map the 128 slots of a node-major sample tile to their
// segments and build each slot's sample (jittered position, weight, local
// coordinates, trilinear corners).  Shared by the SIMT and tcgen05 tile
// kernels of the fused step.
#pragma once

#include "neat_common.cuh"
#include "neat_internal.h"
#include "neat_proposal.cuh"

namespace neat
{

constexpr int SLOTS = 128;  // samples per tile

// mark/slot_seg: shared int[128] each; starts (optional): shared int[129].
// On return mark[s] is the node-major segment of slot s (tile samples
// g0 .. g0+127; slots past S map to the last segment) and, if given,
// starts[mark[s] - seg_lo] is that segment's first sample.  All threads of
// the block must call it.
__device__ __forceinline__ void tile_slot_segments(int64_t g0, int seg_lo, int nseg, const int* __restrict__ samp_off,
                                                   int* mark, int* slot_seg, int* starts = nullptr)
{
    const int t = threadIdx.x;
    for (int i = t; i < SLOTS; i += blockDim.x) mark[i] = (i == 0) ? seg_lo : -1;
    __syncthreads();
    for (int i = t; i <= SLOTS; i += blockDim.x)
    {
        const int seg = seg_lo + i;
        if (seg < nseg)
        {
            const int64_t o = samp_off[seg];
            if (starts) starts[i] = (int)o;
            if (o > g0 && o < g0 + SLOTS) mark[(int)(o - g0)] = seg;
        }
    }
    __syncthreads();
    if (t < SLOTS)
    {
        int v = mark[t];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if ((t & 31) >= o) v = max(v, y);
        }
        slot_seg[t] = v;
    }
    __syncthreads();
    if (t < SLOTS)
    {
        int v = slot_seg[t];
        for (int w2 = 0; w2 < (t >> 5); ++w2) v = max(v, slot_seg[w2 * 32 + 31]);
        mark[t] = v;
    }
    __syncthreads();
}

struct SlotSample
{
    bool valid;
    float weight;
    float lu, lv, lw;  // local coordinates in [-1,1]
    float u;           // stratified CDF position (j + a) / n of the sample
    float t;           // ray parameter of the sample
    int ray, rm, row;
};

// Sample of a slot whose segment record is r and whose index in the segment
// is j: stratified jitter (a = 0.5 when jitter is off), o + d t, local
// coordinates.
__device__ __forceinline__ SlotSample slot_sample(const SegRec& r, int j, bool valid, bool jitter, uint64_t seed,
                                                  uint32_t step)
{
    SlotSample q;
    q.valid = valid;
    if (!valid) j = 0;
    float ts, ws;
    seg_sample(r.tmin, r.tmax, r.n, j, jitter, seed, step, r.ray, r.local_base, ts, ws);
    q.t             = ts;
    q.lu            = local_coord(__fadd_rn(r.o[0], __fmul_rn(r.d[0], ts)), r.mn[0], r.mx[0]);
    q.lv            = local_coord(__fadd_rn(r.o[1], __fmul_rn(r.d[1], ts)), r.mn[1], r.mx[1]);
    q.lw            = local_coord(__fadd_rn(r.o[2], __fmul_rn(r.d[2], ts)), r.mn[2], r.mx[2]);
    q.weight        = q.valid ? ws : 0.0f;
    q.u             = 0.0f;
    q.ray           = r.ray;
    q.rm            = r.rm;
    q.row           = r.row;
    return q;
}

// slot_sample for a full warp of consecutive slots: each lane draws the
// jitter of its own sample and takes t of samples j-1 and j+1 from its
// neighbour lanes (consecutive slots of one segment are consecutive samples);
// lanes 0 and 31 need the one neighbour outside the warp, which every lane
// draws alongside its own (two independent Philox chains that interleave,
// instead of a second chain on two diverged lanes).  Same values as
// slot_sample when cdf is null; with a proposal CDF (8 bin ends of this slot's
// segment) the positions come from its inverse.  u (the stratified CDF
// position) only when want_u.  All 32 lanes must call it.
__device__ __forceinline__ SlotSample slot_sample_warp(const SegRec& r, int j, bool valid, bool jitter, uint64_t seed,
                                                       uint32_t step, const float* cdf = nullptr, bool want_u = true)
{
    SlotSample q;
    q.valid = valid;
    if (!valid) j = 0;
    float c[PBIN];
    if (cdf)
    {
        const float4 c0 = *reinterpret_cast<const float4*>(cdf);
        const float4 c1 = *reinterpret_cast<const float4*>(cdf + 4);
        c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
        c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
    }
    const int lane = threadIdx.x & 31;
    const int jx   = lane == 0 ? j - 1 : j + 1;  // the neighbour a warp edge lane cannot shuffle in
    const float a  = jitter_a(jitter, seed, step, r.ray, r.local_base + j);
    const float ax = jitter_a(jitter, seed, step, r.ray, r.local_base + jx);
    const float t  = cdf ? proposal_t(r.tmin, r.tmax, r.n, j, a, c) : seg_t(r.tmin, r.step, j, a);
    const float tx = cdf ? proposal_t(r.tmin, r.tmax, r.n, jx, ax, c) : seg_t(r.tmin, r.step, jx, ax);
    float tp       = __shfl_up_sync(0xffffffffu, t, 1);
    float tn       = __shfl_down_sync(0xffffffffu, t, 1);
    if (j > 0 && lane == 0) tp = tx;
    if (j < r.n - 1 && lane == 31) tn = tx;
    const float lo = j == 0 ? r.tmin : __fmul_rn(__fadd_rn(tp, t), 0.5f);
    const float hi = j == r.n - 1 ? r.tmax : __fmul_rn(__fadd_rn(tn, t), 0.5f);
    q.t            = t;
    q.lu           = local_coord(__fadd_rn(r.o[0], __fmul_rn(r.d[0], t)), r.mn[0], r.mx[0]);
    q.lv           = local_coord(__fadd_rn(r.o[1], __fmul_rn(r.d[1], t)), r.mn[1], r.mx[1]);
    q.lw           = local_coord(__fadd_rn(r.o[2], __fmul_rn(r.d[2], t)), r.mn[2], r.mx[2]);
    q.weight       = q.valid ? __fsub_rn(hi, lo) : 0.0f;
    q.u            = want_u ? __fdiv_rn(__fadd_rn((float)j, a), (float)r.n) : 0.0f;
    q.ray          = r.ray;
    q.rm           = r.rm;
    q.row          = r.row;
    return q;
}

}  // namespace neat
