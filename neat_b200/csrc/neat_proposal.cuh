// neat_proposal.cuh -- the learned sample proposal: a tiny MLP that maps a
// ray-node segment to a piecewise-constant sample density along it.
//
// Input (16 floats): the node's descriptor (the method's own density in the
// node on a 4^3 lattice: centroid xyz, spread, log mean, log peak/mean), the
// segment's entry and exit points in node-local coordinates [-1,1]^3, the
// chord length over the node edge, the centroid's projection onto the chord
// and its distance from it over the spread, one zero.  MLP 16 -> 32 -> 32 -> 8 with SiLU; the 8 outputs
// are logits of the sample density over 8 equal sub-intervals of
// [tmin, tmax]: p = (1 - mix) softmax(z) + mix / 8, so every sub-interval keeps
// at least mix / 8 of the samples (uniform stratified sampling is the mix = 1
// limit and stays the fallback).  Samples are placed by inverting the
// piecewise-linear CDF at stratified u_j = (j + a_j) / n; their weights follow
// the reference's midpoint rule on the placed positions.
#pragma once

#include "neat_common.cuh"
#include "neat_internal.h"

namespace neat
{

constexpr int PIN  = NEAT_PROPOSAL_IN;
constexpr int PH   = NEAT_PROPOSAL_HIDDEN;
constexpr int PBIN = NEAT_PROPOSAL_BINS;

struct PropOff
{
    static constexpr int W1    = 0;
    static constexpr int b1    = W1 + PH * PIN;
    static constexpr int W2    = b1 + PH;
    static constexpr int b2    = W2 + PH * PH;
    static constexpr int W3    = b2 + PH;
    static constexpr int b3    = W3 + PBIN * PH;
    // count head: v = bv + Wv . h2 + Uv . f, a prediction of log(a + 1e-4),
    // a = (tmax - tmin) times the total variation of the density along the
    // segment, trained by regression on the trunk's features (the trunk gets
    // no gradient from it)
    static constexpr int VW    = b3 + PBIN;
    static constexpr int VU    = VW + PH;
    static constexpr int VB    = VU + PIN;
    static constexpr int total = VB + 1;
};

// Samples of a segment under the count head's prediction v: the midpoint
// rule with n samples misses about a / (2 n) of the segment's integral at
// density jumps, so n = ceil(exp(v) / eps) keeps that near eps / 2; clamped to
// [min(nmin, n_ref), n_ref] (n_ref: the reference's count at the budget).
// eps <= 0 keeps n_ref.
__device__ __forceinline__ int proposal_count(float v, int n_ref, float eps, int nmin)
{
    if (!(eps > 0.0f)) return n_ref;
    const float x = fminf(expf(v) / eps, (float)n_ref);  // NaN v: fminf keeps n_ref
    const int n   = max((int)ceilf(x), min(nmin, n_ref));
    return min(n, n_ref);
}

__device__ __forceinline__ float prop_sigmoid(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }

constexpr int PDESC = 6;  // node descriptor floats

__device__ __forceinline__ void proposal_features(const SegRec& r, const float* __restrict__ node_desc, float f[PIN])
{
#pragma unroll
    for (int i = 0; i < PDESC; ++i) f[i] = node_desc[PDESC * (int64_t)r.row + i];
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        f[6 + c] = local_coord(__fadd_rn(r.o[c], __fmul_rn(r.d[c], r.tmin)), r.mn[c], r.mx[c]);
        f[9 + c] = local_coord(__fadd_rn(r.o[c], __fmul_rn(r.d[c], r.tmax)), r.mn[c], r.mx[c]);
    }
    f[12] = (r.tmax - r.tmin) / (r.mx[0] - r.mn[0]);
    // where the node's mass lies relative to the segment: the centroid's
    // projection onto the chord (0 at entry, 1 at exit) and its distance from
    // the chord over the spread
    const float ex = f[9] - f[6], ey = f[10] - f[7], ez = f[11] - f[8];
    const float cx = f[0] - f[6], cy = f[1] - f[7], cz = f[2] - f[8];
    const float L2 = ex * ex + ey * ey + ez * ez + 1e-12f;
    const float us = (cx * ex + cy * ey + cz * ez) / L2;
    const float p2 = fmaxf(cx * cx + cy * cy + cz * cz - us * us * L2, 0.0f);
    f[13] = fminf(fmaxf(us, -0.5f), 1.5f);
    f[14] = sqrtf(p2) / (f[3] + 0.05f);
    f[15] = 0.0f;
}

// Forward of the proposal MLP from parameters P (shared or global memory).
// Returns the mixed bin probabilities; keeps z1, z2 (pre-activations) and the
// softmax for the backward when asked.
struct PropAct
{
    float z1[PH], z2[PH];
    float sm[PBIN];
};

__device__ __forceinline__ void proposal_forward(const float* __restrict__ P, const float f[PIN], float mix,
                                                 float p[PBIN], PropAct* act)
{
    float h1[PH], h2[PH];
#pragma unroll
    for (int j = 0; j < PH; ++j)
    {
        float z = P[PropOff::b1 + j];
#pragma unroll
        for (int i = 0; i < PIN; ++i) z = fmaf(P[PropOff::W1 + j * PIN + i], f[i], z);
        if (act) act->z1[j] = z;
        h1[j] = z * prop_sigmoid(z);
    }
#pragma unroll
    for (int k = 0; k < PH; ++k)
    {
        float z = P[PropOff::b2 + k];
#pragma unroll
        for (int j = 0; j < PH; ++j) z = fmaf(P[PropOff::W2 + k * PH + j], h1[j], z);
        if (act) act->z2[k] = z;
        h2[k] = z * prop_sigmoid(z);
    }
    float z3[PBIN], mx = -3.0e38f;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        float z = P[PropOff::b3 + b];
#pragma unroll
        for (int k = 0; k < PH; ++k) z = fmaf(P[PropOff::W3 + b * PH + k], h2[k], z);
        z3[b] = z;
        mx    = fmaxf(mx, z);
    }
    float sum = 0.0f;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        z3[b] = __expf(z3[b] - mx);
        sum += z3[b];
    }
    const float inv = 1.0f / sum;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        const float s = z3[b] * inv;
        if (act) act->sm[b] = s;
        p[b] = fmaf(1.0f - mix, s, mix * (1.0f / PBIN));
    }
}

// proposal_forward for two segments at once in packed f32x2 arithmetic (each
// lane rounds as fmaf does, so each segment's result is proposal_forward's):
// half the FMA instructions, the weight loads shared.
// Also the count head's v of both segments (v0, v1).
__device__ __forceinline__ void proposal_forward2(const float* __restrict__ P, const float f0[PIN],
                                                  const float f1[PIN], float mix, float p0[PBIN], float p1[PBIN],
                                                  float& v0, float& v1)
{
    float2 F[PIN];
#pragma unroll
    for (int i = 0; i < PIN; ++i) F[i] = make_float2(f0[i], f1[i]);
    float2 vh = make_float2(P[PropOff::VB], P[PropOff::VB]);
#pragma unroll
    for (int i = 0; i < PIN; ++i)
    {
        const float u = P[PropOff::VU + i];
        vh            = __ffma2_rn(make_float2(u, u), F[i], vh);
    }
    float2 h1[PH];
#pragma unroll
    for (int j = 0; j < PH; ++j)
    {
        const float b = P[PropOff::b1 + j];
        float2 z      = make_float2(b, b);
#pragma unroll
        for (int i = 0; i < PIN; ++i)
        {
            const float w = P[PropOff::W1 + j * PIN + i];
            z             = __ffma2_rn(make_float2(w, w), F[i], z);
        }
        h1[j] = make_float2(z.x * prop_sigmoid(z.x), z.y * prop_sigmoid(z.y));
    }
    // layer 2 fused into layer 3: each h2 unit goes into the 8 output sums as
    // it is made (each sum still runs over k in order, as proposal_forward's)
    float2 z3[PBIN];
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        const float bb = P[PropOff::b3 + b];
        z3[b]          = make_float2(bb, bb);
    }
#pragma unroll
    for (int k = 0; k < PH; ++k)
    {
        const float b = P[PropOff::b2 + k];
        float2 z      = make_float2(b, b);
#pragma unroll
        for (int j = 0; j < PH; ++j)
        {
            const float w = P[PropOff::W2 + k * PH + j];
            z             = __ffma2_rn(make_float2(w, w), h1[j], z);
        }
        const float2 h2 = make_float2(z.x * prop_sigmoid(z.x), z.y * prop_sigmoid(z.y));
#pragma unroll
        for (int b = 0; b < PBIN; ++b)
        {
            const float w = P[PropOff::W3 + b * PH + k];
            z3[b]         = __ffma2_rn(make_float2(w, w), h2, z3[b]);
        }
        const float wv = P[PropOff::VW + k];
        vh             = __ffma2_rn(make_float2(wv, wv), h2, vh);
    }
    v0 = vh.x;
    v1 = vh.y;
    float mx0 = -3.0e38f, mx1 = -3.0e38f;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        mx0 = fmaxf(mx0, z3[b].x);
        mx1 = fmaxf(mx1, z3[b].y);
    }
    float sum0 = 0.0f, sum1 = 0.0f;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        z3[b].x = __expf(z3[b].x - mx0);
        z3[b].y = __expf(z3[b].y - mx1);
        sum0 += z3[b].x;
        sum1 += z3[b].y;
    }
    const float inv0 = 1.0f / sum0, inv1 = 1.0f / sum1;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        p0[b] = fmaf(1.0f - mix, z3[b].x * inv0, mix * (1.0f / PBIN));
        p1[b] = fmaf(1.0f - mix, z3[b].y * inv1, mix * (1.0f / PBIN));
    }
}

// Cumulative bin ends c[b] = p_0 + .. + p_b, c[7] = 1 exactly.
__device__ __forceinline__ void proposal_cdf(const float p[PBIN], float c[PBIN])
{
    float acc = 0.0f;
#pragma unroll
    for (int b = 0; b < PBIN; ++b)
    {
        acc  = __fadd_rn(acc, p[b]);
        c[b] = acc;
    }
    c[PBIN - 1] = 1.0f;
}

// Position in [0,1] of CDF value u (u in [0,1)): inverse of the piecewise-
// linear CDF with bin ends c[]; every op rounded.
__device__ __forceinline__ float proposal_inverse(const float c[PBIN], float u)
{
    int b    = 0;
    float lo = 0.0f, hi = c[0];  // selected with constant indices: c stays in registers
#pragma unroll
    for (int i = 0; i < PBIN - 1; ++i)
        if (u >= c[i])
        {
            b  = i + 1;
            lo = c[i];
            hi = c[i + 1];
        }
    const float w = __fsub_rn(hi, lo);
    float fr      = w > 0.0f ? __fdiv_rn(__fsub_rn(u, lo), w) : 0.5f;
    fr            = fminf(fmaxf(fr, 0.0f), 1.0f);
    return __fmul_rn(__fadd_rn((float)b, fr), 1.0f / PBIN);
}

// t of sample j (jitter offset a) of a segment under the proposal CDF c.
__device__ __forceinline__ float proposal_t(float tmin, float tmax, int n, int j, float a, const float c[PBIN])
{
    const float u = __fdiv_rn(__fadd_rn((float)j, a), (float)n);
    const float s = proposal_inverse(c, u);
    return __fadd_rn(tmin, __fmul_rn(__fsub_rn(tmax, tmin), s));
}

}  // namespace neat
