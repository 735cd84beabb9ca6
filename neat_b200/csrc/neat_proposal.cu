// neat_proposal.cu -- learned sample proposal: per-segment CDFs for the
// step's sampler and the proposal's online training (cross-entropy against
// the binned contributions of a uniformly sampled step, Adam).
//
// Training kernel: one warp takes 32 segments at a time (one per lane), runs
// the MLP forward and backward per lane, stages activations and gradients of
// the 32 segments in shared memory and accumulates the weight gradients with
// lane j owning hidden unit j (dW1 row j, dW2 row j, dW3 column j): no
// atomics, per-block partials reduced in a fixed order.
#include <algorithm>

#include "neat_internal.h"
#include "neat_proposal.cuh"
#include "neat_tiles.cuh"

namespace neat
{

// Node descriptor from the method's own density: the decoded density of the
// node on a 4^3 lattice at local coordinates (i + 0.5) / 2 - 1, reduced to
// [density-weighted centroid (3), spread = RMS distance from it, log mean,
// log peak / mean].  One 64-thread block per node, one lattice point per thread.
template <int C>
__global__ void __launch_bounds__(64) k_node_desc(const float* __restrict__ grid, int64_t A, int G,
                                                  const float* __restrict__ dec, float beta, float* __restrict__ node_desc)
{
    using O = DecOff<C>;
    __shared__ float sW1[HH * C], sb1[HH], sW2[HH * HH], sb2[HH], sw3[HH];
    __shared__ float red[6][64];
    const int t = threadIdx.x;
    for (int i = t; i < HH * C; i += 64) sW1[i] = dec[O::W1 + i];
    for (int i = t; i < HH * HH; i += 64) sW2[i] = dec[O::W2 + i];
    sb1[t] = dec[O::b1 + t];
    sb2[t] = dec[O::b2 + t];
    sw3[t] = dec[O::W3 + t];
    const float b3 = dec[O::b3];
    __syncthreads();
    const float lx = (float)(t & 3) * 0.5f - 0.75f, ly = (float)((t >> 2) & 3) * 0.5f - 0.75f,
                lz = (float)(t >> 4) * 0.5f - 0.75f;
    for (int64_t node = blockIdx.x; node < A; node += gridDim.x)
    {
        Corners kc;
        igs_corners(lx, ly, lz, G, G, G, kc);
        float x[C];
        gather_cl<C>(grid, node, G, kc, x);
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
        const float rho = softplusf_(y, beta);
        red[0][t] = rho;
        red[1][t] = rho * lx;
        red[2][t] = rho * ly;
        red[3][t] = rho * lz;
        red[4][t] = rho * (lx * lx + ly * ly + lz * lz);
        red[5][t] = rho;
        __syncthreads();
        for (int o = 32; o > 0; o >>= 1)
        {
            if (t < o)
            {
#pragma unroll
                for (int q = 0; q < 5; ++q) red[q][t] += red[q][t + o];
                red[5][t] = fmaxf(red[5][t], red[5][t + o]);
            }
            __syncthreads();
        }
        if (t == 0)
        {
            const float S = red[0][0], mean = S * (1.0f / 64.0f);
            float cx = 0.0f, cy = 0.0f, cz = 0.0f, spread = 0.968246f;  // uniform lattice spread
            if (S > 1e-12f)
            {
                cx           = red[1][0] / S;
                cy           = red[2][0] / S;
                cz           = red[3][0] / S;
                const float v = red[4][0] / S - (cx * cx + cy * cy + cz * cz);
                spread        = sqrtf(fmaxf(v, 0.0f));
            }
            float* dst = node_desc + 6 * node;
            dst[0]     = cx;
            dst[1]     = cy;
            dst[2]     = cz;
            dst[3]     = spread;
            dst[4]     = logf(mean + 1e-3f);
            dst[5]     = logf((red[5][0] + 1e-3f) / (mean + 1e-3f));
        }
        __syncthreads();
    }
}

cudaError_t launch_node_desc(const float* grid, int64_t A, int C, int G, const float* decoder, float beta,
                             float* node_desc, cudaStream_t st)
{
    const int nb = (int)std::min<int64_t>(A, (int64_t)sm_count() * 16);
    switch (C)
    {
        case 4: k_node_desc<4><<<nb, 64, 0, st>>>(grid, A, G, decoder, beta, node_desc); break;
        case 8: k_node_desc<8><<<nb, 64, 0, st>>>(grid, A, G, decoder, beta, node_desc); break;
        case 16: k_node_desc<16><<<nb, 64, 0, st>>>(grid, A, G, decoder, beta, node_desc); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// The count head's sample count for a segment: its record's n (and the step
// between uniform samples, kept consistent) and its seg_n entry.
__device__ __forceinline__ void set_count(SegRec& r, int& sn, float v, float eps, int nmin)
{
    const int n = proposal_count(v, r.n, eps, nmin);
    r.n         = n;
    r.step      = __fdiv_rn(__fsub_rn(r.tmax, r.tmin), (float)n);
    sn          = n;
}

// Per node-major segment: the proposal's CDF bin ends and, when
// count_eps > 0, the segment's sample count from the count head (written to
// the segment record and to seg_n, ahead of the sample-offset scan).
__global__ void k_proposal_cdf(SegRec* __restrict__ segs, int* __restrict__ seg_n, const int64_t* counters,
                               const float* __restrict__ params, const float* __restrict__ node_desc, float mix,
                               float count_eps, int count_min, float* __restrict__ seg_cdf)
{
    __shared__ float P[PropOff::total];
    for (int i = threadIdx.x; i < PropOff::total; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int64_t n = counters[0];
    // two segments a thread (i and i + stride) per iteration, packed f32x2
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 2 * stride)
    {
        const int64_t i1 = i + stride;
        const bool two   = i1 < n;
        float f0[PIN], f1[PIN], p0[PBIN], p1[PBIN], c[PBIN], v0, v1;
        proposal_features(segs[i], node_desc, f0);
        proposal_features(segs[two ? i1 : i], node_desc, f1);
        proposal_forward2(P, f0, f1, mix, p0, p1, v0, v1);
        proposal_cdf(p0, c);
        float4* dst = reinterpret_cast<float4*>(seg_cdf + 8 * i);
        dst[0]      = make_float4(c[0], c[1], c[2], c[3]);
        dst[1]      = make_float4(c[4], c[5], c[6], c[7]);
        if (count_eps > 0.0f) set_count(segs[i], seg_n[i], v0, count_eps, count_min);
        if (two)
        {
            proposal_cdf(p1, c);
            dst    = reinterpret_cast<float4*>(seg_cdf + 8 * i1);
            dst[0] = make_float4(c[0], c[1], c[2], c[3]);
            dst[1] = make_float4(c[4], c[5], c[6], c[7]);
            if (count_eps > 0.0f) set_count(segs[i1], seg_n[i1], v1, count_eps, count_min);
        }
    }
}

cudaError_t launch_proposal_cdf(SegRec* segs, int* seg_n, const int64_t* counters, const neat_proposal* pr,
                                float* seg_cdf, cudaStream_t st)
{
    k_proposal_cdf<<<sm_count() * 4, 128, 0, st>>>(segs, seg_n, counters, pr->params, pr->node_desc, pr->mix,
                                                    pr->count_eps, pr->count_min, seg_cdf);
    return cudaGetLastError();
}

constexpr int PT_WARPS  = 4;
constexpr int PT_MAXSEG = 65536;  // segments per training iteration (a strided subset)
constexpr int SF        = PIN + 1;   // padded row strides of the per-warp staging (no bank conflicts)
constexpr int SH        = PH + 1;
constexpr int SB        = PBIN + 1;
constexpr int PT_STAGE  = 32 * (SF + 4 * SH + SB);  // floats staged per warp
// gradient, then: cross-entropy sum, total variation weight, target entropy sum,
// count-head squared error sum, count-head segments
constexpr int PT_PARTS  = PropOff::total + 5;
// the count head learns at this multiple of the proposal's learning rate (a
// linear regression on the trunk's features, it has to follow the trunk and
// the method's changing density within a few TRAIN steps)
constexpr float HEAD_LR_SCALE = 10.0f;

int proposal_grad_blocks() { return sm_count() * 2; }

// One iteration's gradient partials of the weighted cross-entropy between the
// proposal and the variation targets (each segment weighs by its total
// variation, so empty or flat space does not drown the segments that decide
// the quadrature error): part[block][0 .. total) gradient sums, [total]
// weighted cross-entropy sum, [total + 1] total weight, [total + 2] weighted
// sum of the targets' entropies (cross-entropy - entropy = KL to the targets),
// [total + 3] the count head's sum of (v - y)^2 / 2 over the segments, y =
// log(a + 1e-4) with a from k_seg_variation, and [total + 4] their number.
// The count head's gradient (rows VW .. total) stops at the trunk's features.
__global__ void __launch_bounds__(32 * PT_WARPS) k_prop_grad(const SegRec* __restrict__ segs, const int64_t* counters,
                                                               const float* __restrict__ seg_hist,
                                                               const float* __restrict__ seg_tv,
                                                               const float* __restrict__ params,
                                                               const float* __restrict__ node_desc, float mix, int it,
                                                               float* __restrict__ part)
{
    extern __shared__ float psm[];
    float* P     = psm;                 // parameters
    float* stage = P + PropOff::total;  // [warp][...]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < PropOff::total; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    float* sf   = stage + w * PT_STAGE;  // [32][SF] inputs
    float* sh1  = sf + 32 * SF;          // [32][SH] h1
    float* sh2  = sh1 + 32 * SH;         // [32][SH] h2
    float* sdz1 = sh2 + 32 * SH;         // [32][SH] silu'(z1), then dz1
    float* sdz2 = sdz1 + 32 * SH;        // [32][SH] silu'(z2), then dz2
    float* sdz3 = sdz2 + 32 * SH;        // [32][SB]
    float* mf   = sf + lane * SF;        // this lane's rows
    float* mh1  = sh1 + lane * SH;
    float* mh2  = sh2 + lane * SH;
    float* md1  = sdz1 + lane * SH;
    float* md2  = sdz2 + lane * SH;

    // accumulators owned by this lane (hidden unit j = lane)
    float gW1[PIN - 1] = {}, gb1 = 0.0f, gW2[PH] = {}, gb2 = 0.0f, gW3[PBIN] = {}, gb3 = 0.0f;
    float gWv = 0.0f, gUv = 0.0f, gbv = 0.0f;  // count head: Wv[lane], Uv[lane], bv (lane 0)
    float lsum = 0.0f, cnt = 0.0f, hsum = 0.0f, vsum = 0.0f, vcnt = 0.0f;

    const int64_t n      = counters[0];
    const int64_t stride = n > PT_MAXSEG ? (n + PT_MAXSEG - 1) / PT_MAXSEG : 1;
    const int64_t off    = it % stride;
    const int64_t nsub   = n > off ? (n - off + stride - 1) / stride : 0;
    const int64_t nwarps = (int64_t)gridDim.x * PT_WARPS;
    for (int64_t base = ((int64_t)blockIdx.x * PT_WARPS + w) * 32; base < nsub; base += nwarps * 32)
    {
        const int64_t k = base + lane;
        float f[PIN], q[PBIN], mass = 0.0f, vy = 0.0f;
        bool use = false, valid = false;
#pragma unroll
        for (int i = 0; i < PIN; ++i) f[i] = 0.0f;
#pragma unroll
        for (int b = 0; b < PBIN; ++b) q[b] = 0.0f;
        if (k < nsub)
        {
            const SegRec r  = segs[k * stride + off];
            const float4 q0 = *reinterpret_cast<const float4*>(seg_hist + 8 * (int64_t)r.rm);
            const float4 q1 = *reinterpret_cast<const float4*>(seg_hist + 8 * (int64_t)r.rm + 4);
            q[0] = q0.x; q[1] = q0.y; q[2] = q0.z; q[3] = q0.w;
            q[4] = q1.x; q[5] = q1.y; q[6] = q1.z; q[7] = q1.w;
            // target: where the density changes along the segment -- bin b
            // gets |m_b - m_b-1| + |m_b+1 - m_b| of the binned masses m -- and
            // the segment weighs by its total variation (constant or linear
            // stretches are integrated exactly by the midpoint rule anyway)
            float v[PBIN], tv = 0.0f;
#pragma unroll
            for (int b = 0; b < PBIN; ++b) v[b] = 0.0f;
#pragma unroll
            for (int b = 1; b < PBIN; ++b)
            {
                const float dm = fabsf(q[b] - q[b - 1]);
                v[b] += dm;
                v[b - 1] += dm;
                tv += dm;
            }
            use            = tv > 1e-20f;
            const float sv = seg_tv[r.rm];  // the count head's target: log(a + 1e-4)
            valid          = sv >= 0.0f;
            vy             = logf(sv + 1e-4f);
            proposal_features(r, node_desc, f);
            if (use)
            {
                const float inv = 0.5f / tv;
#pragma unroll
                for (int b = 0; b < PBIN; ++b) q[b] = v[b] * inv;
                mass = tv;
            }
        }
#pragma unroll
        for (int i = 0; i < PIN; ++i) mf[i] = f[i];
        // forward: h1, h2 and the SiLU derivatives into this lane's rows
#pragma unroll 4
        for (int j = 0; j < PH; ++j)
        {
            float z = P[PropOff::b1 + j];
#pragma unroll
            for (int i = 0; i < PIN - 1; ++i) z = fmaf(P[PropOff::W1 + j * PIN + i], f[i], z);
            const float sg = prop_sigmoid(z);
            mh1[j]         = z * sg;
            md1[j]         = sg * (1.0f + z * (1.0f - sg));
        }
        float h1[PH];
#pragma unroll
        for (int j = 0; j < PH; ++j) h1[j] = mh1[j];
#pragma unroll 4
        for (int kk = 0; kk < PH; ++kk)
        {
            float z = P[PropOff::b2 + kk];
#pragma unroll
            for (int j = 0; j < PH; ++j) z = fmaf(P[PropOff::W2 + kk * PH + j], h1[j], z);
            const float sg = prop_sigmoid(z);
            mh2[kk]        = z * sg;
            md2[kk]        = sg * (1.0f + z * (1.0f - sg));
        }
        // count head on the trunk's h2 and the inputs: v, and dv = v - y
        {
            float vh = P[PropOff::VB];
#pragma unroll
            for (int i = 0; i < PIN; ++i) vh = fmaf(P[PropOff::VU + i], f[i], vh);
#pragma unroll 4
            for (int kk = 0; kk < PH; ++kk) vh = fmaf(P[PropOff::VW + kk], mh2[kk], vh);
            const float dv = valid ? vh - vy : 0.0f;
            if (valid)
            {
                vsum = fmaf(0.5f * dv, dv, vsum);
                vcnt += 1.0f;
            }
            sdz3[lane * SB + PBIN] = dv;
        }
        float sm[PBIN], mxz = -3.0e38f;
#pragma unroll
        for (int b = 0; b < PBIN; ++b) sm[b] = P[PropOff::b3 + b];
#pragma unroll 4
        for (int kk = 0; kk < PH; ++kk)
        {
            const float hv = mh2[kk];
#pragma unroll
            for (int b = 0; b < PBIN; ++b) sm[b] = fmaf(P[PropOff::W3 + b * PH + kk], hv, sm[b]);
        }
#pragma unroll
        for (int b = 0; b < PBIN; ++b) mxz = fmaxf(mxz, sm[b]);
        float ssum = 0.0f;
#pragma unroll
        for (int b = 0; b < PBIN; ++b)
        {
            sm[b] = __expf(sm[b] - mxz);
            ssum += sm[b];
        }
        float dz3[PBIN];
        {
            const float inv = 1.0f / ssum;
            float pg = 0.0f, ce = 0.0f, hq = 0.0f, g[PBIN];
#pragma unroll
            for (int b = 0; b < PBIN; ++b)
            {
                sm[b]         = sm[b] * inv;
                const float p = fmaf(1.0f - mix, sm[b], mix * (1.0f / PBIN));
                g[b]          = -q[b] / p;
                pg += sm[b] * g[b];
                ce -= q[b] * __logf(p);
                if (q[b] > 0.0f) hq -= q[b] * __logf(q[b]);
            }
#pragma unroll
            for (int b = 0; b < PBIN; ++b) dz3[b] = use ? mass * (1.0f - mix) * sm[b] * (g[b] - pg) : 0.0f;
            if (use)
            {
                lsum += mass * ce;
                hsum += mass * hq;
                cnt += mass;
            }
        }
#pragma unroll
        for (int b = 0; b < PBIN; ++b) sdz3[lane * SB + b] = dz3[b];
        // backward through the hidden layers (in place over the derivatives)
#pragma unroll 4
        for (int kk = 0; kk < PH; ++kk)
        {
            float d = 0.0f;
#pragma unroll
            for (int b = 0; b < PBIN; ++b) d = fmaf(P[PropOff::W3 + b * PH + kk], dz3[b], d);
            md2[kk] = d * md2[kk];
        }
        float dz2[PH];
#pragma unroll
        for (int kk = 0; kk < PH; ++kk) dz2[kk] = md2[kk];
#pragma unroll 4
        for (int j = 0; j < PH; ++j)
        {
            float d = 0.0f;
#pragma unroll
            for (int kk = 0; kk < PH; ++kk) d = fmaf(P[PropOff::W2 + kk * PH + j], dz2[kk], d);
            md1[j] = d * md1[j];
        }
        __syncwarp();
        // lane j accumulates hidden unit j over the warp's 32 segments
        for (int s2 = 0; s2 < 32; ++s2)
        {
            const float d1 = sdz1[s2 * SH + lane];
            const float d2 = sdz2[s2 * SH + lane];
            const float hh = sh2[s2 * SH + lane];
            gb1 += d1;
            gb2 += d2;
#pragma unroll
            for (int i = 0; i < PIN - 1; ++i) gW1[i] = fmaf(d1, sf[s2 * SF + i], gW1[i]);
#pragma unroll
            for (int j = 0; j < PH; ++j) gW2[j] = fmaf(d2, sh1[s2 * SH + j], gW2[j]);
#pragma unroll
            for (int b = 0; b < PBIN; ++b) gW3[b] = fmaf(sdz3[s2 * SB + b], hh, gW3[b]);
            if (lane < PBIN) gb3 += sdz3[s2 * SB + lane];
            const float dv = sdz3[s2 * SB + PBIN];
            gWv            = fmaf(dv, hh, gWv);
            if (lane < PIN) gUv = fmaf(dv, sf[s2 * SF + lane], gUv);
            gbv += dv;
        }
        __syncwarp();
    }
    // per-warp results -> block partial (fixed order over the warps)
    __syncthreads();  // the staging area becomes the reduction area
    float* red = stage;  // [warp][PT_PARTS]
    float* rw  = red + w * PT_PARTS;
    for (int i = lane; i < PT_PARTS; i += 32) rw[i] = 0.0f;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < PIN - 1; ++i) rw[PropOff::W1 + lane * PIN + i] = gW1[i];
    rw[PropOff::b1 + lane] = gb1;
#pragma unroll
    for (int j = 0; j < PH; ++j) rw[PropOff::W2 + lane * PH + j] = gW2[j];
    rw[PropOff::b2 + lane] = gb2;
#pragma unroll
    for (int b = 0; b < PBIN; ++b) rw[PropOff::W3 + b * PH + lane] = gW3[b];
    if (lane < PBIN) rw[PropOff::b3 + lane] = gb3;
    rw[PropOff::VW + lane] = gWv;
    if (lane < PIN) rw[PropOff::VU + lane] = gUv;
    if (lane == 0) rw[PropOff::VB] = gbv;
    float ls = lsum, cn = cnt, hs = hsum, vs = vsum, vc = vcnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        ls += __shfl_xor_sync(0xffffffffu, ls, o);
        cn += __shfl_xor_sync(0xffffffffu, cn, o);
        hs += __shfl_xor_sync(0xffffffffu, hs, o);
        vs += __shfl_xor_sync(0xffffffffu, vs, o);
        vc += __shfl_xor_sync(0xffffffffu, vc, o);
    }
    if (lane == 0)
    {
        rw[PropOff::total]     = ls;
        rw[PropOff::total + 1] = cn;
        rw[PropOff::total + 2] = hs;
        rw[PropOff::total + 3] = vs;
        rw[PropOff::total + 4] = vc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < PT_PARTS; i += blockDim.x)
    {
        float acc = 0.0f;
        for (int ww = 0; ww < PT_WARPS; ++ww) acc += red[ww * PT_PARTS + i];
        part[(int64_t)blockIdx.x * PT_PARTS + i] = acc;
    }
}

// Adam step number and bias corrections of the proposal (one thread).
__global__ void k_prop_begin(int* counter, float lr, float b1, float b2, float* scal)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int t  = *counter + 1;
    *counter     = t;
    const double bc1 = 1.0 - pow((double)b1, (double)t);
    const double bc2 = 1.0 - pow((double)b2, (double)t);
    scal[0]      = (float)((double)lr / bc1);
    scal[1]      = (float)sqrt(bc2);
}

// Reduce the block partials, normalise, Adam.  The trunk and placement head
// are normalised by the total variation weight, the count head by its number
// of segments (and steps HEAD_LR_SCALE times as far).  A block takes 32
// parameters (one per lane, so each partial row is read coalesced); its 8
// warps split the partial rows (warp w: rows w, w + 8, ..) and their sums are
// added in warp order: a fixed association, the same every call.  Every block
// forms the normalisers the same way.
constexpr int PA_WARPS = 8;
__global__ void __launch_bounds__(32 * PA_WARPS)
    k_prop_adam(const float* __restrict__ part, int nblocks, const float* __restrict__ scal, neat_proposal pr)
{
    constexpr int NS = 5;                 // cross-entropy, weight, target entropy, head error, head count
    __shared__ float red[PA_WARPS][32 + NS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i    = blockIdx.x * 32 + lane;
    float g = 0.0f, x[NS] = {};
    for (int b = w; b < nblocks; b += PA_WARPS)
    {
        const float* pb = part + (int64_t)b * PT_PARTS;
        if (i < PropOff::total) g += pb[i];
        if (lane == 0)
        {
#pragma unroll
            for (int q = 0; q < NS; ++q) x[q] += pb[PropOff::total + q];
        }
    }
    red[w][lane] = g;
    if (lane == 0)
    {
#pragma unroll
        for (int q = 0; q < NS; ++q) red[w][32 + q] = x[q];
    }
    __syncthreads();
    if (w != 0 || i >= PropOff::total) return;
    g = 0.0f;
#pragma unroll
    for (int q = 0; q < NS; ++q) x[q] = 0.0f;
#pragma unroll
    for (int k = 0; k < PA_WARPS; ++k)
    {
        g += red[k][lane];
#pragma unroll
        for (int q = 0; q < NS; ++q) x[q] += red[k][32 + q];
    }
    const float ls = x[0], cnt = x[1], hs = x[2], vs = x[3], vc = x[4];
    const bool head = i >= PropOff::VW;
    const float nrm = head ? vc : cnt;
    g               = nrm > 0.0f ? g / nrm : 0.0f;
    pr.grad[i]      = g;
    if (i == 0 && pr.loss)
    {
        pr.loss[0] = cnt > 0.0f ? ls / cnt : 0.0f;
        pr.loss[1] = cnt > 0.0f ? hs / cnt : 0.0f;
        pr.loss[2] = vc > 0.0f ? vs / vc : 0.0f;
    }
    float m = pr.m[i], v = pr.v[i];
    m       = fmaf(1.0f - pr.beta1, g, m * pr.beta1);
    v       = fmaf((1.0f - pr.beta2) * g, g, v * pr.beta2);
    pr.m[i] = m;
    pr.v[i] = v;
    const float lr = head ? HEAD_LR_SCALE * scal[0] : scal[0];
    pr.params[i]   = fmaf(-lr, m / (sqrtf(v) / scal[1] + pr.eps), pr.params[i]);
}

// One thread a node-major segment: a = (tmax - tmin) sum_j |rho_j - rho_j-1|
// over its consecutive samples.  The midpoint rule with n samples misses
// about a / (2 n) of the segment's integral at density jumps, so a is what
// the count head predicts (as log(a + 1e-4)).
__global__ void k_seg_variation(const SegRec* __restrict__ segs, const int* __restrict__ samp_off,
                                const int64_t* counters, const float* __restrict__ seg_dens, int64_t dens_cap,
                                float* __restrict__ seg_tv)
{
    const int64_t n = counters[0];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const SegRec& r = segs[i];
        const int64_t o = samp_off[i];
        float tv        = -1.0f;
        if (o + r.n <= dens_cap)
        {
            tv          = 0.0f;
            float prev  = seg_dens[o];
            for (int j = 1; j < r.n; ++j)
            {
                const float x = seg_dens[o + j];
                tv += fabsf(x - prev);
                prev = x;
            }
            tv = (r.tmax - r.tmin) * tv;
        }
        seg_tv[r.rm] = tv;
    }
}

cudaError_t launch_seg_variation(const SegRec* segs, const int* samp_off, const int64_t* counters,
                                 const float* seg_dens, int64_t dens_cap, float* seg_tv, cudaStream_t st)
{
    k_seg_variation<<<sm_count() * 8, 128, 0, st>>>(segs, samp_off, counters, seg_dens, dens_cap, seg_tv);
    return cudaGetLastError();
}

cudaError_t launch_proposal_train(const SegRec* segs, const int64_t* counters, const float* seg_hist,
                                  const float* seg_tv, const neat_proposal* pr, float* part, int iters,
                                  cudaStream_t st)
{
    const int nb      = proposal_grad_blocks();
    static_assert(PT_STAGE >= PT_PARTS, "reduction area must fit the staging area of a warp");
    const size_t smem = (size_t)(PropOff::total + PT_WARPS * PT_STAGE) * 4;
    static bool init  = false;
    if (!init)
    {
        cudaFuncSetAttribute(k_prop_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        init = true;
    }
    float* scal = part + (size_t)nb * PT_PARTS;
    for (int it = 0; it < iters; ++it)
    {
        k_prop_grad<<<nb, 32 * PT_WARPS, smem, st>>>(segs, counters, seg_hist, seg_tv, pr->params, pr->node_desc,
                                                     pr->mix, it, part);
        k_prop_begin<<<1, 32, 0, st>>>(pr->step_counter, pr->lr, pr->beta1, pr->beta2, scal);
        k_prop_adam<<<(PropOff::total + 31) / 32, 32 * PA_WARPS, 0, st>>>(part, nb, scal, *pr);
    }
    return cudaGetLastError();
}

size_t proposal_part_floats() { return (size_t)proposal_grad_blocks() * PT_PARTS + 4; }

}  // namespace neat

extern "C" int64_t neat_proposal_params(void) { return neat::PropOff::total; }
