// neat_step.cu -- one fused training step of the NeAT forward projector:
// Trainer::TrainStep (samples/reconstruct.cpp:362-403) without per-sample
// tensors in HBM.
//
// Data flow (all on one stream, no host synchronisation):
//   1 rays+counts   warp/ray: f64 camera ray, slab test vs all active nodes
//   2 scans         per-ray segment offsets, per-node bucket offsets
//   3 segments      warp/ray: canonical (tmin,node) lists, bucketed by node
//   4 scan          node-major sample offsets; tile -> first segment table
//   5 forward       128-sample tiles in node-major order: jitter, position,
//                   local coords, IGS, decoder, softplus, weight, per-segment
//                   sums (a segment spans <= 2 tiles: two commutative adds)
//   6 loss          per ray: sum of its segments in tmin order, MSE, dL/dpred
//   7 backward      same tiles: recompute, decoder backward, grid scatter
//   8 Adam          decoder (deterministic reduce of per-CTA partials), grid
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "neat_internal.h"
#include "neat_scan.cuh"
#include "neat_slots.cuh"
#include "neat_tiles.cuh"

namespace neat
{


template <int C, bool BWD>
__global__ void __launch_bounds__(TN, 1) k_step_tiles(StepTileArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    TileSmem<C, BWD>& sm = *reinterpret_cast<TileSmem<C, BWD>*>(smraw);
    const int t          = threadIdx.x;
    tile_load_decoder<C, BWD>(sm, a.decoder);
    DecGradAcc<C> g;
    g.zero();
    const int nseg       = (int)a.counters[0];
    const int64_t S      = a.counters[1];
    const int64_t ntiles = (S + TT - 1) / TT;
    __syncthreads();
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int64_t g0 = tile * TT;
        const int seg_lo = a.tile_seg[tile];
        // ---- slot -> segment: mark segment starts, inclusive max-scan ----
        if (t < TT) sm.mark[t] = (t == 0) ? seg_lo : -1;
        __syncthreads();
        if (t <= TT)
        {
            const int seg = seg_lo + t;
            if (seg < nseg)
            {
                const int64_t o = a.samp_off[seg];
                if (o > g0 && o < g0 + TT) sm.mark[(int)(o - g0)] = seg;
            }
        }
        __syncthreads();
        if (t < TT)
        {
            int v = sm.mark[t];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if ((t & 31) >= o) v = max(v, y);
            }
            sm.slot_seg[t] = v;
        }
        __syncthreads();
        if (t < TT)
        {
            int v = sm.slot_seg[t];
            for (int w2 = 0; w2 < (t >> 5); ++w2) v = max(v, sm.slot_seg[w2 * 32 + 31]);
            sm.mark[t] = v;  // final segment of slot t
        }
        __syncthreads();
        // ---- per-slot sample setup + grid gather ----
        bool valid = false;
        float wgt = 0.0f, lu = 0.0f, lv = 0.0f, lw = 0.0f;
        int ray = 0, rm = 0, row = 0;
        if (t < TT)
        {
            const int64_t gs = g0 + t;
            valid            = gs < S;
            const int seg    = sm.mark[t];
            const SegRec r   = a.segs[seg];
            const SlotSample q =
                slot_sample(r, valid ? (int)(gs - a.samp_off[seg]) : 0, valid, a.jitter != 0, a.seed,
                            a.step_dev ? (uint32_t)*a.step_dev : a.step);
            lu = q.lu;
            lv = q.lv;
            lw = q.lw;
            Corners k;
            igs_corners(lu, lv, lw, a.G, a.G, a.G, k);
            float x[C];
            gather_cl<C>(a.grid, r.row, a.G, k, x);
#pragma unroll
            for (int c = 0; c < C; ++c) sm.XT[c * TT + t] = valid ? x[c] : 0.0f;
            wgt = q.weight;
            ray = r.ray;
            rm  = r.rm;
            row = r.row;
        }
        __syncthreads();
        // ---- decoder forward ----
        tile_layer1<C, BWD>(sm);
        __syncthreads();
        float z2[4][HPW];
        tile_gemm_fwd<C, BWD>(sm, z2);
        tile_ypart<C, BWD>(sm, z2);
        __syncthreads();
        if (t < TT)
        {
            const float y = tile_y(sm, t);
            if (!BWD)
            {
                sm.val[t] = valid ? softplusf_(y, a.beta) * wgt : 0.0f;
            }
            else
            {
                const float dv = valid ? a.dpred[ray] : 0.0f;
                const float dy = dv * wgt * softplus_grad(y, a.beta);
                sm.val[t]      = dy;
                g.db3 += dy;
            }
        }
        __syncthreads();
        if constexpr (!BWD)
        {
            // per-segment sums, in f64 so that the split of a segment across
            // two tiles (which follows the node-bucket order) does not change
            // the result; at most two adds onto a zeroed slot
            if (t < TT && valid)
            {
                const int seg = sm.mark[t];
                if (t == 0 || sm.mark[t - 1] != seg)
                {
                    double sum = 0.0;
                    for (int u = t; u < TT && sm.mark[u] == seg; ++u) sum += (double)sm.val[u];
                    atomicAdd(a.partial + rm, sum);
                }
            }
            __syncthreads();
        }
        else
        {
            float dx[C];
            tile_backward<C>(sm, z2, g, dx);
            if (t < TT && valid)
            {
                Corners k;
                igs_corners(lu, lv, lw, a.G, a.G, a.G, k);
                scatter_cl<C>(a.grid_grad, row, a.G, k, dx);
            }
            __syncthreads();
        }
    }
    if constexpr (BWD) dec_grad_flush<C>(g, a.dec_part + (int64_t)blockIdx.x * DecOff<C>::total, false, sm.ypart);
}

// Zero n = counters[0] * per floats.
__global__ void k_zero_per_segment(float* __restrict__ p, const int64_t* counters, int per)
{
    const int64_t n = counters[0] * per;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0.0f;
}

// Also the samples' capacity check: more samples than sample_cap and the step
// processes nothing (counters[1] = 0); counters[3] = the step's tiles.
__global__ void k_tile_seg(const int* __restrict__ samp_off, const int* __restrict__ seg_n, int64_t* counters,
                           int* __restrict__ tile_seg, int64_t tiles_cap, int64_t sample_cap, int* status)
{
    const int64_t nseg = counters[0];
    const int64_t s0   = counters[1];
    const bool over    = s0 > sample_cap;
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        if (over)
        {
            raise_status(status, NEAT_ERR_CAPACITY);
            counters[1] = 0;
        }
        counters[3] = over ? 0 : (s0 + TT - 1) / TT;
    }
    if (over || s0 == 0) return;
    // grid-stride over the step's segments (the grid is sized for the SMs, not
    // for the segment capacity, most of which a step leaves unused)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t o = samp_off[i], e = o + seg_n[i];
        const int64_t t = (o + TT - 1) / TT;
        if (t * TT < e && t < tiles_cap) tile_seg[t] = (int)i;
    }
}

// Photometric calibration of one ray's integral x (PhotometricCalibration::forward,
// src/modules/ToneMapper.cpp:188-217): returns y and, given dL/dy, accumulates
// the parameter gradients and returns dL/dx.
struct ToneMap
{
    neat_tonemap t;
    const float* uv;
    const int32_t* image_id;
};

__device__ __forceinline__ int tm_off_bias(const neat_tonemap& t) { return 2 * t.num_images; }
__device__ __forceinline__ int tm_off_resp(const neat_tonemap& t) { return 2 * t.num_images + t.bias_w * t.bias_h; }

// Where the forward of one ray landed: what its backward needs.
struct TmPoint
{
    float ef = 1.0f;                  // exposure factor
    int bx0 = 0, bx1 = 0, by0 = 0, by1 = 0;
    float wx = 0.0f, wy = 0.0f;       // sensor-bias bilinear weights
    float slope = 1.0f;               // d response / d input
    int r0      = 0;
    float rf    = 0.0f;               // response segment and its fraction
};

// Forward of the calibration for ray r with integral x (the enabled parts in
// the reference's order: exposure, sensor bias, response).
__device__ __forceinline__ float tonemap_forward(const ToneMap& tm, int64_t r, float x, TmPoint& q)
{
    const neat_tonemap& T = tm.t;
    const int img         = tm.image_id[r];
    float y               = x;
    if (T.exposure)
    {
        if (T.exposure_mult) q.ef = T.params[img];
        y = y * q.ef + T.params[T.num_images + img];
    }
    if (T.sensor_bias)
    {
        // grid_sample, align_corners false, border: ix = u W - 0.5 clamped to [0, W-1]
        const float* sb = T.params + tm_off_bias(T);
        float ix = fminf(fmaxf(tm.uv[2 * r] * (float)T.bias_w - 0.5f, 0.0f), (float)(T.bias_w - 1));
        float iy = fminf(fmaxf(tm.uv[2 * r + 1] * (float)T.bias_h - 0.5f, 0.0f), (float)(T.bias_h - 1));
        q.bx0    = (int)floorf(ix);
        q.by0    = (int)floorf(iy);
        q.bx1    = min(q.bx0 + 1, T.bias_w - 1);
        q.by1    = min(q.by0 + 1, T.bias_h - 1);
        q.wx     = ix - (float)q.bx0;
        q.wy     = iy - (float)q.by0;
        y += (1.0f - q.wy) * ((1.0f - q.wx) * sb[q.by0 * T.bias_w + q.bx0] + q.wx * sb[q.by0 * T.bias_w + q.bx1]) +
             q.wy * ((1.0f - q.wx) * sb[q.by1 * T.bias_w + q.bx0] + q.wx * sb[q.by1 * T.bias_w + q.bx1]);
    }
    if (T.response)
    {
        // x / range * (P-1), clamped (border), linear interpolation; leak above range
        const float* rp = T.params + tm_off_resp(T);
        const float ix  = fminf(fmaxf(y / T.response_range * (float)(NEAT_RESPONSE_PARAMS - 1), 0.0f),
                                (float)(NEAT_RESPONSE_PARAMS - 1));
        q.r0            = min((int)floorf(ix), NEAT_RESPONSE_PARAMS - 2);
        q.rf            = ix - (float)q.r0;
        const float in_range = (y > 0.0f && y < T.response_range) ? 1.0f : 0.0f;
        const float leak     = y > T.response_range ? y - T.response_range : 0.0f;
        q.slope = in_range * (rp[q.r0 + 1] - rp[q.r0]) * ((float)(NEAT_RESPONSE_PARAMS - 1) / T.response_range) +
                  (y > T.response_range ? 1.0f : 0.0f);
        y = (1.0f - q.rf) * rp[q.r0] + q.rf * rp[q.r0 + 1] + leak;
    }
    return y;
}

__global__ void k_ray_loss(int64_t R, const int* __restrict__ ray_seg_off, const double* __restrict__ partial,
                           const float* __restrict__ target, float* __restrict__ dpred, float* __restrict__ pred_out,
                           float* __restrict__ loss_part, float invR, const int64_t* nseg_eff, ToneMap tm)
{
    __shared__ float red[256];
    __shared__ float gresp[NEAT_RESPONSE_PARAMS];
    const neat_tonemap& T = tm.t;
    const bool on         = T.params != nullptr;
    if (on && T.response)
        for (int i = threadIdx.x; i < NEAT_RESPONSE_PARAMS; i += blockDim.x) gresp[i] = 0.0f;
    if (on) __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float sq        = 0.0f;
    if (r < R)
    {
        float pred = 0.0f;
        if (*nseg_eff > 0)
        {
            const int b = ray_seg_off[r], e = ray_seg_off[r + 1];
            double acc  = 0.0;
            for (int k = b; k < e; ++k) acc += partial[k];
            pred = (float)acc;
        }
        if (!on)
        {
            const float diff = pred - target[r];
            dpred[r]         = 2.0f * diff * invR;
            sq               = diff * diff;
            if (pred_out) pred_out[r] = pred;
        }
        else
        {
            // forward
            const int img = tm.image_id[r];
            TmPoint q;
            const float y = tonemap_forward(tm, r, pred, q);
            const float ef = q.ef, wx = q.wx, wy = q.wy, slope = q.slope, rf = q.rf;
            const int bx0 = q.bx0, bx1 = q.bx1, by0 = q.by0, by1 = q.by1, r0 = q.r0;
            const float diff = y - target[r];
            const float dy   = 2.0f * diff * invR;
            sq               = diff * diff;
            if (pred_out) pred_out[r] = y;
            // backward
            if (T.response)
            {
                atomicAdd(&gresp[r0], dy * (1.0f - rf));
                atomicAdd(&gresp[r0 + 1], dy * rf);
            }
            const float d2 = dy * slope;  // dL / d(exposed + bias)
            if (T.sensor_bias)
            {
                float* g = T.grad + tm_off_bias(T);
                atomicAdd(&g[by0 * T.bias_w + bx0], d2 * (1.0f - wy) * (1.0f - wx));
                atomicAdd(&g[by0 * T.bias_w + bx1], d2 * (1.0f - wy) * wx);
                atomicAdd(&g[by1 * T.bias_w + bx0], d2 * wy * (1.0f - wx));
                atomicAdd(&g[by1 * T.bias_w + bx1], d2 * wy * wx);
            }
            if (T.exposure)
            {
                atomicAdd(&T.grad[T.num_images + img], d2);
                if (T.exposure_mult) atomicAdd(&T.grad[img], d2 * pred);
            }
            dpred[r] = d2 * ef;
        }
    }
    if (on && T.response)
    {
        __syncthreads();
        for (int i = threadIdx.x; i < NEAT_RESPONSE_PARAMS; i += blockDim.x)
            atomicAdd(&T.grad[tm_off_resp(T) + i], gresp[i]);
    }
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1)
    {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

__global__ void k_loss_final(const float* __restrict__ loss_part, int nb, float* loss, float invR)
{
    __shared__ float red[1024];
    float s = 0.0f;
    for (int i = threadIdx.x; i < nb; i += 1024) s += loss_part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1)
    {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] * invR;
}

// torch::optim::Adam::step (libtorch 1.11): m = b1 m + (1-b1) g;
// v = b2 v + (1-b2) g^2; p -= (lr/bc1) * m / (sqrt(v)/sqrt(bc2) + eps).
__device__ __forceinline__ void adam_update(float& p, float gr, float& m, float& v, float b1, float b2, float eps,
                                            float step_size, float sqrt_bc2)
{
    m                 = fmaf(1.0f - b1, gr, m * b1);
    v                 = fmaf((1.0f - b2) * gr, gr, v * b2);
    const float denom = sqrtf(v) / sqrt_bc2 + eps;
    p                 = fmaf(-step_size, m / denom, p);
}

// Per-step scalars written on the device at the start of the step: the step
// number (host argument or device counter) and Adam's bias-corrected step
// sizes, computed in double as torch::optim::Adam does.
struct StepScalars
{
    int step;
    float grid_step_size;  // lr_grid / (1 - beta1^t)
    float dec_step_size;   // lr_decoder / (1 - beta1^t)
    float sqrt_bc2;        // sqrt(1 - beta2^t)
};

__global__ void k_step_begin(int* counter, int host_step, double lr_grid, double lr_dec, double b1, double b2,
                             StepScalars* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int t = host_step;
    if (counter)
    {
        t        = *counter + 1;
        *counter = t;
    }
    const double bc1    = 1.0 - pow(b1, (double)t);
    const double bc2    = 1.0 - pow(b2, (double)t);
    out->step           = t;
    out->grid_step_size = (float)(lr_grid / bc1);
    out->dec_step_size  = (float)(lr_dec / bc1);
    out->sqrt_bc2       = (float)sqrt(bc2);
}

// CameraResponseNet::ParamLoss (src/modules/ToneMapper.cpp:100-119): with
// f = P sqrt(1e-5), L = f^2 [r_0^2 + sum_{i=1..P-2} (r_i - (r_{i-1} + r_{i+1}) / 2)^2];
// its gradient joins the response's; then SGD per group and the bias clamps
// (ApplyConstraints), gradients zeroed.
__global__ void k_tonemap_update(neat_tonemap T)
{
    const int P      = NEAT_RESPONSE_PARAMS;
    const int n_all  = 2 * T.num_images + T.bias_w * T.bias_h + P;
    const int ro     = 2 * T.num_images + T.bias_w * T.bias_h;
    const float ff   = (float)P * P * 1e-5f;  // f^2
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_all; i += gridDim.x * blockDim.x)
    {
        float g = T.grad[i], lr = 0.0f;
        bool clamp0 = false;
        if (i < T.num_images)
            lr = (T.exposure && T.exposure_mult) ? T.lr_exposure : 0.0f;
        else if (i < 2 * T.num_images)
        {
            lr     = T.exposure ? T.lr_exposure : 0.0f;
            clamp0 = true;
        }
        else if (i < ro)
        {
            lr     = T.sensor_bias ? T.lr_sensor_bias : 0.0f;
            clamp0 = true;
        }
        else if (T.response)
        {
            lr           = T.lr_response;
            const int k  = i - ro;
            const float* r = T.params + ro;
            auto e = [&](int j) { return r[j] - 0.5f * (r[j - 1] + r[j + 1]); };  // 1 <= j <= P-2
            float gl = 0.0f;
            if (k == 0) gl += 2.0f * r[0];
            if (k >= 1 && k <= P - 2) gl += 2.0f * e(k);
            if (k - 1 >= 1 && k - 1 <= P - 2) gl -= e(k - 1);
            if (k + 1 >= 1 && k + 1 <= P - 2) gl -= e(k + 1);
            g += ff * gl;
        }
        float v = T.params[i] - lr * g;
        if (clamp0) v = fmaxf(v, 0.0f);
        T.params[i] = v;
        T.grad[i]   = 0.0f;
    }
}

__global__ void k_tonemap_param_loss(neat_tonemap T)
{
    if (threadIdx.x != 0 || blockIdx.x != 0 || !T.param_loss) return;
    const int P    = NEAT_RESPONSE_PARAMS;
    const float* r = T.params + 2 * T.num_images + T.bias_w * T.bias_h;
    float l        = 0.0f;
    if (T.response)
    {
        l = r[0] * r[0];
        for (int j = 1; j <= P - 2; ++j)
        {
            const float e = r[j] - 0.5f * (r[j - 1] + r[j + 1]);
            l += e * e;
        }
        l *= (float)P * P * 1e-5f;
    }
    *T.param_loss = l;
}

// Decoder gradient: the sum of the CTA partials (rows of part), then Adam.  A
// block takes 32 parameters; its warp g sums rows g, g + 8, g + 16, .. (each
// warp reads 128 contiguous bytes of a row), and the 8 warp sums are added in
// warp order: a fixed order, so the gradient is reproducible, and ~150
// blocks instead of one thread a parameter walking all rows.
constexpr int DEC_RED_GROUPS = 8;

__global__ void __launch_bounds__(32 * DEC_RED_GROUPS)
    k_dec_reduce_adam(const float* __restrict__ part, int nparts, int P, float* __restrict__ grad,
                      float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float b1, float b2,
                      float eps, const StepScalars* __restrict__ sc)
{
    __shared__ float red[DEC_RED_GROUPS][33];
    const int lx = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int i  = blockIdx.x * 32 + lx;
    float s      = 0.0f;
    if (i < P)
    {
#pragma unroll 4
        for (int b = g; b < nparts; b += DEC_RED_GROUPS) s += part[(int64_t)b * P + i];
    }
    red[g][lx] = s;
    __syncthreads();
    if (g != 0 || i >= P) return;
    const float step_size = sc->dec_step_size, sqrt_bc2 = sc->sqrt_bc2;
    float gsum = red[0][lx];
#pragma unroll
    for (int k = 1; k < DEC_RED_GROUPS; ++k) gsum += red[k][lx];
    grad[i] = gsum;
    float pi = p[i], mi = m[i], vi = v[i];
    adam_update(pi, gsum, mi, vi, b1, b2, eps, step_size, sqrt_bc2);
    p[i] = pi;
    m[i] = mi;
    v[i] = vi;
}

__device__ __forceinline__ uint16_t bf16_rn(float x)
{
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&b);
}

// p_bf16 (optional): BF16 copy of the updated parameters, written alongside.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float b1, float b2, float eps, float step_size, float sqrt_bc2, int zero_grad,
                       const StepScalars* __restrict__ sc, uint16_t* __restrict__ p_bf16 = nullptr)
{
    if (sc)
    {
        step_size = sc->grid_step_size;
        sqrt_bc2  = sc->sqrt_bc2;
    }
    const int64_t n4     = n / 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride)
    {
        float4 pp = reinterpret_cast<float4*>(p)[i];
        float4 gg = reinterpret_cast<float4*>(grad)[i];
        float4 mm = reinterpret_cast<float4*>(m)[i];
        float4 vv = reinterpret_cast<float4*>(v)[i];
        adam_update(pp.x, gg.x, mm.x, vv.x, b1, b2, eps, step_size, sqrt_bc2);
        adam_update(pp.y, gg.y, mm.y, vv.y, b1, b2, eps, step_size, sqrt_bc2);
        adam_update(pp.z, gg.z, mm.z, vv.z, b1, b2, eps, step_size, sqrt_bc2);
        adam_update(pp.w, gg.w, mm.w, vv.w, b1, b2, eps, step_size, sqrt_bc2);
        reinterpret_cast<float4*>(p)[i] = pp;
        reinterpret_cast<float4*>(m)[i] = mm;
        reinterpret_cast<float4*>(v)[i] = vv;
        if (zero_grad) reinterpret_cast<float4*>(grad)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (p_bf16)
            reinterpret_cast<uint2*>(p_bf16)[i] =
                make_uint2((uint32_t)bf16_rn(pp.x) | ((uint32_t)bf16_rn(pp.y) << 16),
                           (uint32_t)bf16_rn(pp.z) | ((uint32_t)bf16_rn(pp.w) << 16));
    }
    for (int64_t i = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        float pi = p[i], mi = m[i], vi = v[i];
        adam_update(pi, grad[i], mi, vi, b1, b2, eps, step_size, sqrt_bc2);
        p[i] = pi;
        m[i] = mi;
        v[i] = vi;
        if (zero_grad) grad[i] = 0.0f;
        if (p_bf16) p_bf16[i] = bf16_rn(pi);
    }
}

int sm_count()
{
    static int n = 0;
    if (n == 0)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int resident_ctas(const void* kernel, int threads, size_t dyn_smem, int cap)
{
    int dev = 0;
    cudaGetDevice(&dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 1;
    int regs_sm = 0, smem_sm = 0, max_thr = 0, max_blocks = 0, reserved = 0;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&max_thr, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    cudaDeviceGetAttribute(&max_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    // registers are allocated per warp in units of 256
    const int warps     = (threads + 31) / 32;
    const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
    int n               = max_blocks > 0 ? max_blocks : 32;
    if (regs_warp > 0) n = std::min(n, regs_sm / (regs_warp * warps));
    const size_t smem_blk = fa.sharedSizeBytes + dyn_smem + (size_t)reserved;
    if (smem_blk > 0) n = std::min<int>(n, (int)(smem_sm / smem_blk));
    n = std::min(n, max_thr / (warps * 32));
    if (cap > 0) n = std::min(n, cap);
    return std::max(n, 1);
}

template <int C, bool BWD>
static int tile_grid(size_t& smem)
{
    smem = sizeof(TileSmem<C, BWD>);
    static int blocks = 0;
    if (blocks == 0)
    {
        cudaFuncSetAttribute(k_step_tiles<C, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        blocks = resident_ctas((const void*)k_step_tiles<C, BWD>, TN, smem, 0) * sm_count();
    }
    return blocks;
}

static int tile_grid_any(int C, bool bwd, size_t& smem)
{
    switch (C)
    {
        case 4: return bwd ? tile_grid<4, true>(smem) : tile_grid<4, false>(smem);
        case 8: return bwd ? tile_grid<8, true>(smem) : tile_grid<8, false>(smem);
        case 16: return bwd ? tile_grid<16, true>(smem) : tile_grid<16, false>(smem);
        default: return 0;
    }
}

int64_t decoder_params(int C) { return (int64_t)HH * C + HH + (int64_t)HH * HH + HH + HH + 1; }

// Workspace carve-out, shared by the size query and the step.
struct StepLayout
{
    enum
    {
        ORIGIN, DIRECTION, RAY_NSEG, RAY_SEG_OFF, NODE_NSEG, NODE_SEG_OFF, RAY_HITS, SEGS, SEG_N,
        SAMP_OFF, TILE_SEG, PARTIAL, DPRED, LOSS_PART, DEC_PART, SCAN_SCRATCH, SCAL, SEG_CDF, SEG_HIST,
        SEG_DENS, SEG_TV, PROP_PART, SEG_PGRAD, RAY_PGRAD, REC, NUM
    };
    size_t off[NUM];
    size_t total;
    int64_t tiles_cap, sample_cap, rec_cap, dens_cap;
    int loss_blocks, bwd_grid, cap_ray;
};

static size_t align256(size_t b) { return (b + 255) / 256 * 256; }

static bool step_layout(const neat_step_desc* d, int64_t R, StepLayout& L)
{
    const int64_t cap = d->seg_capacity, A = d->num_active, M = d->max_samples_per_node;
    L.cap_ray         = (int)std::max<int64_t>(1, std::min<int64_t>(NEAT_MAX_HITS_PER_RAY, R > 0 ? cap / R : 1));
    L.sample_cap      = cap * (M + 1);
    L.tiles_cap       = (L.sample_cap + TT - 1) / TT + 1;
    // per-sample records from the forward to the backward: room for 4 (M + 1)
    // samples per ray by default (a step with more recomputes them in the backward)
    const int64_t rec_per_ray = d->record_samples_per_ray == 0 ? (M + 1) * 4
                                : d->record_samples_per_ray < 0 ? 0
                                                                : d->record_samples_per_ray;
    L.rec_cap = std::min<int64_t>(L.sample_cap, std::max<int64_t>(R, 1) * rec_per_ray);
    // proposal TRAIN steps: the densities of up to 4 (M + 1) samples a ray (a
    // step with more trains the count head on the segments inside that room)
    L.dens_cap = d->proposal ? std::min<int64_t>(L.sample_cap, std::max<int64_t>(R, 1) * (M + 1) * 4) : 0;
    L.loss_blocks     = (int)((R + 255) / 256);
    size_t smem       = 0;
    L.bwd_grid        = d->decoder_path == NEAT_DECODER_SIMT_FP32
                            ? tile_grid_any(d->C, true, smem)
                            : tc_backward_grid(d->C, d->decoder_path == NEAT_DECODER_TC_BF16 ? 0 : 1);
    if (L.bwd_grid <= 0) return false;
    const int64_t P        = decoder_params(d->C);
    const int64_t scan_max = std::max(std::max(R, A), cap) + 1;
    size_t sz[] = {
        (size_t)R * 3 * 4, (size_t)R * 3 * 4, (size_t)R * 4, (size_t)(R + 1) * 4, (size_t)A * 4,
        (size_t)(A + 1) * 4, (size_t)R * L.cap_ray * sizeof(SegRec), (size_t)cap * sizeof(SegRec), (size_t)cap * 4,
        (size_t)(cap + 1) * 4,
        (size_t)L.tiles_cap * 4, (size_t)cap * 8, (size_t)R * 4, (size_t)L.loss_blocks * 4,
        (size_t)L.bwd_grid * P * 4, (size_t)scan_scratch_elems(scan_max) * 4, sizeof(StepScalars),
        d->proposal ? (size_t)cap * 8 * 4 : 0, d->proposal ? (size_t)cap * 8 * 4 : 0, (size_t)L.dens_cap * 4,
        d->proposal ? (size_t)cap * 4 : 0,
        d->proposal ? proposal_part_floats() * 4 : 0, d->pose_grad ? (size_t)cap * 6 * 4 : 0,
        d->pose_grad ? (size_t)R * 6 * 4 : 0,
        d->decoder_path != NEAT_DECODER_SIMT_FP32 ? (size_t)L.rec_cap * (8 + d->C) * 4 : 0};
    static_assert(sizeof(sz) / sizeof(sz[0]) == StepLayout::NUM, "one size per workspace buffer");
    size_t o = 0;
    for (int i = 0; i < StepLayout::NUM; ++i)
    {
        L.off[i] = o;
        o += align256(sz[i]);
    }
    L.total = o;
    return true;
}

template <int C>
static cudaError_t launch_tiles(bool bwd, const StepTileArgs& args, cudaStream_t st)
{
    size_t smem = 0;
    if (!bwd)
    {
        const int grid = tile_grid<C, false>(smem);
        k_step_tiles<C, false><<<grid, TN, smem, st>>>(args);
    }
    else
    {
        const int grid = tile_grid<C, true>(smem);
        k_step_tiles<C, true><<<grid, TN, smem, st>>>(args);
    }
    return cudaGetLastError();
}

static cudaError_t launch_tiles_any(int C, bool bwd, const StepTileArgs& args, cudaStream_t st)
{
    switch (C)
    {
        case 4: return launch_tiles<4>(bwd, args, st);
        case 8: return launch_tiles<8>(bwd, args, st);
        case 16: return launch_tiles<16>(bwd, args, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace neat

using namespace neat;

extern "C" int64_t neat_decoder_params(int C) { return decoder_params(C); }

extern "C" size_t neat_train_step_workspace_bytes(const neat_step_desc* desc, int64_t num_rays)
{
    if (!desc || num_rays < 0) return 0;
    StepLayout L;
    if (!step_layout(desc, num_rays, L)) return 0;
    return L.total;
}

extern "C" int neat_adam(float* param, float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, float lr, float beta1,
                         float beta2, float eps, int step, int zero_grad, neat_stream_t stream)
{
    if (n < 0 || step < 1) return NEAT_ERR_BAD_INPUT;
    if (n == 0) return NEAT_OK;
    if (!param || !grad || !exp_avg || !exp_avg_sq) return NEAT_ERR_BAD_INPUT;
    if (((uintptr_t)param | (uintptr_t)grad | (uintptr_t)exp_avg | (uintptr_t)exp_avg_sq) & 15)
        return NEAT_ERR_BAD_INPUT;
    const double bc1 = 1.0 - std::pow((double)beta1, step);
    const double bc2 = 1.0 - std::pow((double)beta2, step);
    const int grid   = std::min<int64_t>((n / 4 + 255) / 256 + 1, (int64_t)sm_count() * 8);
    k_adam<<<grid, 256, 0, (cudaStream_t)stream>>>(param, grad, exp_avg, exp_avg_sq, n, beta1, beta2, eps,
                                                   (float)(lr / bc1), (float)std::sqrt(bc2), zero_grad, nullptr);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

namespace neat
{

// Device pointers of the step workspace.
struct StepBufs
{
    float *origin, *direction;
    int *ray_nseg, *ray_seg_off, *node_nseg, *node_seg_off;
    SegRec *ray_hits, *segs;
    int *seg_n, *samp_off, *tile_seg;
    double* partial;
    float *dpred, *loss_part, *dec_part;
    int* scratch;
    StepScalars* scal;
    float *seg_cdf, *seg_hist, *seg_dens, *seg_tv, *prop_part;
    float *seg_pgrad, *ray_pgrad;
    float* rec;
};

static StepBufs step_bufs(const StepLayout& L, void* workspace)
{
    char* ws = (char*)workspace;
    auto P_  = [&](int i) { return (void*)(ws + L.off[i]); };
    StepBufs w;
    w.origin       = (float*)P_(StepLayout::ORIGIN);
    w.direction    = (float*)P_(StepLayout::DIRECTION);
    w.ray_nseg     = (int*)P_(StepLayout::RAY_NSEG);
    w.ray_seg_off  = (int*)P_(StepLayout::RAY_SEG_OFF);
    w.node_nseg    = (int*)P_(StepLayout::NODE_NSEG);
    w.node_seg_off = (int*)P_(StepLayout::NODE_SEG_OFF);
    w.ray_hits     = (SegRec*)P_(StepLayout::RAY_HITS);
    w.segs         = (SegRec*)P_(StepLayout::SEGS);
    w.seg_n        = (int*)P_(StepLayout::SEG_N);
    w.samp_off     = (int*)P_(StepLayout::SAMP_OFF);
    w.tile_seg     = (int*)P_(StepLayout::TILE_SEG);
    w.partial      = (double*)P_(StepLayout::PARTIAL);
    w.dpred        = (float*)P_(StepLayout::DPRED);
    w.loss_part    = (float*)P_(StepLayout::LOSS_PART);
    w.dec_part     = (float*)P_(StepLayout::DEC_PART);
    w.scratch      = (int*)P_(StepLayout::SCAN_SCRATCH);
    w.scal         = (StepScalars*)P_(StepLayout::SCAL);
    w.seg_cdf      = (float*)P_(StepLayout::SEG_CDF);
    w.seg_hist     = (float*)P_(StepLayout::SEG_HIST);
    w.seg_dens     = (float*)P_(StepLayout::SEG_DENS);
    w.seg_tv       = (float*)P_(StepLayout::SEG_TV);
    w.prop_part    = (float*)P_(StepLayout::PROP_PART);
    w.seg_pgrad    = (float*)P_(StepLayout::SEG_PGRAD);
    w.ray_pgrad    = (float*)P_(StepLayout::RAY_PGRAD);
    w.rec          = (float*)P_(StepLayout::REC);
    return w;
}

// Host-side checks shared by the step and the projection.
static int check_desc(const neat_step_desc* d, const neat_step_batch* b)
{
    if (d->C != 4 && d->C != 8 && d->C != 16) return NEAT_ERR_UNSUPPORTED;
    if (d->decoder_path != NEAT_DECODER_SIMT_FP32 && d->decoder_path != NEAT_DECODER_TC_BF16X3 &&
        d->decoder_path != NEAT_DECODER_TC_BF16)
        return NEAT_ERR_UNSUPPORTED;
    const int64_t R = b->num_rays;
    if (R < 1 || R > (1ll << 23) || d->num_active < 1 || d->max_depth < 1 || d->max_depth > kMaxDepth ||
        d->G < 2 || d->max_samples_per_node < 1 || d->seg_capacity < 1 || d->w < 2 || d->h < 2)
        return NEAT_ERR_BAD_INPUT;
    if (d->seg_capacity * (int64_t)(d->max_samples_per_node + 1) >= (1ll << 31)) return NEAT_ERR_BAD_INPUT;
    if (!d->tree_table || !d->node_min || !d->node_max || !d->intrinsics || !d->rotation || !d->translation ||
        !b->uv || !b->image_id)
        return NEAT_ERR_BAD_INPUT;
    return NEAT_OK;
}

// Rays -> per-ray hit lists -> node-major segments -> sample offsets -> tile
// map (phases 0..1 of the step).  counters[0..3] and *status are written.
// pr != nullptr (a SAMPLE step of the learned proposal): the CDF of every
// segment, and its sample count from the count head, before the sample offsets.
static bool build_segments(const neat_step_desc* d, const neat_step_batch* b, const StepLayout& L, const StepBufs& w,
                           int64_t* cnt, int* status, cudaStream_t st, const neat_proposal* pr = nullptr)
{
    const int64_t R = b->num_rays, cap = d->seg_capacity;
    const int A = d->num_active, D = d->max_depth, M = d->max_samples_per_node;
    bool ok = true;
    ok      = ok && cudaMemsetAsync(w.node_nseg, 0, (size_t)A * 4, st) == cudaSuccess;
    ok      = ok && cudaMemsetAsync(cnt, 0, 4 * sizeof(int64_t), st) == cudaSuccess;
    ok = ok && launch_step_rays(b->uv, b->image_id, R, d->w, d->h, d->intrinsics, d->rotation, d->translation,
                                d->tree_table, D, M, L.cap_ray, w.origin, w.direction, w.ray_hits, w.ray_nseg,
                                w.node_nseg, cnt, status, st, d->cell_node) == cudaSuccess;
    ok = ok && scan_exclusive<int>(w.ray_nseg, nullptr, R, w.ray_seg_off, w.scratch, cnt + 0, st) == cudaSuccess;
    ok = ok && scan_exclusive<int>(w.node_nseg, nullptr, A, w.node_seg_off, w.scratch, nullptr, st) == cudaSuccess;
    ok = ok && launch_step_place(w.ray_hits, w.ray_nseg, w.ray_seg_off, R, L.cap_ray, w.node_seg_off, w.segs,
                                 w.seg_n, cnt, cap, w.partial, status, st) == cudaSuccess;
    if (pr) ok = ok && launch_proposal_cdf(w.segs, w.seg_n, cnt, pr, w.seg_cdf, st) == cudaSuccess;
    ok = ok && scan_exclusive<int>(w.seg_n, cnt + 0, cap, w.samp_off, w.scratch, cnt + 1, st) == cudaSuccess;
    k_tile_seg<<<(unsigned)std::min<int64_t>((cap + 255) / 256, (int64_t)sm_count() * 8), 256, 0, st>>>(
        w.samp_off, w.seg_n, cnt, w.tile_seg, L.tiles_cap, L.sample_cap, status);
    return ok;
}

static StepTileArgs tile_args(const neat_step_desc* d, const StepBufs& w, const float* grid, float* grid_grad,
                              const float* decoder, int64_t* cnt, int* status, uint64_t seed, int step, int jitter)
{
    StepTileArgs ta;
    ta.segs      = w.segs;
    ta.samp_off  = w.samp_off;
    ta.tile_seg  = w.tile_seg;
    ta.counters  = cnt;
    ta.origin    = w.origin;
    ta.direction = w.direction;
    ta.node_min  = d->node_min;
    ta.node_max  = d->node_max;
    ta.grid      = grid;
    ta.grid_bf16 = nullptr;
    ta.grid_grad = grid_grad;
    ta.decoder   = decoder;
    ta.dec_part  = w.dec_part;
    ta.dpred     = w.dpred;
    ta.partial   = w.partial;
    ta.status    = status;
    ta.seed      = seed;
    ta.step      = (uint32_t)step;
    ta.step_dev  = &w.scal->step;
    ta.seg_cdf   = nullptr;
    ta.seg_hist  = nullptr;
    ta.seg_dens  = nullptr;
    ta.dens_cap  = 0;
    ta.seg_pgrad = nullptr;
    ta.rec       = nullptr;
    ta.rec_cap   = 0;
    ta.rec_skip  = 0;
    ta.jitter    = jitter;
    ta.G         = d->G;
    ta.beta      = d->softplus_beta;
    return ta;
}

static cudaError_t launch_tiles_path(const neat_step_desc* d, bool bwd, const StepTileArgs& ta, cudaStream_t st)
{
    const int prec = d->decoder_path == NEAT_DECODER_TC_BF16 ? 0 : 1;
    return d->decoder_path == NEAT_DECODER_SIMT_FP32 ? launch_tiles_any(d->C, bwd, ta, st)
                                                     : launch_tiles_tc(d->C, prec, bwd, ta, st);
}

// Projection of each ray = sum of its segment partials in (tmin, node) order;
// optional per-block squared and absolute error sums against the target.
__global__ void k_ray_project(int64_t R, const int* __restrict__ ray_seg_off, const double* __restrict__ partial,
                              const float* __restrict__ target, float* __restrict__ pred_out,
                              double* __restrict__ err_part, const int64_t* nseg_eff, ToneMap tm)
{
    __shared__ double red[2][256];
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double sq = 0.0, ab = 0.0;
    if (r < R)
    {
        float pred = 0.0f;
        if (*nseg_eff > 0)
        {
            const int b = ray_seg_off[r], e = ray_seg_off[r + 1];
            double acc  = 0.0;
            for (int k = b; k < e; ++k) acc += partial[k];
            pred = (float)acc;
        }
        if (tm.t.params != nullptr)
        {
            // the evaluation applies the tone mapper to the prediction
            // (EvalStepProjection, samples/reconstruct.cpp:559)
            TmPoint q;
            pred = tonemap_forward(tm, r, pred, q);
        }
        pred_out[r] = pred;
        if (target)
        {
            const float diff = pred - target[r];
            sq               = (double)diff * (double)diff;
            ab               = fabs((double)diff);
        }
    }
    if (!err_part) return;
    red[0][threadIdx.x] = sq;
    red[1][threadIdx.x] = ab;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1)
    {
        if (threadIdx.x < o)
        {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] += red[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        err_part[2 * blockIdx.x]     = red[0][0];
        err_part[2 * blockIdx.x + 1] = red[1][0];
    }
}

// Adds the block sums to out[0..1] in block order (one thread: deterministic).
__global__ void k_err_final(const double* __restrict__ err_part, int nb, double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0, a = 0.0;
    for (int i = 0; i < nb; ++i)
    {
        s += err_part[2 * i];
        a += err_part[2 * i + 1];
    }
    out[0] += s;
    out[1] += a;
}

// The proposal for this call (null when off); false when it cannot be used.
static bool proposal_mode(const neat_step_desc* d, const neat_proposal* pr, int& mode)
{
    mode = pr ? pr->mode : NEAT_PROPOSAL_OFF;
    if (mode == NEAT_PROPOSAL_OFF) return true;
    if (mode != NEAT_PROPOSAL_SAMPLE && mode != NEAT_PROPOSAL_TRAIN) return false;
    if (!d->proposal || d->decoder_path == NEAT_DECODER_SIMT_FP32 || !pr->params || !pr->node_desc) return false;
    if (mode == NEAT_PROPOSAL_TRAIN && (!pr->m || !pr->v || !pr->grad || !pr->step_counter || pr->iters < 0))
        return false;
    if (pr->count_eps > 0.0f && pr->count_min < 1) return false;
    return pr->mix >= 0.0f && pr->mix <= 1.0f && !(pr->count_eps < 0.0f) && pr->count_eps == pr->count_eps;
}

}  // namespace neat

// One training step; `prebuilt`: the segment lists of this batch are already
// in the workspace and out->counters (neat_train_step_segments).
static int train_step(const neat_step_desc* d, const neat_step_state* s, const neat_step_batch* b, uint64_t seed,
                      int step, const neat_step_out* out, void* workspace, size_t workspace_bytes,
                      neat_stream_t stream, bool prebuilt)
{
    if (!d || !s || !b || !out || !out->loss || !out->counters || (!s->step_counter && step < 1))
        return NEAT_ERR_BAD_INPUT;
    const int chk = check_desc(d, b);
    if (chk != NEAT_OK) return chk;
    if (!s->grid || !s->grid_m || !s->grid_v || !s->grid_grad || !s->decoder || !s->decoder_m || !s->decoder_v ||
        !s->decoder_grad || !b->target || !workspace)
        return NEAT_ERR_BAD_INPUT;
    int pmode = NEAT_PROPOSAL_OFF;
    if (!proposal_mode(d, s->proposal, pmode)) return NEAT_ERR_BAD_INPUT;
    if (s->grid_bf16 && (d->decoder_path == NEAT_DECODER_SIMT_FP32 || ((uintptr_t)s->grid_bf16 & 15)))
        return NEAT_ERR_BAD_INPUT;
    if (s->pose && (!d->pose_grad || d->decoder_path == NEAT_DECODER_SIMT_FP32 || !s->pose->grad_tangent ||
                    !s->pose->grad_translation || !s->pose->grad_intrinsics || s->pose->num_images < 1))
        return NEAT_ERR_BAD_INPUT;
    if (s->tonemap && (!s->tonemap->params || !s->tonemap->grad || s->tonemap->num_images < 1 ||
                       (s->tonemap->sensor_bias && (s->tonemap->bias_w < 2 || s->tonemap->bias_h < 2)) ||
                       !(s->tonemap->response_range > 0.0f)))
        return NEAT_ERR_BAD_INPUT;
    const int64_t R = b->num_rays;
    StepLayout L;
    if (!step_layout(d, R, L) || workspace_bytes < L.total) return NEAT_ERR_CAPACITY;
    cudaStream_t st    = (cudaStream_t)stream;
    const StepBufs w   = step_bufs(L, workspace);
    int64_t* cnt       = out->counters;
    const int A        = d->num_active;
    const neat_proposal* pr = s->proposal;

    auto phase = [&](int i) {
        if (out->phase_events && out->phase_events[i]) cudaEventRecord((cudaEvent_t)out->phase_events[i], st);
    };
    bool ok = true;
    phase(0);
    k_step_begin<<<1, 32, 0, st>>>(s->step_counter, step, (double)d->lr_grid, (double)d->lr_decoder,
                                   (double)d->beta1, (double)d->beta2, w.scal);
    if (!prebuilt) ok = build_segments(d, b, L, w, cnt, out->status, st, pmode == NEAT_PROPOSAL_SAMPLE ? pr : nullptr);
    phase(1);

    StepTileArgs ta = tile_args(d, w, s->grid, s->grid_grad, s->decoder, cnt, out->status, seed, step, 1);
    ta.grid_bf16    = s->grid_bf16;
    if (d->decoder_path != NEAT_DECODER_SIMT_FP32)
    {
        ta.rec     = L.rec_cap > 0 ? w.rec : nullptr;
        ta.rec_cap = L.rec_cap;
    }
    if (pmode == NEAT_PROPOSAL_SAMPLE) ta.seg_cdf = w.seg_cdf;  // placed with the segment lists
    else if (pmode == NEAT_PROPOSAL_TRAIN)
    {
        k_zero_per_segment<<<sm_count() * 4, 256, 0, st>>>(w.seg_hist, cnt, 8);
        ta.seg_hist = w.seg_hist;
        ta.seg_dens = w.seg_dens;
        ta.dens_cap = L.dens_cap;
    }
    ok = ok && launch_tiles_path(d, false, ta, st) == cudaSuccess;
    ta.seg_hist = nullptr;
    ta.seg_dens = nullptr;
    if (pmode == NEAT_PROPOSAL_TRAIN)
        ok = ok && launch_seg_variation(w.segs, w.samp_off, cnt, w.seg_dens, L.dens_cap, w.seg_tv, st) == cudaSuccess;
    phase(2);
    const float invR = (float)(1.0 / (double)R);
    ToneMap tm{};
    if (s->tonemap)
    {
        tm.t        = *s->tonemap;
        tm.uv       = b->uv;
        tm.image_id = b->image_id;
    }
    k_ray_loss<<<L.loss_blocks, 256, 0, st>>>(R, w.ray_seg_off, w.partial, b->target, w.dpred, out->prediction,
                                               w.loss_part, invR, cnt + 0, tm);
    k_loss_final<<<1, 1024, 0, st>>>(w.loss_part, L.loss_blocks, out->loss, invR);
    phase(3);
    if (s->pose)
    {
        // per-segment and per-ray pose-gradient accumulators start at zero
        k_zero_per_segment<<<sm_count() * 4, 256, 0, st>>>(w.seg_pgrad, cnt, 6);
        ok           = ok && cudaMemsetAsync(w.ray_pgrad, 0, (size_t)R * 6 * 4, st) == cudaSuccess;
        ta.seg_pgrad = w.seg_pgrad;
    }
    ok           = ok && launch_tiles_path(d, true, ta, st) == cudaSuccess;
    ta.seg_pgrad = nullptr;
    if (s->pose)
        ok = ok && launch_pose_grad(w.segs, cnt, w.seg_pgrad, d->G, w.ray_pgrad, b->uv, b->image_id, R, d->w, d->h,
                                    d->intrinsics, d->rotation, s->pose, st) == cudaSuccess;
    phase(4);

    const int P = (int)decoder_params(d->C);
    k_dec_reduce_adam<<<(P + 31) / 32, 32 * DEC_RED_GROUPS, 0, st>>>(w.dec_part, L.bwd_grid, P, s->decoder_grad, s->decoder,
                                                        s->decoder_m, s->decoder_v, d->beta1, d->beta2, d->eps,
                                                        w.scal);
    const int64_t ngrid = (int64_t)A * d->G * d->G * d->G * d->C;
    // four CTAs per SM (of eight) keep HBM busy and leave room for the next
    // batch's segment build, queued on another stream behind phase [4]
    const int agrid     = (int)std::min<int64_t>((ngrid / 4 + 255) / 256 + 1, (int64_t)sm_count() * 4);
    k_adam<<<agrid, 256, 0, st>>>(s->grid, s->grid_grad, s->grid_m, s->grid_v, ngrid, d->beta1, d->beta2, d->eps,
                                  0.0f, 1.0f, 1, w.scal, s->grid_bf16);
    if (s->tonemap)
    {
        k_tonemap_param_loss<<<1, 32, 0, st>>>(*s->tonemap);
        k_tonemap_update<<<8, 256, 0, st>>>(*s->tonemap);
    }
    if (pmode == NEAT_PROPOSAL_TRAIN)
    {
        ok = ok && launch_node_desc(s->grid, A, d->C, d->G, s->decoder, d->softplus_beta, pr->node_desc, st) ==
                       cudaSuccess;
        ok = ok && launch_proposal_train(w.segs, cnt, w.seg_hist, w.seg_tv, pr, w.prop_part, pr->iters, st) ==
                       cudaSuccess;
    }
    phase(5);
    ok = ok && cudaGetLastError() == cudaSuccess;
    return ok ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_train_step(const neat_step_desc* d, const neat_step_state* s, const neat_step_batch* b,
                               uint64_t seed, int step, const neat_step_out* out, void* workspace,
                               size_t workspace_bytes, neat_stream_t stream)
{
    return train_step(d, s, b, seed, step, out, workspace, workspace_bytes, stream, false);
}

extern "C" int neat_train_step_prebuilt(const neat_step_desc* d, const neat_step_state* s, const neat_step_batch* b,
                                        uint64_t seed, int step, const neat_step_out* out, void* workspace,
                                        size_t workspace_bytes, neat_stream_t stream)
{
    return train_step(d, s, b, seed, step, out, workspace, workspace_bytes, stream, true);
}

extern "C" int neat_train_step_segments(const neat_step_desc* d, const neat_proposal* proposal,
                                        const neat_step_batch* b, int64_t* counters, int* status, void* workspace,
                                        size_t workspace_bytes, neat_stream_t stream)
{
    if (!d || !b || !counters || !status || !workspace) return NEAT_ERR_BAD_INPUT;
    const int chk = check_desc(d, b);
    if (chk != NEAT_OK) return chk;
    int pmode = NEAT_PROPOSAL_OFF;
    if (!proposal_mode(d, proposal, pmode)) return NEAT_ERR_BAD_INPUT;
    StepLayout L;
    if (!step_layout(d, b->num_rays, L) || workspace_bytes < L.total) return NEAT_ERR_CAPACITY;
    const StepBufs w = step_bufs(L, workspace);
    cudaStream_t st  = (cudaStream_t)stream;
    // a SAMPLE step's placement CDF and sample counts depend on the segments and
    // on the proposal's parameters and node descriptors, which only a TRAIN
    // step's end changes
    bool ok = build_segments(d, b, L, w, counters, status, st, pmode == NEAT_PROPOSAL_SAMPLE ? proposal : nullptr);
    return ok && cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_project(const neat_step_desc* d, const float* grid, const float* decoder,
                            const neat_proposal* proposal, const neat_step_batch* b, const neat_project_out* out,
                            void* workspace, size_t workspace_bytes, neat_stream_t stream)
{
    int pmode = NEAT_PROPOSAL_OFF;
    if (d && !proposal_mode(d, proposal, pmode)) return NEAT_ERR_BAD_INPUT;
    if (pmode == NEAT_PROPOSAL_TRAIN) return NEAT_ERR_BAD_INPUT;
    if (!d || !b || !out || !out->prediction || !out->counters || !out->status || !grid || !decoder || !workspace)
        return NEAT_ERR_BAD_INPUT;
    if (out->error_sums && !b->target) return NEAT_ERR_BAD_INPUT;
    const int chk = check_desc(d, b);
    if (chk != NEAT_OK) return chk;
    const int64_t R = b->num_rays;
    StepLayout L;
    if (!step_layout(d, R, L) || workspace_bytes < L.total) return NEAT_ERR_CAPACITY;
    cudaStream_t st  = (cudaStream_t)stream;
    const StepBufs w = step_bufs(L, workspace);
    int64_t* cnt     = out->counters;
    k_step_begin<<<1, 32, 0, st>>>(nullptr, 1, 0.0, 0.0, 0.5, 0.5, w.scal);
    bool ok = build_segments(d, b, L, w, cnt, out->status, st, pmode == NEAT_PROPOSAL_SAMPLE ? proposal : nullptr);
    StepTileArgs ta = tile_args(d, w, grid, nullptr, decoder, cnt, out->status, 0, 1, 0);
    if (pmode == NEAT_PROPOSAL_SAMPLE) ta.seg_cdf = w.seg_cdf;
    ok = ok && launch_tiles_path(d, false, ta, st) == cudaSuccess;
    // the loss-partials slab holds L.loss_blocks floats; the error sums need two
    // doubles per block, which the (larger) dpred slab of R floats provides
    double* err_part = out->error_sums ? (double*)w.dpred : nullptr;
    ToneMap tm{};
    if (out->tonemap)
    {
        tm.t        = *out->tonemap;
        tm.uv       = b->uv;
        tm.image_id = b->image_id;
    }
    k_ray_project<<<L.loss_blocks, 256, 0, st>>>(R, w.ray_seg_off, w.partial, b->target, out->prediction, err_part,
                                                  cnt + 0, tm);
    if (err_part) k_err_final<<<1, 32, 0, st>>>(err_part, L.loss_blocks, out->error_sums);
    ok = ok && cudaGetLastError() == cudaSuccess;
    return ok ? NEAT_OK : NEAT_ERR_CUDA;
}
