// neat_bwd_rec.cu -- backward sample tiles of the fused step from the
// forward's per-sample records, three-piece BF16 operands (FP32-level
// accuracy), with one warp that only issues the tensor-core work.
//
// A tcgen05.mma of these shapes holds its issuing thread for about its
// execution time, and every GEMM of a tile waits on the CUDA-core work before
// it.  Here eight compute warps (two threads per sample, 32 hidden units
// each) hand operands to a ninth warp whose lane 0 issues every MMA, and the
// CUDA-core work that does not feed the next GEMM runs in the GEMM windows:
//   wait L1_i -> h1 epilogue: silu'(z1) over Z1, h1's BF16 pieces into TMEM
//     (the layer-2 A operand); meanwhile WG_{i-1} runs, and tile i+1's
//     record loads, issued just before, land
//   -> tile i-1's dX from TMEM
//   -> Z2_i, queued behind WG_{i-1}; meanwhile half of the scatter of tile
//     i-1's dX, tile i+1's grid features into the [x | 1] buffer, the
//     dL/dpred of its rays, and (once WG_{i-1}, the last reader of HB and AB,
//     is done) h1's pieces from TMEM into HB
//   -> y epilogue -> dz2 -> dH1_i; meanwhile more of tile i-1's scatter and
//     tile i+1's slot data
//   -> dz1 -> L1_{i+1}, dX_i (into D2's first columns, read by tile i+1
//     before its layer 2) and WG_i = [dz2 | dz1]^T [h1 | x | 1], which runs
//     under tile i+1's h1 epilogue; until L1_{i+1} is done, the last part of
//     tile i-1's scatter.
// Same arithmetic as the record path of k_step_tiles_tc<C, BF16X3, true>
// (operand splits, piece products, TMEM column blocks, f32 epilogues); only
// the order of the grid-gradient atomics differs.
//
// Synchronisation: compute warps announce ready operands with one arrival
// per warp on an mbarrier (count 8), after fence.proxy.async for shared
// stores and tcgen05.wait::st + fence::before_thread_sync for TMEM stores;
// the MMA warp answers each GEMM with tcgen05.commit on its own mbarrier.
// Every wait is bounded.  A compute thread whose wait gives up stops waiting
// but keeps to the loop (so the named barriers of the compute warps always
// see all 256 threads); the decision is joined (bar.red.and) after the loop.
// The MMA warp gives up on its own; both drain and free TMEM before
// returning.
#include <cuda_bf16.h>

#include <algorithm>

#include "neat_internal.h"
#include "neat_slots.cuh"
#include "neat_tc.cuh"
#include "neat_tiles.cuh"

namespace neat
{
namespace tc
{

// Two compute warpgroups and one MMA warpgroup (warp 8 issues; 9-11 idle).
// Launched at 168 registers a thread (three warps share each SM
// sub-partition's register file); setmaxnreg then moves them to the compute
// warps: 8 x 32 x 224 + 4 x 32 x 56 = 384 x 168.
constexpr int BR_THREADS = 384;
constexpr int BR_REGS_COMPUTE = 192, BR_REGS_MMA = 120;
static_assert(8 * BR_REGS_COMPUTE + 4 * BR_REGS_MMA <= 12 * 168, "register split exceeds the launch's registers");

// Shared-memory and TMEM plan of the records backward for precision PREC.
// Shared memory: the tile plan of Cfg<C, PREC, true> up to its slot data,
// then [3][6][128] slot data for the second thread of a sample, the
// reduction scratch and the mbarriers.  TMEM columns:
//   three pieces (one CTA per SM, 512 columns): D1 [0,64) Z1 / silu'(z1);
//     D2 [64,128) Z2; dH1 [64,256) (one block per W2 piece); h1 pieces
//     [128,224); dX [64,112) until the next tile's Z2; weight gradients
//     [256,496);
//   one piece (BF16, 256 columns): D1 [0,64); D2 [64,128) Z2, then dH1, then
//     dX [64, 64 + K1); h1 [128,160); weight gradients [160, 160 + NW).
template <int C, int PREC>
struct BwdRecPlan
{
    using K  = Cfg<C, PREC, true>;
    using PP = Prec<PREC>;
    static constexpr int QB     = 6 * 128;
    static constexpr int OFF_Q  = K::OFF_Q;
    static constexpr int OFF_R0 = OFF_Q + 3 * QB * 4;
    static constexpr int OFF_R  = K::OFF_R > OFF_R0 ? K::OFF_R : OFF_R0;
    static constexpr int OFF_M0 = ((OFF_R + 8 * HH * 4) + 15) / 16 * 16;
    static constexpr int OFF_M  = K::OFF_M > OFF_M0 ? K::OFF_M : OFF_M0;
    static constexpr int BYTES  = OFF_M + 96;  // 10 mbarriers, then the TMEM slot at +88
    static constexpr int TTA    = 128;         // h1 pieces (layer-2 A operand)
    static constexpr int TD4    = PREC == BF16X3 ? 256 : TTA + 32 * PP::PIECES;
    static constexpr uint32_t TMEM_COLS = PREC == BF16X3 ? 512 : 256;
    static_assert(PREC != BF16X3 || (K::CACHE && K::D4 == 256 && K::OFF_R - K::OFF_Q >= 3 * QB * 4 &&
                                     OFF_R == K::OFF_R && OFF_M == K::OFF_M),
                  "three-piece plan: D1 [0,64) Z1 / silu'(z1); D2 [64,128) Z2; dH1 [64,256); "
                  "h1 pieces [128,224); dX [64,112) until the next tile's Z2; weight gradients [256,496)");
    static_assert(K::NX1 == 1 && K::WCAT && K::TA_COL == TTA, "one [x | 1] buffer, piece-concatenated GEMMs");
    static_assert(PP::PIECES * K::K1 <= 64, "dX column blocks must fit below the h1 pieces");
    static_assert(64 + 64 * PP::PIECES <= TD4 && TTA + 32 * PP::PIECES <= TD4 || PREC == BF16X3,
                  "one piece: dH1 and the h1 pieces below the weight gradients");
    static_assert(TD4 + PP::PIECES * K::NW <= (int)TMEM_COLS, "weight gradients must fit the allocation");
    static_assert(BYTES <= 232448, "shared-memory plan exceeds the per-CTA limit");
};

template <int C, int PREC, bool POSE>
__global__ void __launch_bounds__(BR_THREADS, 1) k_bwd_rec(StepTcArgs a)
{
    using K            = Cfg<C, PREC, true>;
    using L            = BwdRecPlan<C, PREC>;
    using P            = Prec<PREC>;
    using HB           = typename K::HB;
    using X1           = typename K::X1;
    using AB           = typename K::AB;
    using W2           = typename K::W2;
    using W1           = typename K::W1;
    using O            = DecOff<C>;
    constexpr int HALF = HH / 2;

    // the step's samples fit the records (the plain kernel runs otherwise)
    const int64_t S = a.counters[1];
    if (a.rec == nullptr || S > a.rec_cap) return;

    extern __shared__ __align__(128) unsigned char sm[];
    const int t = threadIdx.x, w = t >> 5, l = t & 31, s = t & 127, h = (t >> 7) & 1;
    const int c0       = h * HALF;
    // warpgroup role, warp-uniform by construction
    const int wg       = __shfl_sync(0xffffffffu, t >> 7, 0);
    const bool compute = wg < 2;
    float* sb2         = reinterpret_cast<float*>(sm + K::OFF_F);
    float* sw3         = sb2 + HH;
    float* sb3         = sw3 + HH;
    float* sval        = reinterpret_cast<float*>(sm + K::OFF_V);  // [2][128] y halves
    float* sq          = reinterpret_cast<float*>(sm + K::OFF_Q);  // [3][6][128]
    float* sred        = reinterpret_cast<float*>(sm + L::OFF_R);
    uint32_t* tslot    = reinterpret_cast<uint32_t*>(sm + L::OFF_M + 88);
    const uint32_t s_base = smem_u32(sm);
    const uint32_t mbase  = smem_u32(sm + L::OFF_M);
    // MMA completion (tcgen05.commit, count 1)
    const uint32_t m_l1 = mbase, m_z2 = mbase + 8, m_dh1 = mbase + 16, m_wg = mbase + 24, m_end = mbase + 32;
    // operands ready (one arrival per compute warp, count 8)
    const uint32_t r_x1 = mbase + 40, r_z2 = mbase + 48, r_dh1 = mbase + 56, r_dz1 = mbase + 64;
    const uint32_t m_dx = mbase + 72;  // dX (tcgen05.commit, count 1)

    // ---- decoder parameters: b2 / w3 / b3 in fp32, [W1 | b1] and W2 as MMA operand pieces
    for (int i = t; i < HH; i += BR_THREADS)
    {
        sb2[i] = a.decoder[O::b2 + i];
        sw3[i] = a.decoder[O::W3 + i];
    }
    if (t == 0) sb3[0] = a.decoder[O::b3];
    for (int i = t; i < HH * HH + HH * K::K1; i += BR_THREADS)
    {
        float r;
        int off, piece_bytes;
        unsigned char* dst;
        if (i < HH * HH)
        {
            r           = a.decoder[O::W2 + i];
            off         = W2::off(i / HH, i % HH);
            dst         = sm + K::OFF_W2;
            piece_bytes = K::W2_PC;
        }
        else
        {
            const int e = i - HH * HH, hr = e / K::K1, col = e % K::K1;
            r           = col < C ? a.decoder[O::W1 + hr * C + col] : (col == K::ONE ? a.decoder[O::b1 + hr] : 0.0f);
            off         = W1::off(hr, col);
            dst         = sm + K::OFF_W1;
            piece_bytes = K::W1_PC;
        }
#pragma unroll
        for (int p = 0; p < P::PIECES; ++p)
        {
            const __nv_bfloat16 b = __float2bfloat16_rn(r);
            *reinterpret_cast<__nv_bfloat16*>(dst + p * piece_bytes + off) = b;
            r -= __bfloat162float(b);
        }
    }
    if (t == 0)
    {
        for (int k = 0; k < 5; ++k) mbar_init(mbase + 8 * k, 1);
        for (int k = 5; k < 9; ++k) mbar_init(mbase + 8 * k, 8);
        mbar_init(m_dx, 1);
    }
    if (w == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(L::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t lane = (uint32_t)((w & 3) * 32) << 16;  // TMEM lane quadrant of this warp
    const uint32_t tD1 = tmem, tD2 = tmem + 64, tTA = tmem + L::TTA, tD4 = tmem + L::TD4;

    const int64_t ntiles = (S + 127) / 128, T0 = blockIdx.x, G = gridDim.x;
    constexpr uint32_t idF = make_idesc(P::FMT, 0, 0, 128, HH);  // layers 1 and 2
    constexpr int KS1      = K::K1 / P::KI;
    constexpr int KS64     = HH / P::KI;
    constexpr int KS128    = 128 / P::KI;
    bool ok                = true;

    if (compute)
    {
        // ---- compute warps -------------------------------------------------
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(BR_REGS_COMPUTE));
        // The forward's record of slot s of tile tl (zeros past the last
        // sample), read in two parts: its placement by the first thread of
        // the sample, its grid features by the second.
        struct Rec
        {
            float lu, lv, lw, t, dvw;
            int row, seg;
            bool valid;
        };
        auto read_fields = [&](int64_t tl) -> Rec {
            Rec o;
            const int64_t i = tl * 128 + s;
            o.valid         = i < S;
            if (o.valid)
            {
                const int64_t cp = a.rec_cap;
                const float* r   = a.rec;
                o.lu             = __ldcs(r + 0 * cp + i);
                o.lv             = __ldcs(r + 1 * cp + i);
                o.lw             = __ldcs(r + 2 * cp + i);
                const float wgt  = __ldcs(r + 3 * cp + i);
                o.t              = __ldcs(r + 4 * cp + i);
                const int ray    = __float_as_int(__ldcs(r + 5 * cp + i));
                o.row            = __float_as_int(__ldcs(r + 6 * cp + i));
                o.seg            = __float_as_int(__ldcs(r + 7 * cp + i));
                o.dvw            = a.dpred[ray] * wgt;
            }
            else
            {
                o.lu = o.lv = o.lw = o.t = o.dvw = 0.0f;
                o.row = 0;
                o.seg = -1;
            }
            return o;
        };
        // The fields alone, issued a tile phase ahead of use: dL/dpred of the
        // ray (a dependent load) and the slot data come later.
        struct Raw
        {
            float lu, lv, lw, wgt, t;
            int ray, row, seg;
            bool valid;
        };
        auto load_raw = [&](int64_t tl) -> Raw {
            Raw o;
            const int64_t i = tl * 128 + s;
            o.valid         = i < S;
            const int64_t cp = a.rec_cap;
            const float* r   = a.rec;
            o.lu             = o.valid ? __ldcs(r + 0 * cp + i) : 0.0f;
            o.lv             = o.valid ? __ldcs(r + 1 * cp + i) : 0.0f;
            o.lw             = o.valid ? __ldcs(r + 2 * cp + i) : 0.0f;
            o.wgt            = o.valid ? __ldcs(r + 3 * cp + i) : 0.0f;
            o.t              = o.valid ? __ldcs(r + 4 * cp + i) : 0.0f;
            o.ray            = o.valid ? __float_as_int(__ldcs(r + 5 * cp + i)) : 0;
            o.row            = o.valid ? __float_as_int(__ldcs(r + 6 * cp + i)) : 0;
            o.seg            = o.valid ? __float_as_int(__ldcs(r + 7 * cp + i)) : -1;
            return o;
        };
        auto read_x = [&](int64_t tl, float (&x)[C]) {
            const int64_t i = tl * 128 + s;
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = i < S ? __ldcs(a.rec + (8 + c) * a.rec_cap + i) : 0.0f;
        };
        // row s of [x | 1 | 0 ..]: the layer-1 buffer (b >= 0) or HB's columns [64, 64 + K1)
        auto put_x1 = [&](const float (&xv)[C], int b) {
            unsigned char* base = b >= 0 ? sm + K::OFF_X1 : sm + K::OFF_HB;
            const int pbytes    = b >= 0 ? X1::BYTES : K::HB_PC;
#pragma unroll
            for (int cc = 0; cc < K::K1; cc += P::E)
            {
                float v[P::E];
#pragma unroll
                for (int i = 0; i < P::E; ++i)
                {
                    const int c = cc + i;
                    v[i]        = (c < C) ? xv[c < C ? c : 0] : ((c == K::ONE) ? 1.0f : 0.0f);
                }
                store_chunk<PREC>(base, pbytes, b >= 0 ? X1::off(s, cc) : HB::off(s, HH + cc), v);
            }
        };
        // what the second thread of a sample needs of it, into buffer qb
        auto put_q = [&](const Rec& r, int qb) {
            float* qd       = sq + qb * L::QB;
            qd[0 * 128 + s] = r.lu;
            qd[1 * 128 + s] = r.lv;
            qd[2 * 128 + s] = r.lw;
            qd[3 * 128 + s] = r.dvw;
            qd[4 * 128 + s] = __int_as_float(r.valid ? 1 : -1);
            qd[5 * 128 + s] = __int_as_float(r.row);
        };
        // dX scattered with the trilinear weights: of the 8 corners, this
        // thread takes 4 h .. 4 h + 3, in three parts run in different windows
        // (part 0: corners 4 h, 4 h + 1; part 1: 4 h + 2; part 2: 4 h + 3)
        auto scatter = [&](int part, const float (&dx)[C], float lu, float lv, float lw, int row, bool valid) {
            if (!valid) return;
            Corners kc;
            igs_corners(lu, lv, lw, a.G, a.G, a.G, kc);
            if (h == 0)
            {
                if (part == 0)
                    scatter_cl_part<C, 0, 2>(a.grid_grad, row, a.G, kc, dx);
                else if (part == 1)
                    scatter_cl_part<C, 2, 1>(a.grid_grad, row, a.G, kc, dx);
                else
                    scatter_cl_part<C, 3, 1>(a.grid_grad, row, a.G, kc, dx);
            }
            else
            {
                if (part == 0)
                    scatter_cl_part<C, 4, 2>(a.grid_grad, row, a.G, kc, dx);
                else if (part == 1)
                    scatter_cl_part<C, 6, 1>(a.grid_grad, row, a.G, kc, dx);
                else
                    scatter_cl_part<C, 7, 1>(a.grid_grad, row, a.G, kc, dx);
            }
        };
        // the previous tile's scatter, part 0 or 1 (the first thread of a
        // sample holds its placement; the second reads it from sq)
        auto scatter_prev = [&](int part, int pqb, const float (&pdx)[C], float plu, float plv, float plw, int prow,
                                bool pvalid) {
            if (h == 0)
            {
                scatter(part, pdx, plu, plv, plw, prow, pvalid);
            }
            else
            {
                const float* qd = sq + pqb * L::QB;
                scatter(part, pdx, qd[0 * 128 + s], qd[1 * 128 + s], qd[2 * 128 + s], __float_as_int(qd[5 * 128 + s]),
                        __float_as_int(qd[4 * 128 + s]) >= 0);
            }
        };
        // camera pose gradient terms of one sample (first thread of the sample):
        // dL/d(ix, iy, iz) = sum over corners of (grid_q . dX) dw_q/d(ix, iy, iz),
        // and t times it; summed over the warp's runs of one segment
        auto pose_sample = [&](const float (&dx)[C], float lu, float lv, float lw, float ts, int row, int seg,
                               bool valid) {
            float g[6] = {};
            if (valid)
            {
                Corners kc;
                igs_corners(lu, lv, lw, a.G, a.G, a.G, kc);
                const float ax0 = __fsub_rn((float)(kc.x0 + 1), kc.ix), ax1 = __fsub_rn(kc.ix, (float)kc.x0);
                const float ay0 = __fsub_rn((float)(kc.y0 + 1), kc.iy), ay1 = __fsub_rn(kc.iy, (float)kc.y0);
                const float az0 = __fsub_rn((float)(kc.z0 + 1), kc.iz), az1 = __fsub_rn(kc.iz, (float)kc.z0);
                const int64_t base = (int64_t)row * a.G * a.G * a.G;
#pragma unroll
                for (int qq = 0; qq < 8; ++qq)
                {
                    const int64_t cell = (base + corner_cell(kc, qq, a.G, a.G)) * C;
                    float gq           = 0.0f;
                    if (a.grid_bf16)
                    {
#pragma unroll
                        for (int c = 0; c < C; ++c)
                            gq = fmaf(__uint_as_float((uint32_t)__ldg(a.grid_bf16 + cell + c) << 16), dx[c], gq);
                    }
                    else
                    {
#pragma unroll
                        for (int c4 = 0; c4 < C / 4; ++c4)
                        {
                            const float4 v = __ldg(reinterpret_cast<const float4*>(a.grid + cell) + c4);
                            gq             = fmaf(v.x, dx[4 * c4], gq);
                            gq             = fmaf(v.y, dx[4 * c4 + 1], gq);
                            gq             = fmaf(v.z, dx[4 * c4 + 2], gq);
                            gq             = fmaf(v.w, dx[4 * c4 + 3], gq);
                        }
                    }
                    const float fx = (qq & 1) ? ax1 : ax0, fy = (qq & 2) ? ay1 : ay0, fz = (qq & 4) ? az1 : az0;
                    g[0] = fmaf(gq, ((qq & 1) ? 1.0f : -1.0f) * fy * fz, g[0]);
                    g[1] = fmaf(gq, fx * ((qq & 2) ? 1.0f : -1.0f) * fz, g[1]);
                    g[2] = fmaf(gq, fx * fy * ((qq & 4) ? 1.0f : -1.0f), g[2]);
                }
                g[3] = g[0] * ts;
                g[4] = g[1] * ts;
                g[5] = g[2] * ts;
            }
            const int sg = valid ? seg : -1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int sn = __shfl_down_sync(0xffffffffu, sg, o);
#pragma unroll
                for (int k = 0; k < 6; ++k)
                {
                    const float vn = __shfl_down_sync(0xffffffffu, g[k], o);
                    if (l + o < 32 && sn == sg) g[k] += vn;
                }
            }
            const int sp = __shfl_up_sync(0xffffffffu, sg, 1);
            if (valid && (l == 0 || sp != sg))
#pragma unroll
                for (int k = 0; k < 6; ++k) atomicAdd(a.seg_pgrad + 6 * (int64_t)seg + k, g[k]);
        };
        auto csync = [&]() { asm volatile("bar.sync 1, 256;" ::: "memory"); };
        auto csync_and = [&](bool v) -> bool {
            uint32_t r;
            asm volatile(
                "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 256, p;\n\t"
                "selp.u32 %0, 1, 0, q;\n\t}"
                : "=r"(r)
                : "r"((uint32_t)v)
                : "memory");
            return r != 0;
        };
        // an MMA completion (this thread's own bounded wait; none after a failure)
        auto cwait = [&](uint32_t bar, uint32_t& ph, bool also = true) -> bool {
            const bool mine = ok && mbar_wait_bounded(bar, ph);
            ph ^= 1u;
            fence_after();
            return mine && also;
        };
        // this warp's operands are in place (shared stores visible to the
        // tensor core; TMEM stores waited for by the caller)
        auto cready = [&](uint32_t bar) {
            fence_smem_async();
            fence_before();
            __syncwarp();
            if (l == 0) mbar_arrive(bar);
        };

        uint32_t p_l1 = 0, p_z2 = 0, p_dh1 = 0, p_wg = 0, p_dx = 0;
        // dX of the previous tile, from its column blocks in D2 (summed)
        auto read_dx = [&](float (&dx)[C]) {
            uint32_t v[P::PIECES][16];
#pragma unroll
            for (int p = 0; p < P::PIECES; ++p) tmem_ld16_async(tD2 + lane + p * K::K1, v[p]);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < C; ++c)
            {
                float u = __uint_as_float(v[0][c]);
#pragma unroll
                for (int p = 1; p < P::PIECES; ++p) u += __uint_as_float(v[p][c]);
                dx[c] = u;
            }
        };
        float2 dw3[HALF / 2];  // this thread's columns (pairs): sum over its samples of h2 * dy
#pragma unroll
        for (int i = 0; i < HALF / 2; ++i) dw3[i] = make_float2(0.0f, 0.0f);
        float db3       = 0.0f;
        bool wg_started = false;
        Rec cur         = {};
        cur.seg         = -1;
        float cx[C]     = {};  // second thread: the tile's grid features
        // the previous tile's dX and its sample (first thread; the second reads sq)
        float pdx[C] = {};
        float plu = 0.0f, plv = 0.0f, plw = 0.0f, pt = 0.0f;
        int prow = 0, pseg = -1;
        bool pvalid = false, has_prev = false;
        int it = 0;
        if (T0 < ntiles)
        {
            if (h == 0)
            {
                cur = read_fields(T0);
                put_q(cur, 0);
            }
            else
            {
                read_x(T0, cx);
                put_x1(cx, 0);
            }
            cready(r_x1);
        }
        for (int64_t tile = T0; tile < ntiles; tile += G, ++it)
        {
            const int qb = it % 3, nqb = (it + 1) % 3, pqb = (it + 2) % 3;
            const int64_t nxt   = tile + G;
            const bool has_next = nxt < ntiles;
            // ---- layer 1 of this tile
            ok = cwait(m_l1, p_l1) && ok;
            // ---- the next tile's record, in flight during the h1 epilogue:
            //      placement fields (first thread), grid features (second)
            Raw nr;
            float nxx[C];
            if (has_next)
            {
                if (h == 0)
                    nr = load_raw(nxt);
                else
                    read_x(nxt, nxx);
            }
            // ---- h1 = silu(Z1): silu'(z1) over Z1; h1's pieces -> TMEM (layer-2 A operand)
            uint32_t z1r[HALF / 16][16];
#pragma unroll
            for (int j = 0; j < HALF / 16; ++j) tmem_ld16_async(tD1 + lane + c0 + 16 * j, z1r[j]);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < HALF / 16; ++j)
            {
                // pairs of columns in f32x2: sg = sigmoid(z), silu'(z) = sg (1 + z (1 - sg)), h1 = z sg
                float2 hz[8];
                float d1[16];
#pragma unroll
                for (int i = 0; i < 8; ++i)
                {
                    const float2 z  = make_float2(__uint_as_float(z1r[j][2 * i]), __uint_as_float(z1r[j][2 * i + 1]));
                    const float2 sg = sigmoid2<PREC>(z);
                    const float2 u  = __ffma2_rn(z, __ffma2_rn(sg, neg1x2(), one2()), one2());
                    const float2 dd = __fmul2_rn(sg, u);
                    d1[2 * i]       = dd.x;
                    d1[2 * i + 1]   = dd.y;
                    hz[i]           = __fmul2_rn(z, sg);
                }
                tmem_st16(tD1 + lane + c0 + 16 * j, d1);
#pragma unroll
                for (int p = 0; p < P::PIECES; ++p)
                {
                    uint32_t v[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[i] = piece2(hz[i]);
                    tmem_st8(tTA + lane + 32 * p + (c0 + 16 * j) / 2, v);
                }
            }
            tmem_wait_st();
            // ---- the previous tile's dX (issued behind this tile's layer 1),
            //      read before layer 2 overwrites its columns
            bool dx_ok = true;
            if (has_prev)
            {
                dx_ok = ok && mbar_wait_bounded(m_dx, p_dx);
                p_dx ^= 1u;
                fence_after();
                read_dx(pdx);
            }
            cready(r_z2);
            // ---- while layer 2 runs: half of the previous tile's scatter; the
            //      next tile's grid features into the [x | 1] buffer of its
            //      layer 1 (issued behind dX; the buffer's last reader, this
            //      tile's layer 1, has completed); dL/dpred of its rays
            if (has_prev) scatter_prev(0, pqb, pdx, plu, plv, plw, prow, pvalid);
            float ndp = 0.0f;
            if (has_next)
            {
                if (h == 1)
                    put_x1(nxx, 0);
                else if (nr.valid)
                    ndp = a.dpred[nr.ray];
            }
            // ---- once the previous tile's weight gradients (HB's last reader)
            //      are done: h1's pieces TMEM -> HB (the weight-gradient B
            //      operand), x -> HB; layer 2 still reads the pieces in TMEM
            bool wg_ok = true;
            if (has_prev)
            {
                wg_ok = ok && mbar_wait_bounded(m_wg, p_wg);
                p_wg ^= 1u;
                fence_after();
            }
#pragma unroll
            for (int j = 0; j < HALF / 16; ++j)
            {
                uint32_t v[P::PIECES][8];
#pragma unroll
                for (int p = 0; p < P::PIECES; ++p) tmem_ld8_async(tTA + lane + 32 * p + (c0 + 16 * j) / 2, v[p]);
                tmem_wait_ld();
#pragma unroll
                for (int p = 0; p < P::PIECES; ++p)
                {
                    unsigned char* dst = sm + K::OFF_HB + p * K::HB_PC;
                    *reinterpret_cast<uint4*>(dst + HB::off(s, c0 + 16 * j)) =
                        make_uint4(v[p][0], v[p][1], v[p][2], v[p][3]);
                    *reinterpret_cast<uint4*>(dst + HB::off(s, c0 + 16 * j + 8)) =
                        make_uint4(v[p][4], v[p][5], v[p][6], v[p][7]);
                }
            }
            if (h == 1) put_x1(cx, -1);
            // ---- layer 2 done; every thread's reads of the h1 pieces, whose
            //      columns h2 takes below, are done
            fence_before();
            ok = cwait(m_z2, p_z2, wg_ok && dx_ok) && ok;
            // ---- epilogue 1: y = b3 + sum over both halves; h2 and w3 silu'(z2 + b2)
            //      kept in registers for the dz2 epilogue
            float2 gk[HALF / 2], h2k[HALF / 2];
            {
                float2 yp2 = make_float2(0.0f, 0.0f);
                uint32_t z2r[HALF / 16][16];
#pragma unroll
                for (int j = 0; j < HALF / 16; ++j) tmem_ld16_async(tD2 + lane + c0 + 16 * j, z2r[j]);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < HALF / 16; ++j)
                {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                    {
                        const int col   = c0 + 16 * j + 2 * i;
                        const float2 b2 = *reinterpret_cast<const float2*>(sb2 + col);
                        const float2 w3 = *reinterpret_cast<const float2*>(sw3 + col);
                        const float2 zz = __fadd2_rn(
                            make_float2(__uint_as_float(z2r[j][2 * i]), __uint_as_float(z2r[j][2 * i + 1])), b2);
                        const float2 sg = sigmoid2<PREC>(zz);
                        const float2 h2 = __fmul2_rn(zz, sg);
                        yp2             = __ffma2_rn(h2, w3, yp2);
                        h2k[8 * j + i]  = h2;
                        const float2 u  = __ffma2_rn(zz, __ffma2_rn(sg, neg1x2(), one2()), one2());
                        gk[8 * j + i]   = __fmul2_rn(w3, __fmul2_rn(sg, u));
                    }
                }
                sval[h * 128 + s] = yp2.x + yp2.y;
            }
            csync();
            const float y   = sb3[0] + sval[s] + sval[128 + s];
            const float dvw = h == 0 ? cur.dvw : sq[qb * L::QB + 3 * 128 + s];
            const float dy  = dvw * softplus_grad(y, a.beta);
            if (h == 0) db3 += dy;
            // ---- dz2 (this thread's columns) -> AB[:, c0 ..]; dW3 += h2 dy
#pragma unroll
            for (int j = 0; j < HALF / 16; ++j)
            {
                float d[16];
                const float2 dy2 = make_float2(dy, dy);
#pragma unroll
                for (int i = 0; i < 8; ++i)
                {
                    const float2 dd  = __fmul2_rn(dy2, gk[8 * j + i]);
                    d[2 * i]         = dd.x;
                    d[2 * i + 1]     = dd.y;
                    dw3[8 * j + i]   = __ffma2_rn(h2k[8 * j + i], dy2, dw3[8 * j + i]);
                }
#pragma unroll
                for (int i = 0; i < 16; i += P::E)
                    store_chunk<PREC>(sm + K::OFF_AB, AB::BYTES, AB::off(s, c0 + 16 * j + i), d + i);
            }
            cready(r_dh1);
            // ---- while dH1 runs: the rest of the previous tile's scatter; the
            //      next tile's slot data
            if (has_prev)
            {
                scatter_prev(1, pqb, pdx, plu, plv, plw, prow, pvalid);
                if constexpr (POSE)
                {
                    if (h == 0) pose_sample(pdx, plu, plv, plw, pt, prow, pseg, pvalid);
                }
            }
            Rec nx;
            if (has_next && h == 0)
            {
                nx.lu    = nr.lu;
                nx.lv    = nr.lv;
                nx.lw    = nr.lw;
                nx.t     = nr.t;
                nx.dvw   = ndp * nr.wgt;
                nx.row   = nr.row;
                nx.seg   = nr.seg;
                nx.valid = nr.valid;
                put_q(nx, nqb);
            }
            ok = cwait(m_dh1, p_dh1) && ok;
            // ---- dz1 = dH1 silu'(z1) -> AB[:, 64 + c0 ..] (dH1: one column block per
            //      W2 piece); the second chunk's loads in flight during the first's work
            {
                uint32_t gr[HALF / 16][P::PIECES][16], dr[HALF / 16][16];
                auto load = [&](int j) {
#pragma unroll
                    for (int p = 0; p < P::PIECES; ++p)
                        tmem_ld16_async(tD2 + p * HH + lane + c0 + 16 * j, gr[j][p]);
                    tmem_ld16_async(tD1 + lane + c0 + 16 * j, dr[j]);
                };
                load(0);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < HALF / 16; ++j)
                {
                    if (j + 1 < HALF / 16) load(j + 1);
                    float g[16];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                    {
                        auto pr = [&](const uint32_t (&r)[16]) {
                            return make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
                        };
                        float2 v = pr(gr[j][P::PIECES - 1]);
#pragma unroll
                        for (int p = P::PIECES - 2; p >= 0; --p) v = __fadd2_rn(v, pr(gr[j][p]));
                        const float2 gg = __fmul2_rn(v, pr(dr[j]));
                        g[2 * i]        = gg.x;
                        g[2 * i + 1]    = gg.y;
                    }
#pragma unroll
                    for (int i = 0; i < 16; i += P::E)
                        store_chunk<PREC>(sm + K::OFF_AB, AB::BYTES, AB::off(s, HH + c0 + 16 * j + i), g + i);
                    if (j + 1 < HALF / 16) tmem_wait_ld();
                }
            }
            cready(r_dz1);  // the next layer 1, this tile's dX and weight gradients
            // ---- while the next layer 1 runs: the last part of the previous tile's scatter
            if (has_prev) scatter_prev(2, pqb, pdx, plu, plv, plw, prow, pvalid);
            wg_started = true;
            // this tile's sample, for its scatter during the next tile's layer 2
            plu      = cur.lu;
            plv      = cur.lv;
            plw      = cur.lw;
            pt       = cur.t;
            prow     = cur.row;
            pseg     = cur.seg;
            pvalid   = cur.valid;
            has_prev = true;
            if (has_next)
            {
                if (h == 0)
                    cur = nx;
                else
#pragma unroll
                    for (int c = 0; c < C; ++c) cx[c] = nxx[c];
            }
        }
        // every compute thread takes the same branch below (warp-collective TMEM
        // loads and shuffles)
        ok = csync_and(ok);
        // ---- the last tile's dX and scatter
        if (ok && has_prev)
        {
            const bool e = mbar_wait_bounded(m_dx, p_dx);
            fence_after();
            if (!e) ok = false;
            read_dx(pdx);
            scatter_prev(0, (it + 2) % 3, pdx, plu, plv, plw, prow, pvalid);
            scatter_prev(1, (it + 2) % 3, pdx, plu, plv, plw, prow, pvalid);
            scatter_prev(2, (it + 2) % 3, pdx, plu, plv, plw, prow, pvalid);
            if constexpr (POSE)
            {
                if (h == 0) pose_sample(pdx, plu, plv, plw, pt, prow, pseg, pvalid);
            }
        }
        // ---- the last weight-gradient GEMM
        if (wg_started)
        {
            const bool e = mbar_wait_bounded(m_end, 0);
            ok           = csync_and(ok && e);
            fence_after();
        }
        else
        {
            ok = csync_and(ok);
        }
        // ---- per-CTA decoder-gradient partial (the plain kernel's layout): row s of D4.
        // Rows < 64 (dz2 features): columns [0,64) dW2, column 64 + ONE db2;
        // rows >= 64 (dz1 features): columns 64 + c dW1, column 64 + ONE db1.
        float* dst         = a.dec_part + (int64_t)blockIdx.x * O::total;
        constexpr int NCH  = (HH + K::K1) / 16;
#pragma unroll 1
        for (int j = h; j < NCH; j += 2)
        {
            float v[16];
            if (wg_started && ok)
            {
                tmem_ld16(tD4 + lane + 16 * j, v);
#pragma unroll
                for (int p = 1; p < P::PIECES; ++p)
                {
                    float u[16];
                    tmem_ld16(tD4 + lane + p * K::NW + 16 * j, u);
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] += u[i];
                }
            }
            else
            {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i)
            {
                const int n = 16 * j + i;
                if (s < HH)
                {
                    if (n < HH) dst[O::W2 + s * HH + n] = v[i];
                    if (n == HH + K::ONE) dst[O::b2 + s] = v[i];
                }
                else
                {
                    const int k = s - HH;
                    if (n >= HH && n < HH + C) dst[O::W1 + k * C + (n - HH)] = v[i];
                    if (n == HH + K::ONE) dst[O::b1 + k] = v[i];
                }
            }
        }
        // dW3: each thread holds its columns summed over its samples; reduce
        // over the 32 lanes, then over the 4 warps of a half
        {
            float v[HALF];
#pragma unroll
            for (int i = 0; i < HALF / 2; ++i)
            {
                v[2 * i]     = dw3[i].x;
                v[2 * i + 1] = dw3[i].y;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int i = 0; i < HALF; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
#pragma unroll
            for (int i = 0; i < HALF; ++i)
                if (i == l) sred[w * HH + c0 + i] = v[i];
        }
        const float b3w = warp_sum(db3);
        csync();
        if (t < HH)
        {
            const int part = t / HALF;
            float acc      = 0.0f;
            for (int ww = 4 * part; ww < 4 * part + 4; ++ww) acc += sred[ww * HH + t];
            dst[O::W3 + t] = acc;
        }
        csync();
        if (l == 0) sred[w] = b3w;
        csync();
        if (t == 0)
        {
            float acc = 0.0f;
            for (int ww = 0; ww < 8; ++ww) acc += sred[ww];
            dst[O::b3] = acc;
        }
        if (!ok && t == 0) raise_status(a.status, NEAT_ERR_TIMEOUT);
    }
    else
    {
        // ---- the MMA warpgroup: warp 8 issues ------------------------------
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(BR_REGS_MMA));
        if (w == 8 && l == 0 && T0 < ntiles)
        {
            // operand descriptors re-formed at each use: hoisted out of the
            // tile loop, the 78 per-MMA descriptors would not fit the MMA
            // warp's registers
            auto desc = [&](uint32_t addr, uint32_t lbo, uint32_t sbo) -> uint64_t {
                uint64_t d = sdesc(addr, lbo, sbo);
                asm volatile("" : "+l"(d));
                return d;
            };
            auto iwait = [&](uint32_t bar, uint32_t& ph) -> bool {
                const bool r = mbar_wait_bounded(bar, ph);
                ph ^= 1u;
                fence_after();
                return r;
            };
            auto issue_l1 = [&]() {
                gemm<PREC, KS1, X1::BYTES, 256, K::W1_PC, 256>(tD1, desc(s_base + K::OFF_X1, 128, X1::RG),
                                                               desc(s_base + K::OFF_W1, 128, W1::RG), idF, false);
                mma_commit(m_l1);
            };
            uint32_t p_x1 = 0, p_z2 = 0, p_dh1 = 0, p_dz1 = 0;
            bool iok    = iwait(r_x1, p_x1);
            bool wg_acc = false;
            if (iok) issue_l1();
            for (int64_t tile = T0; iok && tile < ntiles; tile += G)
            {
                // layer 2: A = h1's pieces in TMEM, B = W2 (K-major)
                if (!(iok = iwait(r_z2, p_z2))) break;
                gemm_ta<PREC, KS64, 32, K::W2_PC, 256>(tD2, tTA, desc(s_base + K::OFF_W2, 128, W2::RG), idF, false);
                mma_commit(m_z2);
                // dH1 = dz2 . W2 (B read MN-major, its pieces side by side: one MMA per A piece)
                if (!(iok = iwait(r_dh1, p_dh1))) break;
                gemm_cat<PREC, KS64, AB::BYTES, 256, (P::KI / 8) * W2::RG, HH, 0, 1>(
                    tD2, desc(s_base + K::OFF_AB, 128, AB::RG), desc(s_base + K::OFF_W2, W2::RG, 128), false);
                mma_commit(m_dh1);
                // dz1 in AB: the next tile's layer 1 (its Z1 columns were read
                // by the dz1 epilogue), this tile's dX into D2's first columns
                // (free until the next tile's layer 2; read before it), then
                // this tile's weight gradients
                if (!(iok = iwait(r_dz1, p_dz1))) break;
                if (tile + G < ntiles) issue_l1();
                gemm_cat<PREC, KS64, AB::BYTES, 256, (P::KI / 8) * W1::RG, K::K1, 0, 1>(
                    tD2, desc(s_base + K::OFF_AB + (HH / 8) * 128, 128, AB::RG),
                    desc(s_base + K::OFF_W1, W1::RG, 128), false);
                mma_commit(m_dx);
                gemm_cat<PREC, KS128, AB::BYTES, (P::KI / 8) * AB::RG, (P::KI / 8) * HB::RG, K::NW, 1, 1>(
                    tD4, desc(s_base + K::OFF_AB, AB::RG, 128), desc(s_base + K::OFF_HB, HB::RG, 128), wg_acc);
                mma_commit(m_wg);
                wg_acc = true;
            }
            // nothing of this CTA in flight past this point
            mma_commit(m_end);
            const bool drained = mbar_wait_bounded(m_end, 0);
            if (!iok || !drained) raise_status(a.status, NEAT_ERR_TIMEOUT);
        }
        __syncwarp();
    }
    fence_before();
    __syncthreads();
    if (w == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TMEM_COLS)
                     : "memory");
}

template <int C, int PREC, bool POSE>
static cudaError_t launch_bwd_rec_t(int grid, const StepTcArgs& args, cudaStream_t st)
{
    constexpr int smem = BwdRecPlan<C, PREC>::BYTES;
    static bool attr   = false;
    if (!attr)
    {
        cudaFuncSetAttribute(k_bwd_rec<C, PREC, POSE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    k_bwd_rec<C, PREC, POSE><<<grid, BR_THREADS, smem, st>>>(args);
    return cudaGetLastError();
}

template <int C, int PREC>
static cudaError_t launch_bwd_rec_p(int grid, const StepTcArgs& args, cudaStream_t st)
{
    return args.seg_pgrad != nullptr ? launch_bwd_rec_t<C, PREC, true>(grid, args, st)
                                     : launch_bwd_rec_t<C, PREC, false>(grid, args, st);
}

}  // namespace tc

// Three pieces: C = 4, 8 (at C = 16 the three dX blocks do not fit below the
// h1 pieces); one piece (BF16): C = 4, 8, 16.
bool bwd_rec_supported(int C, int prec)
{
    return prec == tc::BF16X3 ? (C == 4 || C == 8) : (C == 4 || C == 8 || C == 16);
}

cudaError_t launch_bwd_rec(int C, int prec, int grid, const StepTcArgs& args, cudaStream_t st)
{
    switch (C * 2 + prec)
    {
        case 4 * 2 + tc::BF16X3: return tc::launch_bwd_rec_p<4, tc::BF16X3>(grid, args, st);
        case 8 * 2 + tc::BF16X3: return tc::launch_bwd_rec_p<8, tc::BF16X3>(grid, args, st);
        case 4 * 2 + tc::BF16: return tc::launch_bwd_rec_p<4, tc::BF16>(grid, args, st);
        case 8 * 2 + tc::BF16: return tc::launch_bwd_rec_p<8, tc::BF16>(grid, args, st);
        case 16 * 2 + tc::BF16: return tc::launch_bwd_rec_p<16, tc::BF16>(grid, args, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace neat
