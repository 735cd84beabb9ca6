// neat_tc.cu -- the fused step's sample tiles with the decoder GEMMs on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM).
//
// One CTA = one or two warpgroups; thread s (and s+128) owns slot s of the
// tile (TMEM lane s); with two warpgroups the 64 hidden units are split.
// Per 128-sample tile (HB row s = [h1 | x | 1 0 ..], AB row s = [dz2 | dz1]):
//   Z1 = HB[:, x|1] . [W1 | b1]^T      tcgen05 (A, B K-major)           -> TMEM D1
//   h1 = silu(Z1) -> HB[:, :64]
//   Z2 = HB[:, :64] . W2^T              tcgen05 (A, B K-major)           -> TMEM D2
//   epilogue: y, softplus (forward: contribution and per-segment sums)
// backward, continuing:
//   dz2 = dy w3 silu'(z2) -> AB[:, :64]
//   dH1 = AB[:, :64] . W2               tcgen05 (B = W2 read MN-major)   -> TMEM D2
//   dz1 = dH1 silu'(Z1) -> AB[:, 64:]   (Z1 still in D1: no recompute)
//   dX  = AB[:, 64:] . [W1 | b1]        tcgen05 (B read MN-major)        -> TMEM D2
//   [dW2|db2 ; dW1|db1] += AB^T . HB    tcgen05 (A and B MN-major, K = samples)
//                                       -> TMEM D4, accumulated over all tiles
//   dX scattered into the grid gradient with the trilinear corner weights.
// The ones column of HB folds b1 into the layer-1 GEMM and yields the bias
// gradients in the weight-gradient GEMM.  A row-major core-matrix buffer
// [row][col] is at the same time a K-major operand (M=row) and an MN-major
// operand (K=row): the reduction over samples reads the very buffers the
// forward GEMMs used, and one [W1 | b1] buffer serves layer 1 and dX.
//
// Precision policies (both on kind::f16 with BF16 operands, FP32 accumulation):
//   BF16X3: every operand split x = x0 + x1 + x2 into three BF16 pieces
//           (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1), 24
//           significant bits in all); the six products with piece orders
//           summing to <= 2 are accumulated, dropping terms below 2^-23 of
//           the product: FP32-level accuracy for the plain path.
//   BF16:   operands rounded to BF16 (the precision variant).
// All mbarrier waits are bounded (clock64 budget); on timeout the CTA raises
// NEAT_ERR_TIMEOUT, stops issuing work, drains with a bounded wait and frees
// its TMEM.
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

// POSE (backward only): also the camera pose gradient terms of every sample
// (a.seg_pgrad); a separate instantiation, so the plain step's code is unchanged.
template <int C, int PREC, bool BWD, bool POSE = false>
__global__ void __launch_bounds__(TcThreads<PREC, BWD>::value, TcThreads<PREC, BWD>::min_blocks)
    k_step_tiles_tc(StepTcArgs a)
{
    using K  = Cfg<C, PREC, BWD>;
    using P  = Prec<PREC>;
    using HB = typename K::HB;
    using X1 = typename K::X1;
    using AB = typename K::AB;
    using W2 = typename K::W2;
    using W1 = typename K::W1;
    constexpr int TC_THREADS = TcThreads<PREC, BWD>::value;
    constexpr int NH         = K::NH;     // threads per sample
    constexpr int HALF       = HH / NH;   // hidden units per thread
    constexpr bool PIPE      = BWD && K::NX1 == 1;   // pipelined backward
    constexpr bool FPIPE     = !BWD && K::NX1 == 1;  // pipelined forward
    // backward with two threads per sample: the next tile's placement runs in
    // the layer-2 window, its gather in the dH1 window (one thread per sample:
    // both in the dH1 window)
    constexpr bool SPLIT_B   = BWD && TcThreads<PREC, BWD>::value == 256;
    // forward with two threads per sample: its own loop (below)
    constexpr bool FSPLIT    = FPIPE && TcThreads<PREC, BWD>::value == 256;
    // epilogue chunk loops unrolled where the registers allow (two threads per sample, backward)
    constexpr int UNR        = SPLIT_B ? HALF / 16 : 1;
    extern __shared__ __align__(128) unsigned char sm[];
    // thread t: sample (TMEM lane) s = t & 127, hidden part h = t >> 7
    // the records backward (k_bwd_rec) has taken this step's tiles
    if (BWD && a.rec_skip && a.rec != nullptr && a.counters[1] <= a.rec_cap) return;
    const int t = threadIdx.x, w = t >> 5, l = t & 31, s = t & 127, h = t >> 7;
    const int c0 = h * HALF;  // first hidden column of this thread
    // The thread that issues every MMA.  A tcgen05.mma of these shapes holds
    // its issuing thread for about its execution time (44-60 cycles), so with
    // two threads per sample the issuer sits in the second half (warp 4),
    // which has no slot set-up to do while the layer-2 and dH1 GEMMs run.
    const bool issuer = t == (NH == 2 ? 128 : 0);
    float* sb2    = reinterpret_cast<float*>(sm + K::OFF_F);
    float* sw3    = sb2 + HH;
    float* sb3    = sw3 + HH;
    int* starts   = reinterpret_cast<int*>(sm + K::OFF_I);  // [2][132] first sample of the tile's segments
    double* wsum  = reinterpret_cast<double*>(starts + 2 * 132);  // forward: per warp, its first run's sum
    int* wseg     = reinterpret_cast<int*>(wsum + 4);              // .. that run's segment
    int* wlast    = wseg + 4;                                      // .. and the segment of its last slot
    float* sval   = reinterpret_cast<float*>(sm + K::OFF_V);  // [2][128]: y halves / contributions
    float* sq     = reinterpret_cast<float*>(sm + K::OFF_Q);  // [2][6][128]: lu, lv, lw, weight, ray, row
    float* sred   = reinterpret_cast<float*>(sm + K::OFF_R);  // end-of-kernel reductions
    uint64_t* mbar_p = reinterpret_cast<uint64_t*>(sm + K::OFF_M);
    uint32_t* tslot  = reinterpret_cast<uint32_t*>(sm + K::OFF_M + 16);
    unsigned char* pW2 = sm + K::OFF_W2;
    unsigned char* pW1 = sm + K::OFF_W1;
    unsigned char* pHB = sm + K::OFF_HB;
    unsigned char* pAB = sm + K::OFF_AB;
    const uint32_t s_base  = smem_u32(sm);
    const uint32_t mbar    = smem_u32(mbar_p);      // layer GEMMs
    const uint32_t mbar_wg = smem_u32(mbar_p + 1);  // forward: layer 1 of the next tile (pipelined)
    const uint32_t mbar_dx = smem_u32(mbar_p + 3);  // backward: dX

    // ---- decoder parameters: b2 / w3 / b3 in fp32, [W1 | b1] and W2 as MMA operand pieces
    using O = DecOff<C>;
    for (int i = t; i < HH; i += TC_THREADS)
    {
        sb2[i] = a.decoder[O::b2 + i];
        sw3[i] = a.decoder[O::W3 + i];
    }
    if (t == 0) sb3[0] = a.decoder[O::b3];
    for (int i = t; i < HH * HH + HH * K::K1; i += TC_THREADS)
    {
        float r;
        int off;
        unsigned char* dst;
        int piece_bytes;
        if (i < HH * HH)
        {
            r           = a.decoder[O::W2 + i];
            off         = W2::off(i / HH, i % HH);
            dst         = pW2;
            piece_bytes = K::W2_PC;
        }
        else
        {
            const int e = i - HH * HH, hr = e / K::K1, col = e % K::K1;
            r           = col < C ? a.decoder[O::W1 + hr * C + col] : (col == K::ONE ? a.decoder[O::b1 + hr] : 0.0f);
            off         = W1::off(hr, col);
            dst         = pW1;
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
        mbar_init(mbar, 1);
        mbar_init(mbar_wg, 1);
        mbar_init(mbar_dx, 1);
    }
    if (w == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(K::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t lane = (uint32_t)((w & 3) * 32) << 16;  // TMEM lane quadrant of this warp
    const uint32_t tD1 = tmem, tD2 = tmem + 64, tD4 = tmem + K::D4, tD3 = tmem + K::D3;
    const uint32_t tH2 = tmem + 128;  // activation cache (K::CACHE)
    constexpr bool CACHE = K::CACHE;

    const int nseg         = (int)a.counters[0];
    const int64_t S        = a.counters[1];
    const int64_t ntiles   = (S + 127) / 128;
    const uint32_t step_no = a.step_dev ? (uint32_t)*a.step_dev : a.step;
    uint32_t phase         = 0;
    uint32_t phase_wg      = 0;
    uint32_t phase_dx      = 0;
    bool ok              = true;
    bool wg_pending      = false;
    bool wg_started      = false;
    float dw3[BWD ? HALF : 1] = {};  // this thread's columns: sum over its samples of h2 * dy
    float db3                = 0.0f;

    auto wait_on = [&](uint32_t bar, uint32_t& ph) -> bool {
        const bool mine = mbar_wait_bounded(bar, ph);
        ph ^= 1u;
        const bool all = __syncthreads_and(mine) != 0;
        fence_after();
        return all;
    };
    // this thread's own bounded wait (none after a failure; the loop goes on
    // so that every barrier sees all threads)
    auto wait_own = [&](uint32_t bar, uint32_t& ph) -> bool {
        const bool mine = ok && mbar_wait_bounded(bar, ph);
        ph ^= 1u;
        fence_after();
        return mine;
    };
    constexpr uint32_t idF  = make_idesc(P::FMT, 0, 0, 128, HH);       // layers 1 and 2
    constexpr uint32_t idW  = make_idesc(P::FMT, 1, 1, 128, K::NW);    // weight gradients
    constexpr int KS1       = K::K1 / P::KI;
    constexpr int KS64      = HH / P::KI;
    constexpr int KS128     = 128 / P::KI;
    auto x1_addr = [&](int b) -> uint32_t { return s_base + K::OFF_X1 + b * K::X1SZ; };

    // Tile set-up, run one tile ahead inside the MMA waits.  The sample
    // offsets of the 129 segments from tile_seg[tile] on (the segments that
    // can own one of the tile's 128 slots) are fetched into registers a tile
    // ahead of use (fetch_starts) and put into the starts buffer of that tile
    // before a barrier (put_starts); stage_b then finds each slot's segment by
    // a binary search over them, loads its segment record, draws its sample
    // and gathers its grid features (first thread of a sample only).
    auto fetch_starts = [&](int lo, int& oa, int& ob) {
        oa = INT_MAX;
        ob = INT_MAX;
        if (t <= 128 && lo + t < nseg) oa = a.samp_off[lo + t];
        if (TC_THREADS == 128 && t == 0 && lo + 128 < nseg) ob = a.samp_off[lo + 128];
    };
    auto put_starts = [&](int b, int oa, int ob) {
        if (t <= 128) starts[132 * b + t] = oa;
        if (TC_THREADS == 128 && t == 0) starts[132 * b + 128] = ob;
    };
    struct Slot
    {
        SlotSample q;
        float x[C];
        float dvw;  // backward: dL/dpred of the sample's ray times its weight (0 when invalid)
        int seg;    // the slot's segment (-1 when the slot is past the last sample)
    };
    // stage_b in two parts: place_b (segment, record, sample position) and
    // gather_b (grid features, dL/dpred); the backward runs them in different
    // MMA windows.
    struct Place
    {
        SlotSample q;
        int seg;
    };
    auto place_b = [&](int64_t tl, int b, int lo) -> Place {
        Place o;
        const int* st    = starts + 132 * b;
        const int64_t gs = tl * 128 + s;
        const bool valid = gs < S;
        // last segment starting at or before the slot: st[0] <= tl * 128 by
        // construction of tile_seg, the segments past the last hold INT_MAX, and
        // an empty segment shares its start with the next one
        int i = 0;
#pragma unroll
        for (int d = 128; d > 0; d >>= 1)
            if (i + d <= 128 && (int64_t)st[i + d] <= gs) i += d;
        const int seg    = lo + i;
        const SegRec r   = a.segs[seg];
        const int j      = valid ? (int)(gs - st[i]) : 0;
        o.seg            = valid ? seg : -1;
        o.q              = slot_sample_warp(r, j, valid, a.jitter != 0, a.seed, step_no,
                                            a.seg_cdf ? a.seg_cdf + 8 * (int64_t)seg : nullptr, a.seg_hist != nullptr);
        return o;
    };
    auto gather_b = [&](const Place& pl) -> Slot {
        Slot o;
        o.q              = pl.q;
        o.seg            = pl.seg;
        const bool valid = pl.q.valid;
        Corners kc;
        igs_corners(o.q.lu, o.q.lv, o.q.lw, a.G, a.G, a.G, kc);
        if (a.grid_bf16)
            gather_cl_bf16<C>(a.grid_bf16, o.q.row, a.G, kc, o.x);
        else
            gather_cl<C>(a.grid, o.q.row, a.G, kc, o.x);
        if (!valid)
#pragma unroll
            for (int c = 0; c < C; ++c) o.x[c] = 0.0f;
        o.dvw = (BWD && valid) ? a.dpred[o.q.ray] * o.q.weight : 0.0f;
        return o;
    };
    auto stage_b = [&](int64_t tl, int b, int lo) -> Slot { return gather_b(place_b(tl, b, lo)); };
    // Forward, two threads per sample (K::STG): the corner rows of a sample
    // placed a tile ahead are copied into shared memory by cp.async when the
    // tile before it starts, and gathered from there after its h1 epilogue --
    // the L2 round trip runs under the epilogue.  Each thread stages and reads
    // only its own sample's slots, so its own cp.async.wait_all orders them.
    // Same products in the same order as gather_cl: the same features.
    const bool use_stg = K::STG && a.grid_bf16 == nullptr;
    float4* stg        = reinterpret_cast<float4*>(sm + K::OFF_STG);
    auto stage_corners = [&](const Place& pl) {
        if constexpr (K::STG)
        {
            Corners kc;
            igs_corners(pl.q.lu, pl.q.lv, pl.q.lw, a.G, a.G, a.G, kc);
            const int64_t base = (int64_t)pl.q.row * a.G * a.G * a.G;
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                const float* src = a.grid + (base + corner_cell(kc, q, a.G, a.G)) * C;
#pragma unroll
                for (int c4 = 0; c4 < C / 4; ++c4) cp_async16(smem_u32(stg + (q * (C / 4) + c4) * 128 + s), src + 4 * c4);
            }
            cp_async_commit();
        }
    };
    auto gather_staged = [&](const Place& pl) -> Slot {
        Slot o;
        o.q   = pl.q;
        o.seg = pl.seg;
        o.dvw = 0.0f;
        if constexpr (K::STG)
        {
            Corners kc;
            igs_corners(o.q.lu, o.q.lv, o.q.lw, a.G, a.G, a.G, kc);
            cp_async_wait_all();
#pragma unroll
            for (int c4 = 0; c4 < C / 4; ++c4)
            {
                float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                {
                    const float4 v = stg[(q * (C / 4) + c4) * 128 + s];
                    a0             = fmaf(v.x, kc.w[q], a0);
                    a1             = fmaf(v.y, kc.w[q], a1);
                    a2             = fmaf(v.z, kc.w[q], a2);
                    a3             = fmaf(v.w, kc.w[q], a3);
                }
                o.x[4 * c4]     = a0;
                o.x[4 * c4 + 1] = a1;
                o.x[4 * c4 + 2] = a2;
                o.x[4 * c4 + 3] = a3;
            }
            if (!o.q.valid)
#pragma unroll
                for (int c = 0; c < C; ++c) o.x[c] = 0.0f;
        }
        return o;
    };
    // placement records in shared memory (slot s), see K::OFF_P
    float* prec = reinterpret_cast<float*>(sm + K::OFF_P);
    auto store_p = [&](const Place& pl) {
        if constexpr (K::NP > 0)
        {
            prec[0 * 128 + s] = pl.q.weight;
            prec[1 * 128 + s] = pl.q.lu;
            prec[2 * 128 + s] = pl.q.lv;
            prec[3 * 128 + s] = pl.q.lw;
            prec[4 * 128 + s] = pl.q.t;
            prec[5 * 128 + s] = __int_as_float(pl.q.ray);
            prec[6 * 128 + s] = __int_as_float(pl.q.rm);
            prec[7 * 128 + s] = __int_as_float(pl.q.row);
            prec[8 * 128 + s] = __int_as_float(pl.seg);
            prec[9 * 128 + s] = pl.q.u;
        }
    };
    // Per-sample records (a.rec): the forward stores the slot set-up of every
    // sample it runs (placement and gathered features), the backward loads it
    // instead of recomputing it.  Coalesced: field f of sample i at f * rec_cap + i.
    const bool rec_ok = a.rec != nullptr && S <= a.rec_cap;
    auto write_rec = [&](const Slot& sl, int64_t tl) {
        const int64_t i = tl * 128 + s;
        if (!rec_ok || i >= S) return;
        const int64_t cp = a.rec_cap;
        float* r         = a.rec;
        r[0 * cp + i]    = sl.q.lu;
        r[1 * cp + i]    = sl.q.lv;
        r[2 * cp + i]    = sl.q.lw;
        r[3 * cp + i]    = sl.q.weight;
        r[4 * cp + i]    = sl.q.t;
        r[5 * cp + i]    = __int_as_float(sl.q.ray);
        r[6 * cp + i]    = __int_as_float(sl.q.row);
        r[7 * cp + i]    = __int_as_float(sl.seg);
#pragma unroll
        for (int c = 0; c < C; ++c) r[(8 + c) * cp + i] = sl.x[c];
    };
    auto read_rec = [&](int64_t tl) -> Slot {
        Slot o;
        const int64_t i = tl * 128 + s;
        const bool valid = i < S;
        o.q.valid        = valid;
        o.q.u            = 0.0f;
        o.q.rm           = 0;
        if (valid)
        {
            const int64_t cp = a.rec_cap;
            const float* r   = a.rec;
            o.q.lu           = __ldcs(r + 0 * cp + i);
            o.q.lv           = __ldcs(r + 1 * cp + i);
            o.q.lw           = __ldcs(r + 2 * cp + i);
            o.q.weight       = __ldcs(r + 3 * cp + i);
            o.q.t            = __ldcs(r + 4 * cp + i);
            o.q.ray          = __float_as_int(__ldcs(r + 5 * cp + i));
            o.q.row          = __float_as_int(__ldcs(r + 6 * cp + i));
            o.seg            = __float_as_int(__ldcs(r + 7 * cp + i));
#pragma unroll
            for (int c = 0; c < C; ++c) o.x[c] = __ldcs(r + (8 + c) * cp + i);
            o.dvw = a.dpred[o.q.ray] * o.q.weight;
        }
        else
        {
            o.q.lu = o.q.lv = o.q.lw = o.q.weight = o.q.t = 0.0f;
            o.q.ray = o.q.row = 0;
            o.seg             = -1;
#pragma unroll
            for (int c = 0; c < C; ++c) o.x[c] = 0.0f;
            o.dvw = 0.0f;
        }
        return o;
    };
    auto load_p = [&]() -> Place {
        Place pl = {};
        if constexpr (K::NP > 0)
        {
            pl.q.weight = prec[0 * 128 + s];
            pl.q.lu     = prec[1 * 128 + s];
            pl.q.lv     = prec[2 * 128 + s];
            pl.q.lw     = prec[3 * 128 + s];
            pl.q.t      = prec[4 * 128 + s];
            pl.q.ray    = __float_as_int(prec[5 * 128 + s]);
            pl.q.rm     = __float_as_int(prec[6 * 128 + s]);
            pl.q.row    = __float_as_int(prec[7 * 128 + s]);
            pl.seg      = __float_as_int(prec[8 * 128 + s]);
            pl.q.u      = prec[9 * 128 + s];
            pl.q.valid  = pl.seg >= 0;
        }
        return pl;
    };
    // Row s of an [x | 1 | 0 ..] block: the separate buffer b (b >= 0) or the
    // columns [64, 64 + K1) of HB (b < 0).
    auto put_x1 = [&](const float (&xv)[C], int b) {
        unsigned char* base = b >= 0 ? sm + K::OFF_X1 + b * K::X1SZ : pHB;
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
    // Slot data the second thread of a sample needs (backward), into buffer qb.
    auto put_q = [&](const Slot& sl, int qb) {
        if constexpr (K::NQ > 0)
        {
            float* qd       = sq + qb * 6 * 128;
            qd[0 * 128 + s] = sl.q.lu;
            qd[1 * 128 + s] = sl.q.lv;
            qd[2 * 128 + s] = sl.q.lw;
            qd[3 * 128 + s] = sl.dvw;
            qd[4 * 128 + s] = __int_as_float(sl.q.valid ? sl.q.ray : -1);
            qd[5 * 128 + s] = __int_as_float(sl.q.row);
        }
    };
    // layer 1 from the separate buffer b (pipelined) or from HB's [x | 1] columns
    // (the pipelined forward signals layer 1 on mbar_wg: its layer 2 is still
    // pending on mbar, and one barrier must never run two phases ahead of its waiter)
    auto issue_l1 = [&](int b) {
        if constexpr (PIPE || FPIPE)
            gemm<PREC, KS1, X1::BYTES, 256, K::W1_PC, 256>(tD1, sdesc(x1_addr(b), 128, X1::RG),
                                                           sdesc(s_base + K::OFF_W1, 128, W1::RG), idF, false);
        else
            gemm<PREC, KS1, K::HB_PC, 256, K::W1_PC, 256>(tD1, sdesc(s_base + K::OFF_HB + (HH / 8) * 128, 128, HB::RG),
                                                          sdesc(s_base + K::OFF_W1, 128, W1::RG), idF, false);
        mma_commit(FPIPE ? mbar_wg : mbar);
    };
    // dX of this tile (registers), scattered with the trilinear weights; each
    // thread of a sample takes 8 / NH corners.
    auto scatter_dx = [&](const float (&dx)[C], const SlotSample& q, int qb) {
        float lu, lv, lw;
        int row;
        bool valid;
        if (h == 0)
        {
            lu = q.lu; lv = q.lv; lw = q.lw; row = q.row; valid = q.valid;
        }
        else
        {
            const float* qd = sq + qb * 6 * 128;
            lu    = qd[0 * 128 + s];
            lv    = qd[1 * 128 + s];
            lw    = qd[2 * 128 + s];
            valid = __float_as_int(qd[4 * 128 + s]) >= 0;
            row   = __float_as_int(qd[5 * 128 + s]);
        }
        if (valid)
        {
            Corners kc;
            igs_corners(lu, lv, lw, a.G, a.G, a.G, kc);
            if constexpr (NH == 2)
            {
                // constant halves keep the corner arrays in registers
                if (h == 0)
                    scatter_cl_half<C>(a.grid_grad, row, a.G, kc, dx, 0);
                else
                    scatter_cl_half<C>(a.grid_grad, row, a.G, kc, dx, 1);
            }
            else
            {
                scatter_cl<C>(a.grid_grad, row, a.G, kc, dx);
            }
        }
    };

    // Camera pose gradients of one sample (first thread of the sample): with
    // g_q = sum_c grid_q[c] dX[c] over the 8 corners (re-read: the gather summed
    // them into x), dL/d(ix, iy, iz) = sum_q g_q dw_q/d(ix, iy, iz) -- the
    // IGS uv gradient before its (W-1)/2 scale -- and t times it; summed over
    // the warp's runs of one segment, one atomic per run into seg_pgrad.
    auto pose_sample = [&](const float (&dx)[C], const SlotSample& q, int seg) {
        float g[6] = {};
        if (q.valid)
        {
            Corners kc;
            igs_corners(q.lu, q.lv, q.lw, a.G, a.G, a.G, kc);
            const float ax0 = __fsub_rn((float)(kc.x0 + 1), kc.ix), ax1 = __fsub_rn(kc.ix, (float)kc.x0);
            const float ay0 = __fsub_rn((float)(kc.y0 + 1), kc.iy), ay1 = __fsub_rn(kc.iy, (float)kc.y0);
            const float az0 = __fsub_rn((float)(kc.z0 + 1), kc.iz), az1 = __fsub_rn(kc.iz, (float)kc.z0);
            const int64_t base = (int64_t)q.row * a.G * a.G * a.G;
#pragma unroll
            for (int qq = 0; qq < 8; ++qq)
            {
                const int64_t cell = (base + corner_cell(kc, qq, a.G, a.G)) * C;
                float gq = 0.0f;
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
            g[3] = g[0] * q.t;
            g[4] = g[1] * q.t;
            g[5] = g[2] * q.t;
        }
        const int sg = q.valid ? seg : -1;
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
        if (q.valid && (l == 0 || sp != sg))
#pragma unroll
            for (int k = 0; k < 6; ++k) atomicAdd(a.seg_pgrad + 6 * (int64_t)seg + k, g[k]);
    };

    int it = 0;
    if constexpr (FSPLIT)
    {
        // Forward with two threads per sample.  Per tile: layer 1 (issued a
        // tile ahead) -> h1 epilogue -> layer 2, while the first half gathers
        // the next tile's grid features (placed a tile earlier) and queues its
        // layer 1 -> y epilogue -> the second half sums the contributions per
        // segment (slot records of the first half, in sq) while the first half
        // places the tile after next.
        auto put_sr = [&](const Slot& sl, int qb) {
            float* qd       = sq + qb * 6 * 128;
            qd[0 * 128 + s] = sl.q.weight;
            qd[1 * 128 + s] = sl.q.u;
            qd[2 * 128 + s] = __int_as_float(sl.q.rm);
            qd[3 * 128 + s] = __int_as_float(sl.seg);
        };
        const int64_t T0 = blockIdx.x, G = gridDim.x;
        Place pl_next;  // first half: placement of the next tile
        pl_next.q.valid = false;
        pl_next.seg     = -1;
        int lo_n2       = 0;  // tile_seg two tiles ahead
        if (T0 < ntiles)
        {
            const int lo0 = a.tile_seg[T0];
            int oa, ob;
            fetch_starts(lo0, oa, ob);
            put_starts(0, oa, ob);
            const bool has1 = T0 + G < ntiles;
            const int lo1   = has1 ? a.tile_seg[T0 + G] : 0;
            if (has1)
            {
                fetch_starts(lo1, oa, ob);
                put_starts(1, oa, ob);
            }
            __syncthreads();
            if (h == 0)
            {
                const Slot c0s = gather_b(place_b(T0, 0, lo0));
                put_x1(c0s.x, 0);
                put_sr(c0s, 0);
                write_rec(c0s, T0);
            }
            fence_smem_async();
            fence_before();
            __syncthreads();
            if (issuer)
            {
                fence_after();
                issue_l1(0);
            }
            if (has1 && h == 0) pl_next = place_b(T0 + G, 1, lo1);
            if (T0 + 2 * G < ntiles) lo_n2 = a.tile_seg[T0 + 2 * G];
        }
        for (int64_t tile = T0; tile < ntiles; tile += G, ++it)
        {
            const int64_t nxt = tile + G, nxt2 = nxt + G;
            const bool has_next = nxt < ntiles, has_next2 = nxt2 < ntiles;
            const int buf       = it & 1;  // [x | 1] buffer and slot records of this tile
            // segment starts of the tile after next (stored before the barrier
            // ahead of its placement) and the tile_seg of the one after that
            int oa2 = INT_MAX, ob2 = INT_MAX;
            // the next tile's corner rows into shared memory, under this tile's h1 epilogue
            if (use_stg && has_next && h == 0) stage_corners(pl_next);
            if (has_next2) fetch_starts(lo_n2, oa2, ob2);
            const int lo_n3 = nxt2 + G < ntiles ? a.tile_seg[nxt2 + G] : 0;
            ok = wait_own(mbar_wg, phase_wg) && ok;
            // ---- h1 = silu(Z1), this thread's columns -> layer-2 A operand: TMEM
            //      (TA: BF16 pieces, two per column) or HB[:, c0 .. c0 + HALF)
#pragma unroll 1
            for (int j = 0; j < HALF / 16; ++j)
            {
                float z[16];
                tmem_ld16(tD1 + lane + c0 + 16 * j, z);
                if constexpr (K::TA)
                {
                    float2 hz[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                    {
                        const float2 zz = make_float2(z[2 * i], z[2 * i + 1]);
                        hz[i]           = __fmul2_rn(zz, sigmoid2<PREC>(zz));
                    }
#pragma unroll
                    for (int p = 0; p < P::PIECES; ++p)
                    {
                        uint32_t v[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) v[i] = piece2(hz[i]);
                        tmem_st8(tmem + lane + K::TA_COL + 32 * p + (c0 + 16 * j) / 2, v);
                    }
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < 16; ++i) z[i] = silu1<PREC>(z[i]);
                    store_chunk<PREC>(pHB, K::HB_PC, HB::off(s, c0 + 16 * j), z);
                    store_chunk<PREC>(pHB, K::HB_PC, HB::off(s, c0 + 16 * j + 8), z + 8);
                }
            }
            if constexpr (K::TA) tmem_wait_st();
            fence_smem_async();
            fence_before();
            __syncthreads();
            // ---- Z2 = h1 . W2^T
            if (issuer)
            {
                fence_after();
                if constexpr (K::TA)
                    gemm_ta<PREC, KS64, 32, K::W2_PC, 256>(tD2, tmem + K::TA_COL,
                                                            sdesc(s_base + K::OFF_W2, 128, W2::RG), idF, false);
                else
                    gemm<PREC, KS64, K::HB_PC, 256, K::W2_PC, 256>(tD2, sdesc(s_base + K::OFF_HB, 128, HB::RG),
                                                                    sdesc(s_base + K::OFF_W2, 128, W2::RG), idF, false);
                mma_commit(mbar);
            }
            // ---- the next tile: grid gather, slot records, layer 1 (queued behind layer 2)
            if (has_next)
            {
                if (h == 0)
                {
                    const Slot nx = use_stg ? gather_staged(pl_next) : gather_b(pl_next);
                    put_x1(nx.x, 0);
                    put_sr(nx, buf ^ 1);
                    write_rec(nx, nxt);
                }
                fence_smem_async();
                fence_before();
                __syncthreads();
                if (issuer)
                {
                    fence_after();
                    issue_l1(0);
                }
            }
            ok = wait_own(mbar, phase) && ok;
            // ---- epilogue 1: this thread's part of y
            {
                float2 yp2 = make_float2(0.0f, 0.0f);
#pragma unroll 1
                for (int j = 0; j < HALF / 16; ++j)
                {
                    float z[16];
                    tmem_ld16(tD2 + lane + c0 + 16 * j, z);
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                    {
                        const int col   = c0 + 16 * j + 2 * i;
                        const float2 zz = __fadd2_rn(make_float2(z[2 * i], z[2 * i + 1]),
                                                     *reinterpret_cast<const float2*>(sb2 + col));
                        const float2 h2 = __fmul2_rn(zz, sigmoid2<PREC>(zz));
                        yp2             = __ffma2_rn(h2, *reinterpret_cast<const float2*>(sw3 + col), yp2);
                    }
                }
                sval[h * 128 + s] = yp2.x + yp2.y;
            }
            if (has_next2) put_starts(buf, oa2, ob2);
            fence_before();
            __syncthreads();
            if (h == 1)
            {
                // Per-segment sums of the contributions in f64, in a fixed order:
                // a segmented suffix scan inside each warp (a segment's slots are
                // consecutive), then a run's first slot adds the first runs of the
                // following warps that continue it.  One f64 atomic per segment
                // and tile (a segment spans at most two tiles: its two partials
                // commute), so the projection is reproducible.
                const float* qd = sq + buf * 6 * 128;
                const int seg   = __float_as_int(qd[3 * 128 + s]);
                const bool vld  = seg >= 0;
                const int rm    = __float_as_int(qd[2 * 128 + s]);
                const float y   = sb3[0] + sval[s] + sval[128 + s];
                const float c   = vld ? softplusf_(y, a.beta) * qd[s] : 0.0f;
                // proposal targets: contribution mass per eighth of the segment
                if (a.seg_hist && vld) atomicAdd(a.seg_hist + 8 * (int64_t)rm + min(7, (int)(qd[128 + s] * 8.0f)), c);
                // .. and each sample's density (the count head's variation target)
                if (a.seg_dens && vld && tile * 128 + s < a.dens_cap) a.seg_dens[tile * 128 + s] = softplusf_(y, a.beta);
                double v = (double)c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const double vn = __shfl_down_sync(0xffffffffu, v, o);
                    const int sn    = __shfl_down_sync(0xffffffffu, seg, o);
                    if (l + o < 32 && sn == seg) v += vn;
                }
                const int sp = __shfl_up_sync(0xffffffffu, seg, 1);
                const int wq = w & 3;
                if (l == 0)
                {
                    wsum[wq] = v;
                    wseg[wq] = seg;
                }
                if (l == 31) wlast[wq] = seg;
                asm volatile("bar.sync 1, 128;" ::: "memory");  // the 128 second threads of the samples
                const bool head = l == 0 ? (wq == 0 || wlast[wq - 1] != seg) : sp != seg;
                if (head && vld)
                {
                    for (int ww = wq + 1; ww < 4 && wseg[ww] == seg; ++ww) v += wsum[ww];
                    atomicAdd(a.partial + rm, v);
                }
            }
            else if (has_next2)
            {
                pl_next = place_b(nxt2, buf, lo_n2);
            }
            lo_n2 = lo_n3;
        }
    }
    else
    {
        Slot cur;
        cur.q.valid = false;
        cur.dvw     = 0.0f;
        cur.seg     = -1;
#pragma unroll
        for (int c = 0; c < C; ++c) cur.x[c] = 0.0f;
        int lo_next = 0;  // tile_seg of the next tile, loaded a tile ahead
        int lo_p2   = 0;  // SPLIT_B: tile_seg of the tile after next (placed this iteration)
        if (blockIdx.x < ntiles)
        {
            const int lo0 = a.tile_seg[blockIdx.x];
            int oa, ob;
            fetch_starts(lo0, oa, ob);
            put_starts(0, oa, ob);
            const bool has1 = blockIdx.x + gridDim.x < ntiles;
            const int lo1   = has1 ? a.tile_seg[blockIdx.x + gridDim.x] : 0;
            if (SPLIT_B && has1)
            {
                fetch_starts(lo1, oa, ob);
                put_starts(1, oa, ob);
            }
            __syncthreads();
            if (h == 0)
            {
                cur = (BWD && rec_ok) ? read_rec(blockIdx.x) : stage_b(blockIdx.x, 0, lo0);
                if (!BWD) write_rec(cur, blockIdx.x);
            }
            if constexpr (SPLIT_B)
            {
                // the next tile placed by the second half (its records read in the first layer-2 window)
                if (has1 && h == 1 && !rec_ok) store_p(place_b(blockIdx.x + gridDim.x, 1, lo1));
                if (blockIdx.x + 2 * gridDim.x < ntiles) lo_p2 = a.tile_seg[blockIdx.x + 2 * gridDim.x];
            }
            lo_next = lo1;
            if constexpr (PIPE || FPIPE)
            {
                if (h == 0)
                {
                    put_x1(cur.x, 0);
                    put_q(cur, 0);
                }
                fence_smem_async();
                fence_before();
                __syncthreads();
                if (issuer)
                {
                    fence_after();
                    issue_l1(0);
                }
            }
        }
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it)
        {
            const int64_t nxt   = tile + gridDim.x;
            const bool has_next = nxt < ntiles;
            const int buf       = it & 1;                 // segment starts and slot data of this tile
            const SlotSample& q = cur.q;
            Slot nx;
            nx.q.valid = false;
            nx.dvw     = 0.0f;
            nx.seg     = -1;
            // the next tile's segment starts (stored before the barrier ahead of
            // its stage_b) and the tile_seg of the one after it; SPLIT_B: the same
            // one tile further ahead (the tile after next is placed here)
            const bool has_next2 = nxt + gridDim.x < ntiles;
            int oa_nx = INT_MAX, ob_nx = INT_MAX;
            if (!SPLIT_B && has_next) fetch_starts(lo_next, oa_nx, ob_nx);
            if (SPLIT_B && has_next2) fetch_starts(lo_p2, oa_nx, ob_nx);
            const int lo_nx2 = !SPLIT_B ? (has_next2 ? a.tile_seg[nxt + gridDim.x] : 0)
                                        : (nxt + 2 * gridDim.x < ntiles ? a.tile_seg[nxt + 2 * gridDim.x] : 0);
            // ---- without the pipelined layer 1: the previous tile's weight-gradient
            //      GEMM reads HB's [x | 1] columns, rewritten next
            if (BWD && wg_pending)
            {
                wg_pending = false;
                if constexpr (!PIPE)
                {
                    if (!wait_on(mbar, phase))
                    {
                        ok = false;
                        break;
                    }
                }
            }
            // ---- Z1 = [x | 1] . [W1 | b1]^T (already in flight when pipelined)
            if constexpr (!PIPE && !FPIPE)
            {
                if (h == 0)
                {
                    put_x1(cur.x, -1);
                    put_q(cur, buf);
                }
                fence_smem_async();
                fence_before();
                __syncthreads();
                if (issuer)
                {
                    fence_after();
                    issue_l1(0);
                }
            }
            if (!(FPIPE ? wait_on(mbar_wg, phase_wg) : wait_on(mbar, phase)))
            {
                ok = false;
                break;
            }
            // ---- h1 = silu(Z1), this thread's columns -> HB[:, c0 .. c0 + HALF)
#pragma unroll UNR
            for (int j = 0; j < HALF / 16; ++j)
            {
                float z[16];
                tmem_ld16(tD1 + lane + c0 + 16 * j, z);
                if constexpr (CACHE)
                {
                    float d1[16];  // silu'(z1) over z1, kept for the dz1 epilogue
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                    {
                        const float sg = sigmoid1<PREC>(z[i]);
                        d1[i]          = sg * (1.0f + z[i] * (1.0f - sg));
                        z[i]           = z[i] * sg;
                    }
                    tmem_st16(tD1 + lane + c0 + 16 * j, d1);
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < 16; ++i) z[i] = silu1<PREC>(z[i]);
                }
                store_chunk<PREC>(pHB, K::HB_PC, HB::off(s, c0 + 16 * j), z);
                store_chunk<PREC>(pHB, K::HB_PC, HB::off(s, c0 + 16 * j + 8), z + 8);
            }
            if constexpr (CACHE) tmem_wait_st();
            if (PIPE && h == 0) put_x1(cur.x, -1);  // HB's [x | 1] columns for the weight gradients
            if (!BWD && has_next) put_starts(buf ^ 1, oa_nx, ob_nx);
            fence_smem_async();
            fence_before();
            __syncthreads();
            // ---- Z2 = h1 . W2^T
            if (issuer)
            {
                fence_after();
                gemm<PREC, KS64, K::HB_PC, 256, K::W2_PC, 256>(tD2, sdesc(s_base + K::OFF_HB, 128, HB::RG),
                                                                 sdesc(s_base + K::OFF_W2, 128, W2::RG), idF, false);
                mma_commit(mbar);
            }
            if (!BWD && has_next && h == 0)
            {
                nx = stage_b(nxt, buf ^ 1, lo_next);
                write_rec(nx, nxt);
            }
            // backward, two threads per sample: the next tile's gather (placed a tile
            // ago by the second half) while layer 2 runs
            if constexpr (SPLIT_B)
            {
                if (has_next && h == 0)
                {
                    nx = rec_ok ? read_rec(nxt) : gather_b(load_p());
                    if constexpr (PIPE)
                    {
                        put_x1(nx.x, 0);  // the [x | 1] buffer's last reader, this tile's layer 1, is done
                        put_q(nx, buf ^ 1);
                    }
                }
            }
            if constexpr (FPIPE)
            {
                // the next tile's layer 1, queued behind this tile's layer 2 (the
                // [x | 1] buffer was last read by this tile's layer 1, completed)
                if (has_next)
                {
                    if (h == 0) put_x1(nx.x, 0);
                    fence_smem_async();
                    fence_before();
                    __syncthreads();
                    if (issuer)
                    {
                        fence_after();
                        issue_l1(0);
                    }
                }
            }
            if (!wait_on(mbar, phase))
            {
                ok = false;
                break;
            }
            // ---- epilogue 1: y = b3 + sum over both halves
            {
                float yp = 0.0f;
#pragma unroll UNR
                for (int j = 0; j < HALF / 16; ++j)
                {
                    float z[16];
                    tmem_ld16(tD2 + lane + c0 + 16 * j, z);
                    if constexpr (CACHE)
                    {
                        // h2 and w3 silu'(z2 + b2), kept for the dz2 epilogue
                        float g[16];
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                        {
                            const int col  = c0 + 16 * j + i;
                            const float zz = z[i] + sb2[col];
                            const float sg = sigmoid1<PREC>(zz);
                            z[i]           = zz * sg;
                            yp             = fmaf(z[i], sw3[col], yp);
                            g[i]           = sw3[col] * (sg * (1.0f + zz * (1.0f - sg)));
                        }
                        tmem_st16(tD2 + lane + c0 + 16 * j, g);
                        tmem_st16(tH2 + lane + c0 + 16 * j, z);
                    }
                    else
                    {
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            yp = fmaf(silu1<PREC>(z[i] + sb2[c0 + 16 * j + i]), sw3[c0 + 16 * j + i], yp);
                    }
                }
                if constexpr (CACHE) tmem_wait_st();
                sval[h * 128 + s] = yp;
            }
            fence_before();
            __syncthreads();
            const float y = sb3[0] + sval[s] + (NH == 2 ? sval[128 + s] : 0.0f);
            if constexpr (!BWD)
            {
                // Per-segment sums of the contributions in f64, in a fixed order:
                // a segmented suffix scan inside each warp (a segment's slots are
                // consecutive), then a run's first slot adds the first runs of the
                // following warps that continue it.  One f64 atomic per segment
                // and tile (a segment spans at most two tiles: its two partials
                // commute), so the projection is reproducible.
                if (h == 0)
                {
                    const float c = q.valid ? softplusf_(y, a.beta) * q.weight : 0.0f;
                    // proposal targets: contribution mass per eighth of the segment
                    if (a.seg_hist && q.valid) atomicAdd(a.seg_hist + 8 * (int64_t)q.rm + min(7, (int)(q.u * 8.0f)), c);
                    // .. and each sample's density (the count head's variation target)
                    if (a.seg_dens && q.valid && tile * 128 + s < a.dens_cap)
                        a.seg_dens[tile * 128 + s] = softplusf_(y, a.beta);
                    const int seg = cur.seg;
                    double v      = (double)c;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1)
                    {
                        const double vn = __shfl_down_sync(0xffffffffu, v, o);
                        const int sn    = __shfl_down_sync(0xffffffffu, seg, o);
                        if (l + o < 32 && sn == seg) v += vn;
                    }
                    const int sp = __shfl_up_sync(0xffffffffu, seg, 1);
                    if (l == 0)
                    {
                        wsum[w] = v;
                        wseg[w] = seg;
                    }
                    if (l == 31) wlast[w] = seg;
                    asm volatile("bar.sync 1, 128;" ::: "memory");  // the 128 first threads of the samples
                    const bool head = l == 0 ? (w == 0 || wlast[w - 1] != seg) : sp != seg;
                    if (head && q.valid)
                    {
                        for (int ww = w + 1; ww < 4 && wseg[ww] == seg; ++ww) v += wsum[ww];
                        atomicAdd(a.partial + q.rm, v);
                    }
                }
            }
            else
            {
                const float dvw = h == 0 ? cur.dvw : sq[buf * 6 * 128 + 3 * 128 + s];
                const float dy  = dvw * softplus_grad(y, a.beta);
                if (h == 0) db3 += dy;
                // dz2 (this thread's columns) -> AB[:, c0 ..]; dW3 += h2 dy
#pragma unroll
                for (int j = 0; j < HALF / 16; ++j)
                {
                    float d[16];
                    if constexpr (CACHE)
                    {
                        uint32_t g[16], h2[16];
                        tmem_ld16_async(tD2 + lane + c0 + 16 * j, g);
                        tmem_ld16_async(tH2 + lane + c0 + 16 * j, h2);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                        {
                            d[i]            = dy * __uint_as_float(g[i]);
                            dw3[16 * j + i] = fmaf(__uint_as_float(h2[i]), dy, dw3[16 * j + i]);
                        }
                    }
                    else
                    {
                        float z[16];
                        tmem_ld16(tD2 + lane + c0 + 16 * j, z);
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                        {
                            const int col   = c0 + 16 * j + i;
                            const float zz  = z[i] + sb2[col];
                            const float sg  = sigmoid1<PREC>(zz);
                            d[i]            = dy * sw3[col] * (sg * (1.0f + zz * (1.0f - sg)));
                            dw3[16 * j + i] = fmaf(zz * sg, dy, dw3[16 * j + i]);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 16; i += P::E) store_chunk<PREC>(pAB, AB::BYTES, AB::off(s, c0 + 16 * j + i), d + i);
                }
                if (!SPLIT_B && has_next) put_starts(buf ^ 1, oa_nx, ob_nx);
            if (SPLIT_B && has_next2) put_starts(buf, oa_nx, ob_nx);  // for the placement below
                fence_smem_async();
                fence_before();
                __syncthreads();
                // ---- dH1 = dz2 . W2  (B = W2 read MN-major: N = k, K = h) -> D2
                //      (two threads per sample: issued by warp 0, whose half has no
                //      work in this window; the second half places a tile meanwhile)
                if (SPLIT_B ? t == 0 : issuer)
                {
                    fence_after();
                    gemm_cat<PREC, KS64, AB::BYTES, 256, (P::KI / 8) * W2::RG, HH, 0, 1>(
                        tD2, sdesc(s_base + K::OFF_AB, 128, AB::RG), sdesc(s_base + K::OFF_W2, W2::RG, 128), false);
                    mma_commit(mbar);
                }
                if constexpr (SPLIT_B)
                {
                    // the tile after next: placement into the records (read by the
                    // next iteration's gather; this iteration's were read above)
                    if (has_next2 && h == 1 && !rec_ok) store_p(place_b(nxt + gridDim.x, buf, lo_p2));
                }
                else if (has_next && h == 0)
                {
                    nx = rec_ok ? read_rec(nxt) : stage_b(nxt, buf ^ 1, lo_next);
                    // the [x | 1] buffer was last read by this tile's layer 1,
                    // which has completed
                    if constexpr (PIPE)
                    {
                        put_x1(nx.x, 0);
                        put_q(nx, buf ^ 1);
                    }
                }
                if (!wait_on(mbar, phase))
                {
                    ok = false;
                    break;
                }
                // ---- epilogue 2: dz1 = dH1 silu'(Z1) (this thread's columns) -> AB[:, 64 + c0 ..]
#pragma unroll UNR
                for (int j = 0; j < HALF / 16; ++j)
                {
                    float g[16];
                    if constexpr (CACHE)
                    {
                        // dH1: one column block per W2 piece (gemm_cat), summed
                        // smallest first; times the cached silu'(z1)
                        uint32_t gr[P::PIECES][16], dr[16];
#pragma unroll
                        for (int p = 0; p < P::PIECES; ++p) tmem_ld16_async(tD2 + p * HH + lane + c0 + 16 * j, gr[p]);
                        tmem_ld16_async(tD1 + lane + c0 + 16 * j, dr);
                        tmem_wait_ld();
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                        {
                            float v = __uint_as_float(gr[P::PIECES - 1][i]);
#pragma unroll
                            for (int p = P::PIECES - 2; p >= 0; --p) v += __uint_as_float(gr[p][i]);
                            g[i] = v * __uint_as_float(dr[i]);
                        }
                    }
                    else
                    {
                        float z[16];
                        tmem_ld16(tD2 + lane + c0 + 16 * j, g);
                        tmem_ld16(tD1 + lane + c0 + 16 * j, z);
#pragma unroll
                        for (int i = 0; i < 16; ++i) g[i] *= silu_grad1<PREC>(z[i]);
                    }
#pragma unroll
                    for (int i = 0; i < 16; i += P::E)
                        store_chunk<PREC>(pAB, AB::BYTES, AB::off(s, HH + c0 + 16 * j + i), g + i);
                }
                fence_smem_async();
                fence_before();
                __syncthreads();
                // ---- dX = dz1 . [W1 | b1] -> D3, read into registers before the next
                //      GEMM is issued (a TMEM load waits while the tensor core
                //      accumulates into TMEM)
                if (issuer)
                {
                    fence_after();
                    gemm_cat<PREC, KS64, AB::BYTES, 256, (P::KI / 8) * W1::RG, K::K1, 0, 1>(
                        tD3, sdesc(s_base + K::OFF_AB + (HH / 8) * 128, 128, AB::RG), sdesc(s_base + K::OFF_W1, W1::RG, 128),
                        false);
                    mma_commit(mbar_dx);
                }
                if (!wait_on(mbar_dx, phase_dx))
                {
                    ok = false;
                    break;
                }
                float dx[C];
                {
                    uint32_t dxv[P::PIECES][16];  // one column block per [W1 | b1] piece
#pragma unroll
                    for (int p = 0; p < P::PIECES; ++p) tmem_ld16_async(tD3 + lane + p * K::K1, dxv[p]);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < C; ++c)
                    {
                        float v = __uint_as_float(dxv[0][c]);
#pragma unroll
                        for (int p = 1; p < P::PIECES; ++p) v += __uint_as_float(dxv[p][c]);
                        dx[c] = v;
                    }
                }
                fence_before();
                __syncthreads();
                // ---- [dW2 ; dW1 | db] += AB^T . [h1 | x 1] -> D4, then (pipelined) the
                //      next tile's layer 1 -> D1 (one signal on mbar for both)
                if (issuer)
                {
                    fence_after();
                    if constexpr (K::WCAT)
                        gemm_cat<PREC, KS128, AB::BYTES, (P::KI / 8) * AB::RG, (P::KI / 8) * HB::RG, K::NW, 1, 1>(
                            tD4, sdesc(s_base + K::OFF_AB, AB::RG, 128), sdesc(s_base + K::OFF_HB, HB::RG, 128), wg_started);
                    else
                        gemm<PREC, KS128, AB::BYTES, (P::KI / 8) * AB::RG, K::HB_PC, (P::KI / 8) * HB::RG>(
                            tD4, sdesc(s_base + K::OFF_AB, AB::RG, 128), sdesc(s_base + K::OFF_HB, HB::RG, 128), idW,
                            wg_started);
                    if (PIPE && has_next)
                        issue_l1(0);
                    else
                        mma_commit(mbar);
                }
                wg_started = true;
                wg_pending = true;
                // ---- this tile's dX scattered while the weight-gradient GEMM runs
                scatter_dx(dx, cur.q, buf);
                if constexpr (POSE)
                {
                    if (h == 0) pose_sample(dx, cur.q, cur.seg);
                }
            }
            if (has_next && h == 0) cur = nx;
            if constexpr (SPLIT_B)
                lo_p2 = lo_nx2;
            else
                lo_next = lo_nx2;
        }
    }
    // ---- drain: the last tile's weight gradients
    if (BWD && wg_pending)
    {
        if (!wait_on(mbar, phase)) ok = false;
    }
    if (!ok) raise_status(a.status, NEAT_ERR_TIMEOUT);
    if constexpr (BWD)
    {
        // per-CTA decoder-gradient partial (deterministic layout): row s of D4.
        // Rows < 64 (dz2 features): columns [0,64) dW2, column 64 + ONE db2;
        // rows >= 64 (dz1 features): columns 64 + c dW1, column 64 + ONE db1.
        float* dst = a.dec_part + (int64_t)blockIdx.x * O::total;
        constexpr int NCH = (HH + K::K1) / 16;
#pragma unroll 1
        for (int j = h; j < NCH; j += NH)
        {
            float v[16];
            if (wg_started && ok)
            {
                tmem_ld16(tD4 + lane + 16 * j, v);
                if constexpr (K::WCAT)  // one column block per HB piece
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
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.0f;
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
        // dW3: every thread holds its columns summed over its samples; reduce
        // over the 32 lanes (transpose-reduce) and then over the 4 warps of a part
        __syncthreads();
        {
            float v[HALF];
#pragma unroll
            for (int i = 0; i < HALF; ++i) v[i] = dw3[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
            {
#pragma unroll
                for (int i = 0; i < HALF; ++i)
                {
                    const float other = __shfl_xor_sync(0xffffffffu, v[i], o);
                    v[i] += other;
                }
            }
            // every lane holds the warp's sums; lane l writes columns c0 + l (+ 32)
#pragma unroll
            for (int i = 0; i < HALF; ++i)
                if ((i & 31) == l) sred[w * HH + c0 + i] = v[i];
        }
        const float b3w = warp_sum(db3);
        __syncthreads();
        if (t < HH)
        {
            const int part = t / HALF;
            float acc      = 0.0f;
            for (int ww = 4 * part; ww < 4 * part + 4; ++ww) acc += sred[ww * HH + t];
            dst[O::W3 + t] = acc;
        }
        __syncthreads();
        if (l == 0) sred[w] = b3w;
        __syncthreads();
        if (t == 0)
        {
            float acc = 0.0f;
            for (int ww = 0; ww < TC_THREADS / 32; ++ww) acc += sred[ww];
            dst[O::b3] = acc;
        }
    }
    fence_before();
    __syncthreads();
    if (w == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(K::TMEM_COLS)
                     : "memory");
}

template <int C, int PREC, bool BWD, bool POSE = false>
static int tc_grid(size_t& smem)
{
    using K = Cfg<C, PREC, BWD>;
    smem    = K::BYTES;
    static int blocks = 0;
    if (blocks == 0)
    {
        cudaFuncSetAttribute(k_step_tiles_tc<C, PREC, BWD, POSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        // TMEM: 512 columns per SM shared by the resident CTAs
        blocks = resident_ctas((const void*)k_step_tiles_tc<C, PREC, BWD, POSE>, TcThreads<PREC, BWD>::value, smem,
                               (int)(512 / K::TMEM_COLS)) *
                 sm_count();
    }
    return blocks;
}

template <int C, int PREC>
static cudaError_t launch(bool bwd, const StepTcArgs& args, cudaStream_t st)
{
    size_t smem = 0;
    if (!bwd)
    {
        const int g = tc_grid<C, PREC, false>(smem);
        k_step_tiles_tc<C, PREC, false><<<g, TcThreads<PREC, false>::value, smem, st>>>(args);
    }
    else
    {
        // the step's decoder partials are sized by the plain backward's grid
        const int g = tc_grid<C, PREC, true>(smem);
        StepTcArgs a2 = args;
        if (args.rec != nullptr && bwd_rec_supported(C, PREC))
        {
            // the records backward (one CTA per SM); the plain kernel below
            // then runs only when the step's samples exceed the records.  The
            // decoder partials have a row per CTA of the plain kernel's grid:
            // the rows past the records kernel's grid are zeroed first (the
            // plain kernel, when it runs, writes every row)
            const int gr          = std::min(g, sm_count());
            const cudaError_t e = launch_bwd_rec(C, PREC, gr, args, st);
            if (e != cudaSuccess) return e;
            if (gr < g)
            {
                const size_t row = (size_t)DecOff<C>::total;
                const cudaError_t z =
                    cudaMemsetAsync(args.dec_part + (size_t)gr * row, 0, (size_t)(g - gr) * row * sizeof(float), st);
                if (z != cudaSuccess) return z;
            }
            a2.rec_skip = 1;
        }
        if (args.seg_pgrad)
        {
            tc_grid<C, PREC, true, true>(smem);  // its shared-memory attribute
            k_step_tiles_tc<C, PREC, true, true><<<g, TcThreads<PREC, true>::value, smem, st>>>(a2);
        }
        else
        {
            k_step_tiles_tc<C, PREC, true><<<g, TcThreads<PREC, true>::value, smem, st>>>(a2);
        }
    }
    return cudaGetLastError();
}

}  // namespace tc

int tc_backward_grid(int C, int prec)
{
    size_t smem = 0;
    switch (C * 2 + prec)
    {
        case 4 * 2 + tc::BF16: return tc::tc_grid<4, tc::BF16, true>(smem);
        case 4 * 2 + tc::BF16X3: return tc::tc_grid<4, tc::BF16X3, true>(smem);
        case 8 * 2 + tc::BF16: return tc::tc_grid<8, tc::BF16, true>(smem);
        case 8 * 2 + tc::BF16X3: return tc::tc_grid<8, tc::BF16X3, true>(smem);
        case 16 * 2 + tc::BF16: return tc::tc_grid<16, tc::BF16, true>(smem);
        case 16 * 2 + tc::BF16X3: return tc::tc_grid<16, tc::BF16X3, true>(smem);
        default: return 0;
    }
}

cudaError_t launch_tiles_tc(int C, int prec, bool bwd, const StepTcArgs& args, cudaStream_t st)
{
    switch (C * 2 + prec)
    {
        case 4 * 2 + tc::BF16: return tc::launch<4, tc::BF16>(bwd, args, st);
        case 4 * 2 + tc::BF16X3: return tc::launch<4, tc::BF16X3>(bwd, args, st);
        case 8 * 2 + tc::BF16: return tc::launch<8, tc::BF16>(bwd, args, st);
        case 8 * 2 + tc::BF16X3: return tc::launch<8, tc::BF16X3>(bwd, args, st);
        case 16 * 2 + tc::BF16: return tc::launch<16, tc::BF16>(bwd, args, st);
        case 16 * 2 + tc::BF16X3: return tc::launch<16, tc::BF16X3>(bwd, args, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace neat
