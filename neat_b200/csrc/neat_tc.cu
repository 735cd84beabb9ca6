// neat_tc.cu -- the fused step's sample tiles with the decoder GEMMs on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM).
//
// One CTA = one or two warpgroups; thread s (and s+128) owns slot s of the
// tile (TMEM lane s); with two warpgroups the 64 hidden units are split.  Per 128-sample tile:
//   layer 1 (C -> 64, SIMT fp32)  -> h1 row s written into HB (core-matrix layout)
//   Z2 = HB[:, :64] . W2^T          tcgen05 (A K-major, B K-major)          -> TMEM D2
//   epilogue: y, softplus, dy; dz2 = dy w3 silu'(z2) -> AB[:, :64]
//   dH1 = AB[:, :64] . W2           tcgen05 (A K-major, B = W2 read MN-major) -> TMEM D3
//   dz1 = dh1 silu'(z1) -> AB[:, 64:]; dx = dz1 . W1 -> grid scatter
//   [dW2|db2 ; dW1|db1] += AB^T . HB  tcgen05 (A and B MN-major, K = samples)
//                                    -> TMEM D4, accumulated over all tiles
// HB holds [h1 | x | 1] per sample row, so the weight-gradient GEMM yields the
// bias gradients from the ones column and dW1 from the x columns.  A row-major
// core-matrix buffer [row][col] is at the same time a K-major operand (M=row)
// and an MN-major operand (K=row): the reduction over samples reads the very
// buffers the forward GEMM used.
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
#include "neat_tiles.cuh"

namespace neat
{
namespace tc
{

enum
{
    BF16   = 0,
    BF16X3 = 1
};

template <int PREC>
struct Prec;
template <>
struct Prec<BF16>
{
    static constexpr int EB = 2, E = 8, KI = 16, PIECES = 1, FMT = 1, NPROD = 1;
};
template <>
struct Prec<BF16X3>
{
    static constexpr int EB = 2, E = 8, KI = 16, PIECES = 3, FMT = 1, NPROD = 6;
};
// products (a piece, b piece) with piece orders summing to <= 2
__device__ __constant__ int kProdA[6] = {0, 0, 1, 0, 1, 2};
__device__ __constant__ int kProdB[6] = {0, 1, 0, 2, 1, 0};

// Core-matrix ("interleaved", no swizzle) layout of a [ROWS][COLS] operand:
// 8 rows x 16 bytes per core matrix, core matrices of a row group contiguous
// along the columns, row groups RG bytes apart.
template <int PREC, int ROWS, int COLS>
struct Buf
{
    static constexpr int E     = Prec<PREC>::E;
    static constexpr int EB    = Prec<PREC>::EB;
    static constexpr int RG    = (COLS / E) * 128;
    static constexpr int BYTES = (ROWS / 8) * RG;
    static_assert(COLS % E == 0 && ROWS % 8 == 0, "operand tile must be whole core matrices");
    __device__ static __forceinline__ int off(int r, int c)
    {
        return (r >> 3) * RG + (c / E) * 128 + (r & 7) * 16 + (c % E) * EB;
    }
};

template <int C, int PREC, bool BWD>
struct Cfg
{
    using P                     = Prec<PREC>;
    static constexpr int XO     = HH;                     // x block in HB
    static constexpr int XW     = ((C + 7) / 8) * 8;
    static constexpr int OO     = XO + XW;                // ones column block
    static constexpr int NW     = ((OO + 8 + 15) / 16) * 16;
    static constexpr int HBC    = BWD ? NW : HH;          // HB columns
    using HB                    = Buf<PREC, 128, HBC>;
    using AB                    = Buf<PREC, 128, 2 * HH>;
    using W2                    = Buf<PREC, HH, HH>;
    static constexpr int OFF_W2 = 0;
    static constexpr int OFF_HB = OFF_W2 + P::PIECES * W2::BYTES;
    static constexpr int OFF_AB = OFF_HB + P::PIECES * HB::BYTES;
    static constexpr int OFF_F  = OFF_AB + (BWD ? P::PIECES * AB::BYTES : 0);
    static constexpr int NF     = HH * C + 3 * HH + 4;
    static constexpr int OFF_I  = OFF_F + NF * 4;
    static constexpr int OFF_V  = OFF_I + (2 * 128 + 128 + 2 * 132) * 4;
    static constexpr int OFF_R  = OFF_V + 2 * 128 * 4;
    static constexpr int NRED   = std::max(2 * 128 * C, 8 * HH);
    static constexpr int OFF_M  = ((OFF_R + NRED * 4) + 15) / 16 * 16;
    static constexpr int NEED   = OFF_M + 16;
    // BF16 backward: pad so that at most two CTAs share an SM (2 x 256 TMEM columns)
    static constexpr int BYTES = (PREC == BF16 && BWD) ? std::max(NEED, 100 * 1024) : NEED;
    static constexpr uint32_t TMEM_COLS = BWD ? 256 : 64;
    static_assert(!BWD || 128 + NW <= 256, "D4 must fit in the allocation");
};

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version 1 (sm_100); base offset 0, no swizzle
    return d;
}

__host__ __device__ constexpr uint32_t make_idesc(int fmt, int a_mn, int b_mn, int M, int N)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)a_mn << 15) |
           ((uint32_t)b_mn << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// One tcgen05.mma of kind::f16 (BF16 operands, FP32 accumulator in TMEM),
// issued by a single thread; acc = 0 overwrites D.
template <int FMT>
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    static_assert(FMT == 1, "BF16 operands only");
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity)
{
    const long long t0 = clock64();
    while (true)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 32)) return false;  // ~2 s at 2 GHz
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// operand pieces
// ---------------------------------------------------------------------------
// Store E = 8 consecutive values (one 16-byte chunk) as PIECES BF16 pieces,
// piece p at base + p * piece_bytes + off.
template <int PREC>
__device__ __forceinline__ void store_chunk(unsigned char* base, int piece_bytes, int off, const float* v)
{
    float r[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) r[i] = v[i];
#pragma unroll
    for (int p = 0; p < Prec<PREC>::PIECES; ++p)
    {
        __nv_bfloat162 b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            b[i] = __floats2bfloat162_rn(r[2 * i], r[2 * i + 1]);
            r[2 * i] -= __low2float(b[i]);      // exact: the remainder of a bf16 rounding
            r[2 * i + 1] -= __high2float(b[i]);
        }
        *reinterpret_cast<uint4*>(base + p * piece_bytes + off) = *reinterpret_cast<const uint4*>(b);
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Threads per CTA: 128 (one thread per sample) or 256 (two threads per sample
// splitting the hidden units; used where shared memory allows one CTA per SM).
template <int PREC, bool BWD>
struct TcThreads
{
    static constexpr int value = (PREC == BF16X3 && BWD) ? 256 : 128;
};

template <int C, int PREC, bool BWD>
__global__ void __launch_bounds__(TcThreads<PREC, BWD>::value, 1) k_step_tiles_tc(StepTcArgs a)
{
    using K  = Cfg<C, PREC, BWD>;
    using P  = Prec<PREC>;
    using HB = typename K::HB;
    using AB = typename K::AB;
    using W2 = typename K::W2;
    constexpr int TC_THREADS = TcThreads<PREC, BWD>::value;
    constexpr int NH         = TC_THREADS / 128;  // threads per sample
    constexpr int HALF       = HH / NH;           // hidden units per thread
    extern __shared__ __align__(128) unsigned char sm[];
    // thread t: sample (TMEM lane) s = t & 127, hidden part h = t >> 7
    const int t = threadIdx.x, w = t >> 5, l = t & 31, s = t & 127, h = t >> 7;
    const int c0 = h * HALF;  // first hidden column of this thread
    float* sW1    = reinterpret_cast<float*>(sm + K::OFF_F);
    float* sb1    = sW1 + HH * C;
    float* sb2    = sb1 + HH;
    float* sw3    = sb2 + HH;
    float* sb3    = sw3 + HH;
    int* marks    = reinterpret_cast<int*>(sm + K::OFF_I);  // [2][128] slot -> segment, double buffered
    int* slot_seg = marks + 2 * 128;                           // scan scratch
    int* starts   = slot_seg + 128;                            // [2][132] first sample of the tile's segments
    float* sval   = reinterpret_cast<float*>(sm + K::OFF_V);  // [2][128]: y halves / contributions
    float* sred   = reinterpret_cast<float*>(sm + K::OFF_R);  // [2][128][C] dx halves; end: reductions
    uint64_t* mbar_p = reinterpret_cast<uint64_t*>(sm + K::OFF_M);
    uint32_t* tslot  = reinterpret_cast<uint32_t*>(sm + K::OFF_M + 8);
    unsigned char* pW2 = sm + K::OFF_W2;
    unsigned char* pHB = sm + K::OFF_HB;
    unsigned char* pAB = sm + K::OFF_AB;
    const uint32_t s_base = smem_u32(sm);
    const uint32_t mbar   = smem_u32(mbar_p);

    // ---- decoder parameters: W1 / biases / w3 in fp32, W2 as MMA operand pieces
    using O = DecOff<C>;
    for (int i = t; i < HH * C; i += TC_THREADS) sW1[i] = a.decoder[O::W1 + i];
    for (int i = t; i < HH; i += TC_THREADS)
    {
        sb1[i] = a.decoder[O::b1 + i];
        sb2[i] = a.decoder[O::b2 + i];
        sw3[i] = a.decoder[O::W3 + i];
    }
    if (t == 0) sb3[0] = a.decoder[O::b3];
    for (int i = t; i < HH * HH; i += TC_THREADS)
    {
        const int off = W2::off(i / HH, i % HH);
        float r       = a.decoder[O::W2 + i];
#pragma unroll
        for (int p = 0; p < P::PIECES; ++p)
        {
            const __nv_bfloat16 b = __float2bfloat16_rn(r);
            *reinterpret_cast<__nv_bfloat16*>(pW2 + p * W2::BYTES + off) = b;
            r -= __bfloat162float(b);
        }
    }
    if (t == 0) mbar_init(mbar, 1);
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
    const uint32_t tD2 = tmem, tD3 = tmem + 64, tD4 = tmem + 128;

    const int nseg       = (int)a.counters[0];
    const int64_t S      = a.counters[1];
    const int64_t ntiles = (S + 127) / 128;
    uint32_t phase       = 0;
    bool ok              = true;
    bool wg_pending      = false;
    bool wg_started      = false;
    float dw3[BWD ? HALF : 1] = {};  // this thread's columns: sum over its samples of h2 * dy
    float db3                = 0.0f;

    auto wait_mma = [&]() -> bool {
        const bool mine = mbar_wait_bounded(mbar, phase);
        phase ^= 1u;
        const bool all = __syncthreads_and(mine) != 0;
        fence_after();
        return all;
    };
    constexpr uint32_t idF  = make_idesc(P::FMT, 0, 0, 128, HH);
    constexpr uint32_t idH  = make_idesc(P::FMT, 0, 1, 128, HH);
    constexpr uint32_t idW  = make_idesc(P::FMT, 1, 1, 128, K::NW);
    constexpr int KS64      = HH / P::KI;
    constexpr int KS128     = 128 / P::KI;

    // Tile set-up in two stages, run one tile ahead inside the MMA waits:
    // A: slot -> segment map (tile_seg, segment starts, block scan) into buffer b;
    // B: the slot's segment record, its sample and the grid gather.
    auto stage_a = [&](int64_t tl, int b) {
        tile_slot_segments(tl * 128, a.tile_seg[tl], nseg, a.samp_off, marks + 128 * b, slot_seg, starts + 132 * b);
    };
    auto stage_b = [&](int64_t tl, int b, SlotSample& qq, float* xx) {
        const int* mk    = marks + 128 * b;
        const int seg    = mk[s];
        const int64_t gs = tl * 128 + s;
        const bool valid = gs < S;
        const SegRec r   = a.segs[seg];
        const int j      = valid ? (int)(gs - starts[132 * b + (seg - mk[0])]) : 0;
        qq               = slot_sample(r, j, valid, a.jitter != 0, a.seed, a.step);
        Corners kc;
        igs_corners(qq.lu, qq.lv, qq.lw, a.G, a.G, a.G, kc);
        gather_cl<C>(a.grid, qq.row, a.G, kc, xx);
    };
    int buf = 0;
    SlotSample q;
    float x[C];
    if (blockIdx.x < ntiles)
    {
        stage_a(blockIdx.x, 0);
        stage_b(blockIdx.x, 0, q, x);
    }
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int64_t nxt   = tile + gridDim.x;
        const bool has_next = nxt < ntiles;
        const int* mark     = marks + 128 * buf;
        SlotSample qn;
        float xn[C];
        if (!q.valid)
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = 0.0f;
        if (BWD && wg_pending)
        {
            wg_pending = false;
            if (!wait_mma())
            {
                ok = false;
                break;
            }
        }
        // ---- HB row s: h1 columns of this half; half 0 adds [x | 1 0 ..]
#pragma unroll 1
        for (int k0 = c0; k0 < c0 + HALF; k0 += P::E)
        {
            float hv[P::E];
#pragma unroll
            for (int i = 0; i < P::E; ++i)
            {
                float z = sb1[k0 + i];
#pragma unroll
                for (int c = 0; c < C; ++c) z = fmaf(x[c], sW1[(k0 + i) * C + c], z);
                hv[i] = siluf_(z);
            }
            store_chunk<PREC>(pHB, HB::BYTES, HB::off(s, k0), hv);
        }
        if constexpr (BWD)
        {
            if (h == 0)
            {
#pragma unroll
                for (int cc = 0; cc < K::XW + 8; cc += P::E)
                {
                    float v[P::E];
#pragma unroll
                    for (int i = 0; i < P::E; ++i)
                    {
                        const int c = cc + i;
                        v[i]        = (c < C) ? x[c] : ((c == K::XW) ? 1.0f : 0.0f);
                    }
                    store_chunk<PREC>(pHB, HB::BYTES, HB::off(s, K::XO + cc), v);
                }
            }
            if (h == NH - 1)
            {
                for (int cc = K::OO + 8; cc < K::NW; cc += P::E)
                {
                    float v[P::E] = {};
                    store_chunk<PREC>(pHB, HB::BYTES, HB::off(s, cc), v);
                }
            }
        }
        fence_smem_async();
        fence_before();
        __syncthreads();
        // ---- Z2 = h1 . W2^T
        if (t == 0)
        {
            fence_after();
#pragma unroll 1
            for (int p = 0; p < P::NPROD; ++p)
                for (int kk = 0; kk < KS64; ++kk)
                {
                    const uint32_t ab = s_base + K::OFF_HB + kProdA[p] * HB::BYTES + kk * 256;
                    const uint32_t bb = s_base + K::OFF_W2 + kProdB[p] * W2::BYTES + kk * 256;
                    mma<P::FMT>(tD2, sdesc(ab, 128, HB::RG), sdesc(bb, 128, W2::RG), idF, (p | kk) ? 1u : 0u);
                }
            mma_commit(mbar);
        }
        if (has_next)
        {
            stage_a(nxt, buf ^ 1);
            if constexpr (!BWD) stage_b(nxt, buf ^ 1, qn, xn);
        }
        if (!wait_mma())
        {
            ok = false;
            break;
        }
        // ---- epilogue 1: y = b3 + sum over both halves
        {
            float yp = 0.0f;
#pragma unroll 1
            for (int j = 0; j < HALF / 16; ++j)
            {
                float z[16];
                tmem_ld16(tD2 + lane + c0 + 16 * j, z);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    yp = fmaf(siluf_(z[i] + sb2[c0 + 16 * j + i]), sw3[c0 + 16 * j + i], yp);
            }
            sval[h * 128 + s] = yp;
        }
        fence_before();
        __syncthreads();
        const float y = sb3[0] + sval[s] + (NH == 2 ? sval[128 + s] : 0.0f);
        if constexpr (!BWD)
        {
            __syncthreads();  // both halves read the y parts before they are overwritten
            if (h == 0) sval[s] = q.valid ? softplusf_(y, a.beta) * q.weight : 0.0f;
            __syncthreads();
            if (h == 0 && q.valid)
            {
                const int seg = mark[s];
                if (s == 0 || mark[s - 1] != seg)
                {
                    double sum = 0.0;  // f64: independent of where the tile boundary splits the segment
                    for (int u = s; u < 128 && mark[u] == seg; ++u) sum += (double)sval[u];
                    atomicAdd(a.partial + q.rm, sum);
                }
            }
            __syncthreads();
        }
        else
        {
            const float dv = q.valid ? a.dpred[q.ray] : 0.0f;
            const float dy = dv * q.weight * softplus_grad(y, a.beta);
            if (h == 0) db3 += dy;
            // dz2 (this half's columns) -> AB[:, c0:c0+32]; dW3 += h2 dy
#pragma unroll
            for (int j = 0; j < HALF / 16; ++j)
            {
                float z[16];
                tmem_ld16(tD2 + lane + c0 + 16 * j, z);
                float d[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                {
                    const int col  = c0 + 16 * j + i;
                    const float zz = z[i] + sb2[col];
                    const float sg = sigmoidf_(zz);
                    d[i]           = dy * sw3[col] * (sg * (1.0f + zz * (1.0f - sg)));
                    dw3[16 * j + i] = fmaf(zz * sg, dy, dw3[16 * j + i]);
                }
#pragma unroll
                for (int i = 0; i < 16; i += P::E) store_chunk<PREC>(pAB, AB::BYTES, AB::off(s, c0 + 16 * j + i), d + i);
            }
            fence_smem_async();
            fence_before();
            __syncthreads();
            // ---- dH1 = dz2 . W2  (B = W2 read MN-major: N = k, K = h)
            if (t == 0)
            {
                fence_after();
#pragma unroll 1
                for (int p = 0; p < P::NPROD; ++p)
                    for (int kk = 0; kk < KS64; ++kk)
                    {
                        const uint32_t ab = s_base + K::OFF_AB + kProdA[p] * AB::BYTES + kk * 256;
                        const uint32_t bb = s_base + K::OFF_W2 + kProdB[p] * W2::BYTES + kk * (P::KI / 8) * W2::RG;
                        mma<P::FMT>(tD3, sdesc(ab, 128, AB::RG), sdesc(bb, W2::RG, 128), idH, (p | kk) ? 1u : 0u);
                    }
                mma_commit(mbar);
            }
            if (has_next) stage_b(nxt, buf ^ 1, qn, xn);
            if (!wait_mma())
            {
                ok = false;
                break;
            }
            // ---- epilogue 2: dz1 (this half's k) -> AB[:, 64+c0 ..]; dx partial
            float dx[C];
#pragma unroll
            for (int c = 0; c < C; ++c) dx[c] = 0.0f;
#pragma unroll 1
            for (int j = 0; j < HALF / 16; ++j)
            {
                float g[16];
                tmem_ld16(tD3 + lane + c0 + 16 * j, g);
                float d[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                {
                    const int k = c0 + 16 * j + i;
                    float z     = sb1[k];
#pragma unroll
                    for (int c = 0; c < C; ++c) z = fmaf(x[c], sW1[k * C + c], z);
                    d[i] = g[i] * silu_grad(z);
#pragma unroll
                    for (int c = 0; c < C; ++c) dx[c] = fmaf(d[i], sW1[k * C + c], dx[c]);
                }
#pragma unroll
                for (int i = 0; i < 16; i += P::E)
                    store_chunk<PREC>(pAB, AB::BYTES, AB::off(s, HH + c0 + 16 * j + i), d + i);
            }
            if constexpr (NH == 2)
#pragma unroll
                for (int c = 0; c < C; ++c) sred[(h * 128 + s) * C + c] = dx[c];
            fence_smem_async();
            fence_before();
            __syncthreads();
            // ---- [dW2|db2 ; dW1|db1] += AB^T . HB   (K = samples)
            if (t == 0)
            {
                fence_after();
#pragma unroll 1
                for (int p = 0; p < P::NPROD; ++p)
                    for (int kk = 0; kk < KS128; ++kk)
                    {
                        const uint32_t ab = s_base + K::OFF_AB + kProdA[p] * AB::BYTES + kk * (P::KI / 8) * AB::RG;
                        const uint32_t bb = s_base + K::OFF_HB + kProdB[p] * HB::BYTES + kk * (P::KI / 8) * HB::RG;
                        const uint32_t acc = (wg_started || p || kk) ? 1u : 0u;
                        mma<P::FMT>(tD4, sdesc(ab, AB::RG, 128), sdesc(bb, HB::RG, 128), idW, acc);
                    }
                mma_commit(mbar);
            }
            wg_started = true;
            wg_pending = true;
            // dx of sample s (both halves when split; each half scatters four corners)
            if (q.valid)
            {
                Corners kc;
                igs_corners(q.lu, q.lv, q.lw, a.G, a.G, a.G, kc);
                if constexpr (NH == 2)
                {
#pragma unroll
                    for (int c = 0; c < C; ++c) dx[c] = sred[s * C + c] + sred[(128 + s) * C + c];
                    scatter_cl_half<C>(a.grid_grad, q.row, a.G, kc, dx, h);
                }
                else
                {
                    scatter_cl<C>(a.grid_grad, q.row, a.G, kc, dx);
                }
            }
            __syncthreads();  // sred / sval reused by the next tile
        }
        if (has_next)
        {
            q = qn;
#pragma unroll
            for (int c = 0; c < C; ++c) x[c] = xn[c];
        }
        buf ^= 1;
    }
    // ---- drain
    if (BWD && wg_pending)
    {
        if (!wait_mma()) ok = false;
    }
    if (!ok) raise_status(a.status, NEAT_ERR_TIMEOUT);
    if constexpr (BWD)
    {
        // per-CTA decoder-gradient partial (deterministic layout); row s of D4,
        // columns split between the halves
        float* dst = a.dec_part + (int64_t)blockIdx.x * O::total;
        constexpr int NCH = K::NW / 16;
#pragma unroll 1
        for (int j = h; j < NCH; j += NH)
        {
            float v[16];
            if (wg_started && ok)
                tmem_ld16(tD4 + lane + 16 * j, v);
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
                    if (n == K::OO) dst[O::b2 + s] = v[i];
                }
                else
                {
                    const int k = s - HH;
                    if (n >= K::XO && n < K::XO + C) dst[O::W1 + k * C + (n - K::XO)] = v[i];
                    if (n == K::OO) dst[O::b1 + k] = v[i];
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

template <int C, int PREC, bool BWD>
static int tc_grid(size_t& smem)
{
    using K = Cfg<C, PREC, BWD>;
    smem    = K::BYTES;
    static int blocks = 0;
    if (blocks == 0)
    {
        cudaFuncSetAttribute(k_step_tiles_tc<C, PREC, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        // TMEM: 512 columns per SM shared by the resident CTAs
        blocks = resident_ctas((const void*)k_step_tiles_tc<C, PREC, BWD>, TcThreads<PREC, BWD>::value, smem, (int)(512 / K::TMEM_COLS)) *
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
        const int g = tc_grid<C, PREC, true>(smem);
        k_step_tiles_tc<C, PREC, true><<<g, TcThreads<PREC, true>::value, smem, st>>>(args);
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
