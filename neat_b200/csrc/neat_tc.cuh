// neat_tc.cuh -- shared pieces of the tcgen05 tile kernels: BF16 piece
// policies, the no-swizzle core-matrix operand layout, the shared-memory and
// TMEM plan of a tile CTA, and PTX wrappers for tcgen05.mma / ld / st,
// mbarriers and the GEMM issue loops.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "neat_internal.h"
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
__host__ __device__ constexpr int prod_a(int p) { return p == 2 || p == 4 ? 1 : (p == 5 ? 2 : 0); }
__host__ __device__ constexpr int prod_b(int p) { return p == 1 || p == 4 ? 1 : (p == 3 ? 2 : 0); }

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

// Threads per CTA: 256 (two threads per sample splitting the hidden units)
// for the three-piece policy, 128 for BF16; and the CTAs per SM the
// register budget is sized for.
template <int PREC, bool BWD>
struct TcThreads
{
    static constexpr int value      = (PREC == BF16X3) ? 256 : 128;
    static constexpr int min_blocks = (PREC == BF16X3) ? (BWD ? 1 : 2) : (BWD ? 2 : 4);
};

// Shared-memory plan of a tile CTA.  Backward HB rows hold [h1 | x | 1 0 ..]
// (the weight-gradient B operand), forward HB rows h1.  HB and [W1 | b1] keep
// their BF16 pieces side by side along the columns (piece p at column
// p * width), so that one MMA multiplies an A piece by several B pieces at
// once (the weight-gradient and dX GEMMs; piece offsets HB_PC, W1_PC bytes);
// W2 [h][k] likewise (W2_PC; dH1 reads it with N = k across its pieces);
// AB and the [x | 1] buffer keep whole pieces one after the other.  NX1
// separate [x | 1] buffers (0 or 1): with one, the next tile's layer-1 GEMM is
// issued from it while the current tile is still in flight (backward: behind
// the weight-gradient GEMM; forward: behind layer 2); its rows are written
// after the current tile's layer 1 has completed.  TA (forward, two threads
// per sample, C <= 8): h1 is the A operand of layer 2 straight from TMEM (no
// HB; its BF16 pieces are written with tcgen05.st instead of shared stores).
template <int C, int PREC, bool BWD, int NX1_>
struct CfgPlan
{
    using P                     = Prec<PREC>;
    static constexpr int NX1    = NX1_;
    static constexpr int XW     = ((C + 7) / 8) * 8;          // x columns (C padded)
    static constexpr int K1     = ((XW + 1 + 15) / 16) * 16;  // layer-1 K: [x | 1 | 0 ..]
    static constexpr int ONE    = XW;                         // column of the 1 in [x | 1]
    static constexpr int NW     = HH + K1;                    // weight-gradient N: [h1 | x | 1 ..]
    static constexpr bool TA    = !BWD && TcThreads<PREC, BWD>::value == 256 && C <= 8;
    static constexpr int HBW    = BWD ? NW : (TA ? 0 : HH);   // HB columns of one piece (forward: h1 only)
    using HB                    = Buf<PREC, 128, P::PIECES * HBW>;
    using X1                    = Buf<PREC, 128, K1>;         // [x | 1 | 0 ..] rows
    using AB                    = Buf<PREC, 128, 2 * HH>;     // [dz2 | dz1] rows
    using W2                    = Buf<PREC, HH, P::PIECES * HH>;  // [h][k]: W2
    using W1                    = Buf<PREC, HH, P::PIECES * K1>;  // [h][x | 1]: W1 | b1
    static constexpr int HB_PC  = HBW * 16;                   // byte offset of the next piece's columns
    static constexpr int W1_PC  = K1 * 16;
    static constexpr int W2_PC  = HH * 16;
    static constexpr int NH     = TcThreads<PREC, BWD>::value / 128;
    static constexpr int OFF_W2 = 0;
    static constexpr int OFF_W1 = OFF_W2 + W2::BYTES;
    static constexpr int OFF_HB = OFF_W1 + W1::BYTES;
    static constexpr int OFF_X1 = OFF_HB + HB::BYTES;
    static constexpr int X1SZ   = P::PIECES * X1::BYTES;      // one [x | 1] buffer, all pieces
    static constexpr int OFF_AB = OFF_X1 + NX1 * X1SZ;
    static constexpr int OFF_F  = OFF_AB + (BWD ? P::PIECES * AB::BYTES : 0);
    static constexpr int NF     = 2 * HH + 4;                 // b2, w3, b3
    static constexpr int OFF_I  = OFF_F + NF * 4;             // [2][132] segment starts, then 4 f64 + 8 int
    static constexpr int OFF_V  = OFF_I + 2 * 132 * 4 + 4 * 8 + 8 * 4;
    static constexpr int OFF_Q  = OFF_V + 2 * 128 * 4;        // [2][6][128] slot data for the second thread (both directions)
    static constexpr int NQ     = (NH == 2) ? 2 * 6 * 128 : 0;
    // backward, two threads per sample: placement records of the next tile
    // [weight, lu, lv, lw, t, ray, rm, row, seg, u][128], written by the second
    // half, read by the first half's gather
    static constexpr int NP     = (BWD && NH == 2) ? 10 * 128 : 0;
    static constexpr int OFF_P  = OFF_Q + NQ * 4;
    static constexpr int OFF_R  = OFF_P + NP * 4;
    static constexpr int NRED   = BWD ? 8 * HH : 0;
    // forward with two threads per sample, C <= 8: the next tile's corner rows,
    // staged by cp.async while the current tile's h1 epilogue runs
    // ([8 corners][C / 4][128 samples] float4)
    static constexpr bool STG    = !BWD && NH == 2 && C <= 8 && C % 4 == 0;
    static constexpr int NSTG    = STG ? 8 * C * 128 : 0;  // floats
    static constexpr int OFF_STG = ((OFF_R + NRED * 4) + 15) / 16 * 16;
    static constexpr int OFF_M   = OFF_STG + NSTG * 4;
    static constexpr int NEED   = OFF_M + 32;                 // mbarriers at +0, +8, +24; TMEM slot at +16
};

template <int C, int PREC, bool BWD>
struct Cfg : CfgPlan<C, PREC, BWD, (CfgPlan<C, PREC, BWD, 1>::NEED <= 232448) ? 1 : 0>
{
    using Base = CfgPlan<C, PREC, BWD, (CfgPlan<C, PREC, BWD, 1>::NEED <= 232448) ? 1 : 0>;
    // TMEM columns: D1 [0,64) Z1; D2 [64,128) Z2 / dH1; backward: D4 weight
    // gradients (h1 columns, then [x | 1] columns; with WCAT one such block per B
    // piece, summed at the end), D3 dX (one block of K1 columns per B piece).
    // The three-piece backward (one CTA per SM) also caches activations: D1
    // holds silu'(z1) once Z1 is read, [128,192) h2 = silu(z2 + b2), and D2
    // w3 silu'(z2 + b2) between the y and dz2 epilogues.  Its dH1 takes one
    // 64-column block per W2 piece, [64,256), after the dz2 epilogue has read
    // h2; its D4 starts at 256 and its dX reuses dH1's last block when it fits
    // (read before dX).
    using PP                            = Prec<PREC>;
    static constexpr bool CACHE         = BWD && PREC == BF16X3;
    static constexpr bool WCAT          = PP::PIECES * Base::NW <= 256;  // one MMA per A piece
    static constexpr int D4             = CACHE ? 256 : 128;
    static constexpr int D4W            = WCAT ? PP::PIECES * Base::NW : Base::NW;
    static constexpr int D3W            = PP::PIECES * Base::K1;
    static constexpr int D3             = (CACHE && D3W <= 64) ? 192 : D4 + D4W;
    // forward with TA: h1 pieces as the layer-2 A operand at [128, 128 + 32 PIECES)
    // (two BF16 per 32-bit column)
    static constexpr int TA_COL         = 128;
    static constexpr uint32_t TMEM_COLS = CACHE ? 512 : ((BWD || Base::TA) ? 256 : 128);
    // pad so that no more CTAs share an SM than its 512 TMEM columns hold
    // (233472 B of shared memory per SM, 1 KB reserved per CTA)
    static constexpr int MIN_BYTES = 233472 / (512 / (int)TMEM_COLS + 1) - 1024 + 16;
    static constexpr int BYTES     = Base::NEED > MIN_BYTES ? Base::NEED : MIN_BYTES;
    static_assert(!BWD || (D4 + D4W <= (int)TMEM_COLS && D3 + D3W <= (int)TMEM_COLS), "D4 and D3 must fit");
    static_assert(!BWD || D3 + D3W <= D4 || D3 >= D4 + D4W, "dX must not overlap the weight gradients");
    static_assert(BYTES <= 232448, "shared-memory plan exceeds the per-CTA limit");
    static_assert((Base::OFF_I + 2 * 132 * 4) % 8 == 0, "f64 reduction scratch must be 8-byte aligned");
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

// tcgen05.mma with A in TMEM (K-major, two BF16 per 32-bit column) and B in
// shared memory.
__device__ __forceinline__ void mma_ta(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
        "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
// All MMAs of one GEMM (every piece product, every K step), fully unrolled:
// the operand descriptors advance by compile-time byte offsets (the start
// address field counts 16-byte units and never carries: shared addresses are
// below 2^18).  acc0: accumulate onto D from the first MMA on.
template <int PREC, int KS, int A_PIECE, int A_K, int B_PIECE, int B_K>
__device__ __forceinline__ void gemm(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, bool acc0)
{
    constexpr int NPROD = PREC == 1 ? 6 : 1;
#pragma unroll
    for (int p = 0; p < NPROD; ++p)
#pragma unroll
        for (int kk = 0; kk < KS; ++kk)
        {
            const uint64_t a = da + (uint64_t)((prod_a(p) * A_PIECE + kk * A_K) >> 4);
            const uint64_t b = db + (uint64_t)((prod_b(p) * B_PIECE + kk * B_K) >> 4);
            mma<1>(d, a, b, idesc, (acc0 || p || kk) ? 1u : 0u);
        }
}

// gemm() with A in TMEM: piece p of A at column offset p * A_PIECE_COLS, K
// steps of 16 elements = 8 columns.
template <int PREC, int KS, int A_PIECE_COLS, int B_PIECE, int B_K>
__device__ __forceinline__ void gemm_ta(uint32_t d, uint32_t a_tmem, uint64_t db, uint32_t idesc, bool acc0)
{
    constexpr int NPROD = PREC == 1 ? 6 : 1;
#pragma unroll
    for (int p = 0; p < NPROD; ++p)
#pragma unroll
        for (int kk = 0; kk < KS; ++kk)
        {
            const uint32_t a = a_tmem + (uint32_t)(prod_a(p) * A_PIECE_COLS + kk * 8);
            const uint64_t b = db + (uint64_t)((prod_b(p) * B_PIECE + kk * B_K) >> 4);
            mma_ta(d, a, b, idesc, (acc0 || p || kk) ? 1u : 0u);
        }
}

// A GEMM whose B operand holds its pieces side by side along N (NB columns
// each): per A piece p one MMA against B pieces 0 .. PIECES-1-p (N = (PIECES -
// p) NB), which puts the products of piece orders <= 2 into PIECES column
// blocks of D (block q: the products with B piece q; the reader sums them).
// Half the MMAs of gemm(), and each A piece is read once per K step.
template <int PREC, int KS, int A_PIECE, int A_K, int B_K, int NB, int A_MN, int B_MN>
__device__ __forceinline__ void gemm_cat(uint32_t d, uint64_t da, uint64_t db, bool acc0)
{
    constexpr int NP = Prec<PREC>::PIECES;
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int kk = 0; kk < KS; ++kk)
        {
            const uint64_t a = da + (uint64_t)((p * A_PIECE + kk * A_K) >> 4);
            const uint64_t b = db + (uint64_t)((kk * B_K) >> 4);
            mma<1>(d, a, b, make_idesc(Prec<PREC>::FMT, A_MN, B_MN, 128, (NP - p) * NB), (acc0 || p || kk) ? 1u : 0u);
        }
}

// cp.async (16 bytes, global -> shared, through L1); a thread waits for its own copies
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float v[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t v[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32 lanes x 16 columns into registers without waiting; tmem_wait_ld()
// before the values are used.
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t r[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x 8 columns into registers without waiting.
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t r[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
}

// One arrival on an mbarrier (release semantics at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint32_t mbar)
{
    asm volatile("{\n\t.reg .b64 mb_state;\n\tmbarrier.arrive.shared::cta.b64 mb_state, [%0];\n\t}" ::"r"(mbar) : "memory");
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
// Packed pairs of f32 (sm_100 f32x2 arithmetic, round to nearest).
__device__ __forceinline__ float2 neg1x2() { return make_float2(-1.0f, -1.0f); }
__device__ __forceinline__ float2 one2() { return make_float2(1.0f, 1.0f); }
// a - b (exact when the difference is representable, as a bf16 remainder is)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, neg1x2(), a); }

// sigma(z) of a pair of pre-activations for precision PREC.  BF16X3 keeps
// 1 / (1 + 2^(-z log2 e)) (ex2 + rcp, FP32-level).  BF16, whose GEMM operands
// carry 8 significant bits, uses sigma(z) = 1/2 + tanh(z/2) / 2 with one
// tanh.approx.f32 a value (relative error of tanh below 2^-10.9, so sigma is
// within 2^-11.9 absolute): one SFU op a value instead of two.  h = z sigma(z)
// then stays within |z| 2^-11.9, below the BF16 rounding of h (|h| 2^-9) for
// z > -2 and small against the layer's other activations below it.
template <int PREC>
__device__ __forceinline__ float2 sigmoid2(float2 z)
{
    if constexpr (PREC == BF16)
    {
        const float2 hz = __fmul2_rn(z, make_float2(0.5f, 0.5f));
        float2 th;
        asm("tanh.approx.f32 %0, %1;" : "=f"(th.x) : "f"(hz.x));
        asm("tanh.approx.f32 %0, %1;" : "=f"(th.y) : "f"(hz.y));
        return __ffma2_rn(th, make_float2(0.5f, 0.5f), make_float2(0.5f, 0.5f));
    }
    else
        return make_float2(sigmoidf_(z.x), sigmoidf_(z.y));
}
template <int PREC>
__device__ __forceinline__ float sigmoid1(float z)
{
    if constexpr (PREC == BF16)
    {
        float th;
        asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(0.5f * z));
        return fmaf(0.5f, th, 0.5f);
    }
    else
        return sigmoidf_(z);
}
template <int PREC>
__device__ __forceinline__ float silu1(float z)
{
    return z * sigmoid1<PREC>(z);
}
template <int PREC>
__device__ __forceinline__ float silu_grad1(float z)
{
    const float sg = sigmoid1<PREC>(z);
    return sg * (1.0f + z * (1.0f - sg));
}

// One BF16 piece of a pair: the packed bits, and the pair minus the piece
// (exact: the remainder of a bf16 rounding).
__device__ __forceinline__ uint32_t piece2(float2& r)
{
    const __nv_bfloat162 b = __floats2bfloat162_rn(r.x, r.y);
    r                      = sub2(r, make_float2(__low2float(b), __high2float(b)));
    return *reinterpret_cast<const uint32_t*>(&b);
}

// Store E = 8 consecutive values (one 16-byte chunk) as PIECES BF16 pieces,
// piece p at base + p * piece_bytes + off.
template <int PREC>
__device__ __forceinline__ void store_chunk(unsigned char* base, int piece_bytes, int off, const float* v)
{
    float2 r[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = make_float2(v[2 * i], v[2 * i + 1]);
#pragma unroll
    for (int p = 0; p < Prec<PREC>::PIECES; ++p)
    {
        uint32_t b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) b[i] = piece2(r[i]);
        *reinterpret_cast<uint4*>(base + p * piece_bytes + off) = make_uint4(b[0], b[1], b[2], b[3]);
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tc
}  // namespace neat
