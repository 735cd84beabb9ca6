// neat_scan.cuh -- exclusive prefix sum of int32 counts into int32/int64
// offsets, three launches (block scan, scan of block sums, add), with the
// element count taken either from the host or from a device int64 (counts
// produced earlier on the same stream, so no host synchronisation).
#pragma once

#include "neat_common.cuh"

namespace neat
{

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS   = 8;
constexpr int SCAN_TILE    = SCAN_THREADS * SCAN_ITEMS;  // 2048 elements per block

int sm_count();  // the device's SM count (neat_step.cu)

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* warp_tot, T& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0)
    {
        T w = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : (T)0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_tot[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    T before = (wid > 0) ? warp_tot[wid - 1] : (T)0;
    total    = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__device__ __forceinline__ int64_t scan_count(const int64_t* n_dev, int64_t n_host)
{
    return n_dev ? *n_dev : n_host;
}

template <typename TO>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_blocks(const int* __restrict__ in, const int64_t* n_dev,
                                                               int64_t n_host, TO* __restrict__ out,
                                                               TO* __restrict__ block_sums)
{
    __shared__ TO warp_tot[SCAN_THREADS / 32];
    const int64_t n = scan_count(n_dev, n_host);
    // grid-stride over the 2048-element tiles (uniform per block); the grid is
    // sized for the SMs, n_max only bounds it
    for (int64_t b = blockIdx.x; b * SCAN_TILE < n; b += gridDim.x)
    {
        const int64_t base = b * SCAN_TILE;
        TO loc[SCAN_ITEMS];
        TO sum = 0;
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i)
        {
            int64_t idx = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
            TO v        = (idx < n) ? (TO)in[idx] : (TO)0;
            loc[i]      = sum;
            sum += v;
        }
        TO total;
        TO pre = block_exclusive_scan<TO>(sum, warp_tot, total);  // ends with a barrier: warp_tot reusable
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i)
        {
            int64_t idx = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
            if (idx < n) out[idx] = pre + loc[i];
        }
        if (threadIdx.x == 0) block_sums[b] = total;
    }
}

// One block: exclusive scan of the block sums in place; writes the grand
// total to out[n] (so offsets have n+1 entries) and to total64 if given.
template <typename TO>
__global__ void __launch_bounds__(1024) k_scan_sums(TO* __restrict__ block_sums, const int64_t* n_dev, int64_t n_host,
                                                    TO* __restrict__ out, int64_t* total64)
{
    __shared__ TO warp_tot[32];
    const int64_t n  = scan_count(n_dev, n_host);
    const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    TO carry         = 0;
    for (int64_t b0 = 0; b0 < nb; b0 += 1024)
    {
        int64_t i = b0 + threadIdx.x;
        TO v      = (i < nb) ? block_sums[i] : (TO)0;
        TO total;
        TO pre = block_exclusive_scan<TO>(v, warp_tot, total);
        if (i < nb) block_sums[i] = carry + pre;
        carry += total;
    }
    if (threadIdx.x == 0)
    {
        out[n] = carry;
        if (total64) *total64 = (int64_t)carry;
    }
}

template <typename TO>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(TO* __restrict__ out, const int64_t* n_dev, int64_t n_host,
                                                            const TO* __restrict__ block_sums)
{
    const int64_t n = scan_count(n_dev, n_host);
    for (int64_t b = blockIdx.x; b * SCAN_TILE < n; b += gridDim.x)
    {
        const int64_t base = b * SCAN_TILE;
        const TO add       = block_sums[b];
        for (int i = threadIdx.x; i < SCAN_TILE; i += SCAN_THREADS)
        {
            int64_t idx = base + i;
            if (idx < n) out[idx] += add;
        }
    }
}

// One block for a short array (n <= SCAN_SINGLE): block scan of 8 elements a
// thread, out[n] = total (and total64): one launch instead of three.
constexpr int SCAN_SINGLE_THREADS = 1024;
constexpr int64_t SCAN_SINGLE     = (int64_t)SCAN_SINGLE_THREADS * SCAN_ITEMS;

template <typename TO>
__global__ void __launch_bounds__(SCAN_SINGLE_THREADS) k_scan_single(const int* __restrict__ in, const int64_t* n_dev,
                                                                     int64_t n_host, TO* __restrict__ out,
                                                                     int64_t* total64)
{
    __shared__ TO warp_tot[32];
    const int64_t n = scan_count(n_dev, n_host);  // <= SCAN_SINGLE (checked on the host)
    TO loc[SCAN_ITEMS];
    TO sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
    {
        const int64_t idx = (int64_t)threadIdx.x * SCAN_ITEMS + i;
        const TO v        = (idx < n) ? (TO)in[idx] : (TO)0;
        loc[i]            = sum;
        sum += v;
    }
    TO total;
    const TO pre = block_exclusive_scan<TO>(sum, warp_tot, total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
    {
        const int64_t idx = (int64_t)threadIdx.x * SCAN_ITEMS + i;
        if (idx < n) out[idx] = pre + loc[i];
    }
    if (threadIdx.x == 0)
    {
        out[n] = total;
        if (total64) *total64 = (int64_t)total;
    }
}

// Scratch (in elements of TO) needed for a scan of at most n_max elements.
inline int64_t scan_scratch_elems(int64_t n_max) { return (n_max + SCAN_TILE - 1) / SCAN_TILE + 1; }

// Exclusive scan of in[0..n) into out[0..n], out[n] = total.  n is *n_dev if
// n_dev != NULL (n_max bounds the launch), else n_max.
template <typename TO>
inline cudaError_t scan_exclusive(const int* in, const int64_t* n_dev, int64_t n_max, TO* out, TO* scratch,
                                  int64_t* total64, cudaStream_t st)
{
    if (n_max <= SCAN_SINGLE)
    {
        k_scan_single<TO><<<1, SCAN_SINGLE_THREADS, 0, st>>>(in, n_dev, n_max, out, total64);
        return cudaGetLastError();
    }
    int64_t nb = (n_max + SCAN_TILE - 1) / SCAN_TILE;
    if (nb < 1) nb = 1;
    nb = nb < (int64_t)sm_count() * 4 ? nb : (int64_t)sm_count() * 4;
    k_scan_blocks<TO><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n_dev, n_max, out, scratch);
    k_scan_sums<TO><<<1, 1024, 0, st>>>(scratch, n_dev, n_max, out, total64);
    k_scan_add<TO><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(out, n_dev, n_max, scratch);
    return cudaGetLastError();
}

}  // namespace neat
