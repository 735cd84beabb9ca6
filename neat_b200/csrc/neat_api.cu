// neat_api.cu -- small entry points: status strings, local coordinates,
// grid layout conversion.
#include "neat_common.cuh"

namespace neat
{

__global__ void k_local_samples(const float* __restrict__ g, const int64_t* __restrict__ node_id, int64_t S,
                                const float* __restrict__ nmin, const float* __restrict__ nmax,
                                float* __restrict__ out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int64_t n = node_id[s];
    for (int c = 0; c < 3; ++c) out[3 * s + c] = local_coord(g[3 * s + c], nmin[3 * n + c], nmax[3 * n + c]);
}

// [A, C, G3] <-> [A, G3, C]
__global__ void k_grid_transpose(const float* __restrict__ src, float* __restrict__ dst, int64_t A, int C, int64_t G3,
                                 int to_last)
{
    const int64_t i     = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = A * C * G3;
    if (i >= total) return;
    // i indexes the destination
    if (to_last)
    {
        const int c      = (int)(i % C);
        const int64_t v  = (i / C) % G3;
        const int64_t a  = i / (C * G3);
        dst[i]           = src[(a * C + c) * G3 + v];
    }
    else
    {
        const int64_t v = i % G3;
        const int c     = (int)((i / G3) % C);
        const int64_t a = i / (C * G3);
        dst[i]          = src[(a * G3 + v) * C + c];
    }
}

}  // namespace neat

using namespace neat;

extern "C" const char* neat_status_string(int status)
{
    if (status == NEAT_OK) return "ok";
    if (status & NEAT_ERR_BAD_INPUT) return "bad input (sizes or pointers)";
    if (status & NEAT_ERR_CUDA) return "CUDA launch failed";
    if (status & NEAT_ERR_UNSUPPORTED) return "unsupported configuration";
    if (status & NEAT_ERR_TOO_MANY_HITS) return "more than 256 ray-node intersections on one ray";
    if (status & NEAT_ERR_CAPACITY) return "output or workspace capacity exceeded";
    if (status & NEAT_ERR_NON_DYADIC) return "node box not on the dyadic plane grid of max_depth";
    if (status & NEAT_ERR_TIMEOUT) return "a bounded wait inside a kernel gave up";
    return "unknown status";
}

extern "C" int neat_version(void) { return 1; }

extern "C" int neat_local_samples(const float* global, const int64_t* node_id, int64_t num_samples,
                                  const float* node_min, const float* node_max, float* local, neat_stream_t stream)
{
    if (num_samples < 0) return NEAT_ERR_BAD_INPUT;
    if (num_samples == 0) return NEAT_OK;
    if (!global || !node_id || !node_min || !node_max || !local) return NEAT_ERR_BAD_INPUT;
    k_local_samples<<<(unsigned)((num_samples + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        global, node_id, num_samples, node_min, node_max, local);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

static int grid_convert(const float* src, float* dst, int64_t A, int C, int G, int to_last, cudaStream_t st)
{
    if (A < 0 || C < 1 || G < 1) return NEAT_ERR_BAD_INPUT;
    const int64_t total = A * C * (int64_t)G * G * G;
    if (total == 0) return NEAT_OK;
    if (!src || !dst || src == dst) return NEAT_ERR_BAD_INPUT;
    k_grid_transpose<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(src, dst, A, C, (int64_t)G * G * G, to_last);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_grid_to_channel_last(const float* src, float* dst, int64_t A, int C, int G, neat_stream_t stream)
{
    return grid_convert(src, dst, A, C, G, 1, (cudaStream_t)stream);
}

extern "C" int neat_grid_from_channel_last(const float* src, float* dst, int64_t A, int C, int G,
                                           neat_stream_t stream)
{
    return grid_convert(src, dst, A, C, G, 0, (cudaStream_t)stream);
}
