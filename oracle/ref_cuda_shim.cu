// ref_cuda_shim.cu -- C entry points around the reference's own GPU grid
// sampler, for timing it on the B200 beside this library's kernels
// (BASELINE INFRASTRUCTURE; built by `make -C oracle ref-cuda`, used only by
// bench.py's comparison leg).
//
// The recipe copies, at build time and into the git-ignored oracle/_ref/,
// the unmodified text of
//   * the MIN/MAX/CLIP_COORDINATES/WITHIN_BOUNDS macros
//     (src/modules/IndirectGridSample3D.cu:19-24),
//   * IndirectGridSample3DForwardCUDAKernel / IndirectGridSample3DForwardCUDA
//     and IndirectGridSample3DBackwardCUDAKernel / IndirectGridSample3DBackwardCUDA
//     (src/modules/IndirectGridSample3D.cu:432-801),
// and compiles them for sm_100a against the stand-ins below: saiga's
// StaticDeviceTensor (a pointer, sizes and strides with a variadic element
// accessor), a torch::Tensor carrying the same and converting to it, and
// iDivUp.  The kernels launch on the legacy default stream, as the reference
// does.  Nothing of the reference is committed here.
#include <cstdint>
#include <cuda_runtime.h>

template <typename T, int D>
struct StaticDeviceTensor
{
    T* data;
    int64_t sizes[D];
    int64_t strides[D];

    template <typename... I>
    __device__ T& operator()(I... idx) const
    {
        static_assert(sizeof...(I) == D, "one index per dimension");
        const int64_t ii[D] = {(int64_t)idx...};
        int64_t off         = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) off += ii[k] * strides[k];
        return data[off];
    }
};

namespace torch
{
// a contiguous tensor: pointer + up to 5 sizes (strides derived)
struct Tensor
{
    void* p = nullptr;
    int dim = 0;
    int64_t sz[5] = {0, 0, 0, 0, 0};

    int64_t size(int i) const { return sz[i]; }

    template <typename T, int D>
    operator StaticDeviceTensor<T, D>() const
    {
        StaticDeviceTensor<T, D> t;
        t.data      = (T*)p;
        int64_t st  = 1;
        for (int k = D - 1; k >= 0; --k)
        {
            t.sizes[k]   = sz[k];
            t.strides[k] = st;
            st *= sz[k];
        }
        return t;
    }
};
}  // namespace torch

static inline int iDivUp(int a, int b) { return (a + b - 1) / b; }

#include "igs_cuda_macros.inc"
#include "igs_cuda.inc"

static torch::Tensor make(void* p, int dim, const int64_t* sizes)
{
    torch::Tensor t;
    t.p   = p;
    t.dim = dim;
    for (int k = 0; k < dim; ++k) t.sz[k] = sizes[k];
    return t;
}

// grid [N, C, Z, Y, X] f32, index [S] int64, uv [S, 3] f32, out [S, C] f32.
extern "C" int ref_igs_forward_cuda(float* grid, int64_t N, int C, int Z, int Y, int X, int64_t* index, float* uv,
                                    int64_t S, float* out)
{
    const int64_t gs[5] = {N, C, Z, Y, X}, is[1] = {S}, us[2] = {S, 3}, os[2] = {S, C};
    torch::Tensor output = make(out, 2, os);
    IndirectGridSample3DForwardCUDA(make(grid, 5, gs), make(index, 1, is), make(uv, 2, us), output);
    return (int)cudaGetLastError();
}

// grad_grid and grad_uv accumulate (zero them first, as the reference's zeros_like).
extern "C" int ref_igs_backward_cuda(float* grid, int64_t N, int C, int Z, int Y, int X, int64_t* index, float* uv,
                                     int64_t S, float* grad_out, float* grad_grid, float* grad_uv)
{
    const int64_t gs[5] = {N, C, Z, Y, X}, is[1] = {S}, us[2] = {S, 3}, os[2] = {S, C};
    torch::Tensor gg = make(grad_grid, 5, gs), gu = make(grad_uv, 2, us);
    IndirectGridSample3DBackwardCUDA(make(grid, 5, gs), make(index, 1, is), make(uv, 2, us), gg, gu,
                                     make(grad_out, 2, os));
    return (int)cudaGetLastError();
}
