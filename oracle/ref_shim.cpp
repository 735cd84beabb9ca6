// ref_shim.cpp -- C entry points around the reference's own CPU code, for
// pinning the oracle (TEST INFRASTRUCTURE; built by `make -C oracle ref`).
//
// The recipe copies, at build time and into the git-ignored oracle/_ref/,
// the unmodified text of
//   * IndirectGridSample3DForwardCPU / IndirectGridSample3DBackwardCPU and
//     their macros (src/modules/IndirectGridSample3D.cu:19-429),
//   * IntersectBoxRayPrecise (src/structure/HyperTree.h:41-83),
// and compiles them against the stand-ins below: a torch::Tensor with the
// data_ptr/size/stride the CPU functions use, saiga's vec3, and inert
// declarations for the grid_sample calls of the forward's disabled `if (0)`
// branch (never executed).  Nothing of the reference is committed here.
#include <cmath>
#include <initializer_list>
#include <tuple>

struct vec3
{
    float v[3];
    float& operator()(int i) { return v[i]; }
    float operator()(int i) const { return v[i]; }
};

namespace torch
{
struct Tensor
{
    void* p      = nullptr;
    long sz[5]   = {0, 0, 0, 0, 0};
    long st[5]   = {0, 0, 0, 0, 0};
    template <typename T>
    T* data_ptr() const
    {
        return (T*)p;
    }
    long size(int i) const { return sz[i]; }
    long stride(int i) const { return st[i]; }
    Tensor unsqueeze(int) const { return *this; }
    Tensor squeeze(int) const { return *this; }
};
enum PadMode { kBorder };
enum InterpMode { kBilinear };
inline Tensor index_select(const Tensor& t, int, const Tensor&) { return t; }
namespace nn
{
namespace functional
{
struct GridSampleFuncOptions
{
    GridSampleFuncOptions padding_mode(PadMode) const { return *this; }
    GridSampleFuncOptions mode(InterpMode) const { return *this; }
    GridSampleFuncOptions align_corners(bool) const { return *this; }
};
inline Tensor grid_sample(const Tensor& t, const Tensor&, const GridSampleFuncOptions&) { return t; }
}  // namespace functional
}  // namespace nn
}  // namespace torch

#define HD

#include "igs_cpu.inc"
#include "slab.inc"

static torch::Tensor make(const void* p, std::initializer_list<long> sizes)
{
    torch::Tensor t;
    t.p   = const_cast<void*>(p);
    int d = 0;
    for (long s : sizes) t.sz[d++] = s;
    long stride = 1;
    for (int i = d - 1; i >= 0; --i)
    {
        t.st[i] = stride;
        stride *= t.sz[i];
    }
    return t;
}

extern "C" void ref_igs_forward(const float* grid, long N, int C, int Z, int Y, int X, const long* index,
                                const float* uv, long S, float* out)
{
    torch::Tensor o = make(out, {S, C});
    IndirectGridSample3DForwardCPU(make(grid, {N, C, Z, Y, X}), make(index, {S}), make(uv, {S, 3}), o);
}

extern "C" void ref_igs_backward(const float* grid, long N, int C, int Z, int Y, int X, const long* index,
                                 const float* uv, long S, const float* grad_out, float* grad_grid, float* grad_uv)
{
    torch::Tensor gg = make(grad_grid, {N, C, Z, Y, X});
    torch::Tensor gu = make(grad_uv, {S, 3});
    IndirectGridSample3DBackwardCPU(make(grid, {N, C, Z, Y, X}), make(index, {S}), make(uv, {S, 3}), gg, gu,
                                    make(grad_out, {S, C}));
}

extern "C" int ref_intersect_box(const float* pmin, const float* pmax, const float* o, const float* d, float* tmin,
                                 float* tmax)
{
    auto r = IntersectBoxRayPrecise(const_cast<float*>(pmin), const_cast<float*>(pmax), const_cast<float*>(o),
                                    const_cast<float*>(d), 3);
    *tmin = std::get<1>(r);
    *tmax = std::get<2>(r);
    return std::get<0>(r) ? 1 : 0;
}
