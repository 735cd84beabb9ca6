// ref_sampler_shim.cu -- C entry point around the reference's own GPU ray
// sampler, to pin the oracle's restatement and this library's sampler against
// it (TEST INFRASTRUCTURE; built by `make -C oracle ref-sampler`, used only by
// tests/).
//
// The recipe copies, at build time and into the git-ignored oracle/_ref/, the
// unmodified text of
//   * IntersectBoxRayPrecise (src/structure/HyperTree.h:41-83),
//   * the kernel ComputeRaySamples<D, ThreadsPerBlock>
//     (src/structure/HyperTree.cu:206-391),
// and compiles them for sm_100a with nvcc's defaults (FMA contraction on, as
// the reference's CUDA build) against the stand-ins below:
//   * Eigen::Vector<float, D>: element access, data(), +, -, scalar *, and
//     norm() = sqrt of the squares summed in Eigen's unrolled reduction order
//     a0 + (a1 + a2) (Eigen's redux splits a fixed-size sum in halves);
//   * StaticDeviceTensor<T, D>: pointer, sizes, strides, variadic accessor;
//   * DeviceHyperTree<D>: the three tables the kernel reads;
//   * iCeil(x) = (int)ceil(x); CUDA_KERNEL_ASSERT compiled out (the reference
//     defines CUDA_NDEBUG in HyperTree.cu).
// The kernel is launched as CreateSamplesForRays launches it (one 128-thread
// block per ray, src/structure/HyperTree.cu:406-416).  It writes past its
// outputs when the capacity is short and past its shared arrays beyond 256
// hits on a ray, so the caller must size both from an exact count first.
// Nothing of the reference is committed here.
#include <cmath>
#include <cstdint>
#include <tuple>

#include <cuda_runtime.h>

#define HD __host__ __device__
#define CUDA_KERNEL_ASSERT(x)

namespace Eigen
{
template <typename T, int N>
struct Vector
{
    T v[N];
    HD T& operator()(int i) { return v[i]; }
    HD T operator()(int i) const { return v[i]; }
    HD T* data() { return v; }
    HD Vector operator-(const Vector& o) const
    {
        Vector r;
        for (int i = 0; i < N; ++i) r.v[i] = v[i] - o.v[i];
        return r;
    }
    HD Vector operator+(const Vector& o) const
    {
        Vector r;
        for (int i = 0; i < N; ++i) r.v[i] = v[i] + o.v[i];
        return r;
    }
    HD T norm() const;
};
template <>
HD inline float Vector<float, 3>::norm() const
{
    return sqrtf(v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]));
}
template <typename T, int N>
HD Vector<T, N> operator*(T s, const Vector<T, N>& a)
{
    Vector<T, N> r;
    for (int i = 0; i < N; ++i) r.v[i] = s * a.v[i];
    return r;
}
}  // namespace Eigen

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

template <typename T, int D>
static StaticDeviceTensor<T, D> tensor(T* p, const int64_t* sizes)
{
    StaticDeviceTensor<T, D> t;
    t.data     = p;
    int64_t st = 1;
    for (int k = D - 1; k >= 0; --k)
    {
        t.sizes[k]   = sizes[k];
        t.strides[k] = st;
        st *= sizes[k];
    }
    return t;
}

template <int D>
struct DeviceHyperTree
{
    using Vec = Eigen::Vector<float, D>;
    StaticDeviceTensor<float, 2> node_position_min;
    StaticDeviceTensor<float, 2> node_position_max;
    StaticDeviceTensor<long, 1> active_node_ids;
};

static inline HD int iCeil(float x) { return (int)ceilf(x); }

#include "slab_cuda.inc"
#include "sampler_cuda.inc"

// One launch of the reference kernel.  node_min/max [N, 3] f32, active_ids
// [A] int64, origin/direction [R, 3] f32, sample_rnd [capacity] f32 or NULL
// (a = 0.5), outputs of `capacity` rows (coords [cap, 3]), out_count int32[2]
// (zeroed by the caller: sample total, max samples of one ray).
extern "C" int ref_compute_ray_samples(float* node_min, float* node_max, int64_t num_nodes, int64_t* active_ids,
                                       int64_t num_active, float* origin, float* direction, int64_t num_rays,
                                       float* sample_rnd, int max_samples_per_node, int64_t capacity, float* coords,
                                       float* weight, float* ray_t, int64_t* ray_index, int64_t* local_index,
                                       int64_t* node_id, int* out_count)
{
    if (num_rays <= 0) return 0;
    DeviceHyperTree<3> tree;
    const int64_t nsz[2] = {num_nodes, 3}, asz[1] = {num_active};
    tree.node_position_min = tensor<float, 2>(node_min, nsz);
    tree.node_position_max = tensor<float, 2>(node_max, nsz);
    tree.active_node_ids   = tensor<long, 1>((long*)active_ids, asz);
    const int64_t rsz[2] = {num_rays, 3}, csz[2] = {capacity, 3}, ssz[1] = {capacity};
    ComputeRaySamples<3, 128><<<(unsigned)num_rays, 128>>>(
        tree, tensor<float, 2>(origin, rsz), tensor<float, 2>(direction, rsz), sample_rnd, out_count,
        tensor<float, 2>(coords, csz), tensor<float, 1>(weight, ssz), tensor<float, 1>(ray_t, ssz),
        tensor<long, 1>((long*)ray_index, ssz), tensor<long, 1>((long*)local_index, ssz),
        tensor<long, 1>((long*)node_id, ssz), max_samples_per_node);
    return (int)cudaGetLastError();
}
