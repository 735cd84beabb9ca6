// neat_torch.h -- the training step's reference-facing libtorch API, in C++.
//
// A libtorch program written against darglein/NeAT's modules includes this
// header and links libneat_torch.so (which links libneat_b200.so): the
// functions and types below keep the reference's names, argument meaning,
// tensor layouts and dtypes, and run on the B200 kernels of the C ABI
// (include/neat_b200.h).  Every function takes and returns CUDA tensors;
// there is no CPU path.  Where the reference aborts through a glog CHECK,
// these throw c10::Error (TORCH_CHECK) with the library's status text.
//
//   IndirectGridSample3D          src/modules/IndirectGridSample3D.h:18-30
//   RayList, SampleList           src/structure/HelperStructs.h:92-234
//   HyperTree::CreateSamplesForRays   src/structure/HyperTree.h:157
//   HyperTree::ComputeLocalSamples    src/structure/HyperTree.cu:116-199
//   GetRays                       src/data/SceneBase.h:151 (SceneBase.cpp:171-193)
//   ComputeImage                  src/geometry/geometry.h:170 (geometry.cpp:347-389)
//   Adam                          torch::optim::Adam as NeuralGeometry::OptimizerStep
//                                 drives it (src/geometry/geometry.h:66-88)
#pragma once

#include <torch/torch.h>

#include <cstdint>
#include <vector>

namespace neat_torch
{

// src/structure/HelperStructs.h:92-164: float [num_rays, 3] each.
struct RayList
{
    torch::Tensor origin;
    torch::Tensor direction;
    int64_t size() const { return origin.size(0); }
};

// src/structure/HelperStructs.h:168-234.
struct SampleList
{
    int64_t max_samples_per_ray = 0;
    torch::Tensor global_coordinate;   // float [S, 3]
    torch::Tensor ray_t;               // float [S]
    torch::Tensor weight;              // float [S]
    torch::Tensor ray_index;           // long [S]
    torch::Tensor local_index_in_ray;  // long [S]
    torch::Tensor node_id;             // long [S]

    int64_t size() const { return global_coordinate.size(0); }
    void Allocate(int64_t num_samples, int D, torch::Device device);
    void Shrink(int64_t new_size);
};

// The grid sampler and its autograd Function (IndirectGridSample3D.h:18-30):
// multi_grid [nodes, C, Z, Y, X] float, index [S] long, uv [S, 3] float
// (x, y, z) -> [S, C]; backward returns {grad_grid, undefined, grad_uv}.
struct IndirectGridSample3DFunction : public torch::autograd::Function<IndirectGridSample3DFunction>
{
    static torch::Tensor forward(torch::autograd::AutogradContext* ctx, torch::Tensor multi_grid,
                                 torch::Tensor index, torch::Tensor uv);
    static torch::autograd::variable_list backward(torch::autograd::AutogradContext* ctx,
                                                   torch::autograd::variable_list grad_output);
};
torch::Tensor IndirectGridSample3D(torch::Tensor multi_grid, torch::Tensor index, torch::Tensor uv);

// Octree node tables of HyperTreeBaseImpl (src/structure/HyperTree.h:206-240)
// for the complete breadth-first tree of max_depth: node_position_min/max
// float [N, 3], active_node_ids long [A] (ascending).  The device table of the
// sampler is built on construction; rebuild the object after the active set
// changes (SetActive/UpdateActive).  interval_jitter draws the stratified
// offsets from Philox keyed on (seed; ray, index in ray, call number).
class HyperTree
{
   public:
    HyperTree(torch::Tensor node_position_min, torch::Tensor node_position_max, torch::Tensor active_node_ids,
              int max_depth, uint64_t seed = 0);

    int64_t NumActiveNodes() const { return active_node_ids.size(0); }

    SampleList CreateSamplesForRays(const RayList& rays, int max_samples_per_node, bool interval_jitter);
    torch::Tensor ComputeLocalSamples(torch::Tensor global_samples, torch::Tensor node_indices);
    // node id -> grid row (node_active_prefix_sum), -1 for inactive nodes
    torch::Tensor GlobalNodeIdToLocalActiveId(torch::Tensor node_id);

    torch::Tensor node_position_min, node_position_max, active_node_ids, node_active_prefix_sum;
    int max_depth;
    uint64_t seed;
    uint32_t step = 1;  // call number of CreateSamplesForRays (the jitter's counter)

   private:
    torch::Tensor table_;
};

// Pinhole camera + per-image poses (CameraModelModule / CameraPoseModule):
// intrinsics double [num_cameras, 5] (fx, fy, cx, cy, skew), rotation double
// [num_images, 4] (x, y, z, w), translation double [num_images, 3].
struct Camera
{
    int w = 0, h = 0;
    torch::Tensor intrinsics, rotation, translation;
};

// SceneBase::GetRays: uv float [R, 2] in [0, 1], image_id int [R], camera_id
// int [R] or undefined (camera 0).
RayList GetRays(const Camera& camera, torch::Tensor uv, torch::Tensor image_id, torch::Tensor camera_id = {});

// HierarchicalNeuralGeometry::ComputeImage for the explicit-grid geometry
// (GeometryExEx): local coordinates -> IndirectGridSample3D -> FCBlock(C, 1, 1
// hidden pair of 64, silu) -> softplus(beta) -> * weight -> index_add by ray.
// grid float [rows, C, G, G, G] (reference layout), decoder float packed
// W1|b1|W2|b2|W3|b3 ([out][in] weights).  Returns [1, num_pixels]; autograd
// gives the grid and decoder gradients.
torch::Tensor ComputeImage(const SampleList& all_samples, HyperTree& tree, torch::Tensor grid,
                           torch::Tensor decoder, int num_channels, int num_pixels, double softplus_beta = 2.0);

// torch::optim::Adam with the options NeuralGeometry uses (no weight decay,
// no amsgrad, bias-corrected): one parameter group per (params, lr).
// step() updates every parameter that has a gradient; zero_grad() zeroes them.
class Adam
{
   public:
    struct Group
    {
        std::vector<torch::Tensor> params;
        double lr;
    };
    explicit Adam(std::vector<Group> groups, double beta1 = 0.9, double beta2 = 0.999, double eps = 1e-8);
    void step();
    void zero_grad();
    int64_t steps() const { return step_; }

   private:
    std::vector<Group> groups_;
    std::vector<std::vector<torch::Tensor>> exp_avg_, exp_avg_sq_;
    double beta1_, beta2_, eps_;
    int64_t step_ = 0;
};

}  // namespace neat_torch
