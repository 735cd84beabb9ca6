// neat_torch.cpp -- libtorch implementation of neat_torch.h on the C ABI of
// libneat_b200.so, and its registration as torch operators (namespace "neat")
// so the same code can be driven from Python (torch.ops.load_library).
#include "neat_torch.h"

#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <cmath>

#include "neat_b200.h"

namespace neat_torch
{
namespace
{
neat_stream_t stream_of(const torch::Tensor& t)
{
    return (neat_stream_t)c10::cuda::getCurrentCUDAStream(t.device().index()).stream();
}

void check(int st, const char* what) { TORCH_CHECK(st == NEAT_OK, what, ": ", neat_status_string(st)); }

void need_cuda(const torch::Tensor& t, const char* name)
{
    TORCH_CHECK(t.defined(), name, " is undefined");
    TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor (libneat_b200 has no CPU path)");
}

void need_type(const torch::Tensor& t, torch::ScalarType s, const char* name)
{
    TORCH_CHECK(t.scalar_type() == s, name, " must be ", c10::toString(s), ", got ", c10::toString(t.scalar_type()));
}

torch::TensorOptions on(const torch::Tensor& t, torch::ScalarType s)
{
    return torch::TensorOptions().dtype(s).device(t.device());
}
}  // namespace

// ---------------------------------------------------------------------------
// SampleList
// ---------------------------------------------------------------------------
void SampleList::Allocate(int64_t num_samples, int D, torch::Device device)
{
    auto f = torch::TensorOptions(torch::kFloat32).device(device);
    auto l = torch::TensorOptions(torch::kLong).device(device);
    global_coordinate  = torch::empty({num_samples, D}, f);
    weight             = torch::empty({num_samples}, f);
    ray_t              = torch::empty({num_samples}, f);
    ray_index          = torch::empty({num_samples}, l);
    local_index_in_ray = torch::empty({num_samples}, l);
    node_id            = torch::empty({num_samples}, l);
}

void SampleList::Shrink(int64_t new_size)
{
    global_coordinate  = global_coordinate.slice(0, 0, new_size);
    weight             = weight.slice(0, 0, new_size);
    ray_t              = ray_t.slice(0, 0, new_size);
    ray_index          = ray_index.slice(0, 0, new_size);
    local_index_in_ray = local_index_in_ray.slice(0, 0, new_size);
    node_id            = node_id.slice(0, 0, new_size);
}

// ---------------------------------------------------------------------------
// IndirectGridSample3D
// ---------------------------------------------------------------------------
torch::Tensor IndirectGridSample3DFunction::forward(torch::autograd::AutogradContext* ctx, torch::Tensor multi_grid,
                                                    torch::Tensor index, torch::Tensor uv)
{
    c10::cuda::CUDAGuard guard(multi_grid.device());
    const int64_t S = index.size(0);
    auto out        = torch::zeros({S, multi_grid.size(1)}, multi_grid.options());
    check(neat_igs_forward(multi_grid.data_ptr<float>(), multi_grid.size(0), (int)multi_grid.size(1),
                           (int)multi_grid.size(2), (int)multi_grid.size(3), (int)multi_grid.size(4),
                           index.data_ptr<int64_t>(), uv.data_ptr<float>(), S, out.data_ptr<float>(),
                           stream_of(multi_grid)),
          "neat_igs_forward");
    ctx->save_for_backward({multi_grid, index, uv});
    return out;
}

torch::autograd::variable_list IndirectGridSample3DFunction::backward(torch::autograd::AutogradContext* ctx,
                                                                      torch::autograd::variable_list grad_output)
{
    auto saved = ctx->get_saved_variables();
    auto grid = saved[0], index = saved[1], uv = saved[2];
    c10::cuda::CUDAGuard guard(grid.device());
    auto go = grad_output[0].to(torch::kFloat32).contiguous();
    // zero-initialised, as the reference's torch::zeros_like (IndirectGridSample3D.cu:848-849)
    auto grad_grid = torch::zeros_like(grid);
    auto grad_uv   = torch::zeros_like(uv);
    check(neat_igs_backward(grid.data_ptr<float>(), grid.size(0), (int)grid.size(1), (int)grid.size(2),
                            (int)grid.size(3), (int)grid.size(4), index.data_ptr<int64_t>(), uv.data_ptr<float>(),
                            index.size(0), go.data_ptr<float>(), grad_grid.data_ptr<float>(),
                            grad_uv.data_ptr<float>(), stream_of(grid)),
          "neat_igs_backward");
    return {grad_grid, torch::Tensor(), grad_uv};
}

torch::Tensor IndirectGridSample3D(torch::Tensor multi_grid, torch::Tensor index, torch::Tensor uv)
{
    need_cuda(multi_grid, "multi_grid");
    need_cuda(index, "index");
    need_cuda(uv, "uv");
    TORCH_CHECK(multi_grid.dim() == 5 && index.dim() == 1 && uv.dim() == 2 && uv.size(1) == 3,
                "IndirectGridSample3D: expected multi_grid [N,C,Z,Y,X], index [S], uv [S,3]");
    TORCH_CHECK(index.size(0) == uv.size(0), "IndirectGridSample3D: one index per uv row");
    need_type(multi_grid, torch::kFloat32, "multi_grid");
    need_type(index, torch::kLong, "index");
    need_type(uv, torch::kFloat32, "uv");
    return IndirectGridSample3DFunction::apply(multi_grid.contiguous(), index.contiguous(), uv.contiguous());
}

// ---------------------------------------------------------------------------
// HyperTree
// ---------------------------------------------------------------------------
HyperTree::HyperTree(torch::Tensor node_position_min_, torch::Tensor node_position_max_,
                     torch::Tensor active_node_ids_, int max_depth_, uint64_t seed_)
    : max_depth(max_depth_), seed(seed_)
{
    need_cuda(node_position_min_, "node_position_min");
    const auto dev    = node_position_min_.device();
    node_position_min = node_position_min_.to(dev, torch::kFloat32).contiguous();
    node_position_max = node_position_max_.to(dev, torch::kFloat32).contiguous();
    active_node_ids   = active_node_ids_.to(dev, torch::kLong).contiguous();
    const int64_t N   = node_position_min.size(0);
    TORCH_CHECK(node_position_min.dim() == 2 && node_position_min.size(1) == 3 &&
                    node_position_max.sizes() == node_position_min.sizes(),
                "HyperTree: node_position_min/max must be [N, 3]");
    const size_t bytes = neat_tree_table_bytes(max_depth);
    TORCH_CHECK(bytes > 0, "HyperTree: max_depth ", max_depth, " is not supported");
    c10::cuda::CUDAGuard guard(dev);
    table_      = torch::empty({(int64_t)bytes}, on(node_position_min, torch::kUInt8));
    auto status = torch::zeros({1}, on(node_position_min, torch::kInt32));
    check(neat_tree_prepare(node_position_min.data_ptr<float>(), node_position_max.data_ptr<float>(),
                            active_node_ids.data_ptr<int64_t>(), (int)active_node_ids.size(0), max_depth,
                            table_.data_ptr(), status.data_ptr<int>(), stream_of(node_position_min)),
          "neat_tree_prepare");
    check(status.item<int>(), "neat_tree_prepare");
    node_active_prefix_sum = torch::full({N}, -1, on(node_position_min, torch::kLong));
    node_active_prefix_sum.index_put_({active_node_ids},
                                      torch::arange(active_node_ids.size(0), on(node_position_min, torch::kLong)));
}

SampleList HyperTree::CreateSamplesForRays(const RayList& rays, int max_samples_per_node, bool interval_jitter)
{
    need_cuda(rays.origin, "rays.origin");
    need_cuda(rays.direction, "rays.direction");
    TORCH_CHECK(max_samples_per_node >= 1, "max_samples_per_node must be >= 1");
    c10::cuda::CUDAGuard guard(rays.origin.device());
    auto o          = rays.origin.to(torch::kFloat32).contiguous();
    auto d          = rays.direction.to(torch::kFloat32).contiguous();
    const int64_t R = o.size(0);
    const int64_t A = NumActiveNodes();
    auto ws = torch::empty({std::max<int64_t>((int64_t)neat_samples_workspace_bytes(R), 16)}, on(o, torch::kUInt8));
    // the reference's capacity estimate R * M * A^(1/3) (HyperTree.cu:398), grown if a batch needs more
    int64_t cap        = (int64_t)std::ceil((double)R * max_samples_per_node * std::cbrt((double)A)) + 1;
    const uint32_t stp = step++;
    while (true)
    {
        SampleList out;
        out.Allocate(cap, 3, o.device());
        auto cnt    = torch::zeros({2}, on(o, torch::kLong));
        auto status = torch::zeros({1}, on(o, torch::kInt32));
        check(neat_create_samples(table_.data_ptr(), (int)A, max_depth, o.data_ptr<float>(), d.data_ptr<float>(), R,
                                  max_samples_per_node, interval_jitter ? 1 : 0, seed, stp, cap,
                                  out.global_coordinate.data_ptr<float>(), out.ray_t.data_ptr<float>(),
                                  out.weight.data_ptr<float>(), out.ray_index.data_ptr<int64_t>(),
                                  out.local_index_in_ray.data_ptr<int64_t>(), out.node_id.data_ptr<int64_t>(),
                                  cnt.data_ptr<int64_t>(), status.data_ptr<int>(), ws.data_ptr(), stream_of(o)),
              "neat_create_samples");
        // the count is read on the host, as the reference's .item() (HyperTree.cu:420)
        auto c          = cnt.cpu();
        const int st    = status.item<int>();
        const int64_t S = c[0].item<int64_t>();
        if ((st & NEAT_ERR_CAPACITY) && S > cap)
        {
            cap = S;
            continue;
        }
        check(st, "CreateSamplesForRays");
        out.Shrink(S);
        out.max_samples_per_ray = c[1].item<int64_t>();
        return out;
    }
}

torch::Tensor HyperTree::ComputeLocalSamples(torch::Tensor global_samples, torch::Tensor node_indices)
{
    need_cuda(global_samples, "global_samples");
    need_cuda(node_indices, "node_indices");
    c10::cuda::CUDAGuard guard(global_samples.device());
    auto g   = global_samples.to(torch::kFloat32).contiguous().reshape({-1, 3});
    auto nid = node_indices.to(torch::kLong).contiguous().reshape({-1});
    TORCH_CHECK(nid.size(0) == g.size(0), "ComputeLocalSamples: one node id per sample");
    auto out = torch::empty_like(g);
    check(neat_local_samples(g.data_ptr<float>(), nid.data_ptr<int64_t>(), g.size(0), node_position_min.data_ptr<float>(),
                             node_position_max.data_ptr<float>(), out.data_ptr<float>(), stream_of(g)),
          "neat_local_samples");
    return out.reshape(global_samples.sizes());
}

torch::Tensor HyperTree::GlobalNodeIdToLocalActiveId(torch::Tensor node_id)
{
    return node_active_prefix_sum.index_select(0, node_id.reshape({-1})).reshape(node_id.sizes());
}

// ---------------------------------------------------------------------------
// GetRays
// ---------------------------------------------------------------------------
RayList GetRays(const Camera& camera, torch::Tensor uv, torch::Tensor image_id, torch::Tensor camera_id)
{
    need_cuda(uv, "uv");
    need_cuda(image_id, "image_id");
    TORCH_CHECK(uv.dim() == 2 && uv.size(1) == 2 && image_id.size(0) == uv.size(0),
                "GetRays: uv must be [R,2] and image_id [R]");
    c10::cuda::CUDAGuard guard(uv.device());
    auto u          = uv.to(torch::kFloat32).contiguous();
    auto img        = image_id.to(torch::kInt32).contiguous();
    auto cid        = camera_id.defined() ? camera_id.to(torch::kInt32).contiguous() : torch::Tensor();
    auto intr       = camera.intrinsics.to(u.device(), torch::kFloat64).contiguous();
    auto rot        = camera.rotation.to(u.device(), torch::kFloat64).contiguous();
    auto trans      = camera.translation.to(u.device(), torch::kFloat64).contiguous();
    const int64_t R = u.size(0);
    RayList rays;
    rays.origin    = torch::empty({R, 3}, on(u, torch::kFloat32));
    rays.direction = torch::empty({R, 3}, on(u, torch::kFloat32));
    check(neat_make_rays(u.data_ptr<float>(), img.data_ptr<int32_t>(), cid.defined() ? cid.data_ptr<int32_t>() : nullptr,
                         R, camera.w, camera.h, intr.data_ptr<double>(), rot.data_ptr<double>(),
                         trans.data_ptr<double>(), rays.origin.data_ptr<float>(), rays.direction.data_ptr<float>(),
                         stream_of(u)),
          "neat_make_rays");
    return rays;
}

// ---------------------------------------------------------------------------
// ComputeImage
// ---------------------------------------------------------------------------
namespace
{
struct ComputeImageFunction : public torch::autograd::Function<ComputeImageFunction>
{
    // inputs after grid/decoder: coords, weight, ray_index, node_id, local_id, node_min, node_max
    static torch::Tensor forward(torch::autograd::AutogradContext* ctx, torch::Tensor grid, torch::Tensor decoder,
                                 torch::Tensor coords, torch::Tensor weight, torch::Tensor ray_index,
                                 torch::Tensor node_id, torch::Tensor local_id, torch::Tensor node_min,
                                 torch::Tensor node_max, double softplus_beta, int64_t num_pixels)
    {
        c10::cuda::CUDAGuard guard(grid.device());
        auto image = torch::zeros({num_pixels}, grid.options());
        check(neat_compute_image_forward(grid.data_ptr<float>(), grid.size(0), (int)grid.size(1), (int)grid.size(2),
                                         decoder.data_ptr<float>(), (float)softplus_beta, coords.data_ptr<float>(),
                                         weight.data_ptr<float>(), ray_index.data_ptr<int64_t>(),
                                         node_id.data_ptr<int64_t>(), local_id.data_ptr<int64_t>(),
                                         node_min.data_ptr<float>(), node_max.data_ptr<float>(), coords.size(0),
                                         image.data_ptr<float>(), stream_of(grid)),
              "neat_compute_image_forward");
        ctx->save_for_backward({grid, decoder, coords, weight, ray_index, node_id, local_id, node_min, node_max});
        ctx->saved_data["beta"] = softplus_beta;
        return image.reshape({1, num_pixels});
    }

    static torch::autograd::variable_list backward(torch::autograd::AutogradContext* ctx,
                                                   torch::autograd::variable_list grad_output)
    {
        auto v    = ctx->get_saved_variables();
        auto grid = v[0], decoder = v[1];
        c10::cuda::CUDAGuard guard(grid.device());
        auto gi        = grad_output[0].reshape({-1}).to(torch::kFloat32).contiguous();
        auto grad_grid = torch::zeros_like(grid);
        auto grad_dec  = torch::zeros_like(decoder);
        check(neat_compute_image_backward(grid.data_ptr<float>(), grid.size(0), (int)grid.size(1), (int)grid.size(2),
                                          decoder.data_ptr<float>(), (float)ctx->saved_data["beta"].toDouble(),
                                          v[2].data_ptr<float>(), v[3].data_ptr<float>(), v[4].data_ptr<int64_t>(),
                                          v[5].data_ptr<int64_t>(), v[6].data_ptr<int64_t>(), v[7].data_ptr<float>(),
                                          v[8].data_ptr<float>(), v[2].size(0), gi.data_ptr<float>(),
                                          grad_grid.data_ptr<float>(), grad_dec.data_ptr<float>(), stream_of(grid)),
              "neat_compute_image_backward");
        return {grad_grid,       grad_dec,        torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor(),
                torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor()};
    }
};
}  // namespace

torch::Tensor ComputeImage(const SampleList& all_samples, HyperTree& tree, torch::Tensor grid, torch::Tensor decoder,
                           int num_channels, int num_pixels, double softplus_beta)
{
    TORCH_CHECK(num_channels == 1, "ComputeImage: the X-ray decoder has one output channel");
    need_cuda(grid, "grid");
    need_cuda(decoder, "decoder");
    need_type(grid, torch::kFloat32, "grid");
    need_type(decoder, torch::kFloat32, "decoder");
    TORCH_CHECK(grid.dim() == 5 && grid.size(2) == grid.size(3) && grid.size(3) == grid.size(4),
                "ComputeImage: grid must be [rows, C, G, G, G]");
    TORCH_CHECK(decoder.numel() == neat_decoder_params((int)grid.size(1)),
                "ComputeImage: decoder must hold neat_decoder_params(C) floats");
    auto local_id = tree.GlobalNodeIdToLocalActiveId(all_samples.node_id).contiguous();
    return ComputeImageFunction::apply(grid.contiguous(), decoder.contiguous(),
                                       all_samples.global_coordinate.contiguous(), all_samples.weight.contiguous(),
                                       all_samples.ray_index.contiguous(), all_samples.node_id.contiguous(), local_id,
                                       tree.node_position_min, tree.node_position_max, softplus_beta,
                                       (int64_t)num_pixels);
}

// ---------------------------------------------------------------------------
// Adam
// ---------------------------------------------------------------------------
Adam::Adam(std::vector<Group> groups, double beta1, double beta2, double eps)
    : groups_(std::move(groups)), beta1_(beta1), beta2_(beta2), eps_(eps)
{
    for (auto& g : groups_)
    {
        exp_avg_.emplace_back(g.params.size());
        exp_avg_sq_.emplace_back(g.params.size());
        for (auto& p : g.params)
        {
            need_cuda(p, "parameter");
            need_type(p, torch::kFloat32, "parameter");
            TORCH_CHECK(p.is_contiguous(), "Adam: parameters must be contiguous");
        }
    }
}

void Adam::step()
{
    ++step_;
    for (size_t gi = 0; gi < groups_.size(); ++gi)
    {
        for (size_t pi = 0; pi < groups_[gi].params.size(); ++pi)
        {
            auto& p = groups_[gi].params[pi];
            if (!p.grad().defined()) continue;
            auto g = p.grad();
            TORCH_CHECK(g.is_contiguous() && g.scalar_type() == torch::kFloat32 && g.sizes() == p.sizes(),
                        "Adam: gradient must be a contiguous float tensor of the parameter's shape");
            auto& m = exp_avg_[gi][pi];
            auto& v = exp_avg_sq_[gi][pi];
            if (!m.defined())
            {
                m = torch::zeros_like(p);
                v = torch::zeros_like(p);
            }
            c10::cuda::CUDAGuard guard(p.device());
            torch::NoGradGuard no_grad;
            check(neat_adam(p.data_ptr<float>(), g.data_ptr<float>(), m.data_ptr<float>(), v.data_ptr<float>(),
                            p.numel(), (float)groups_[gi].lr, (float)beta1_, (float)beta2_, (float)eps_, (int)step_, 0,
                            stream_of(p)),
                  "neat_adam");
        }
    }
}

void Adam::zero_grad()
{
    for (auto& g : groups_)
        for (auto& p : g.params)
            if (p.grad().defined()) p.mutable_grad().zero_();
}

}  // namespace neat_torch

// ---------------------------------------------------------------------------
// Torch operators (namespace "neat"): the same API reachable from Python for
// tests and bindings.  Tree and camera are passed as their tensors.
// ---------------------------------------------------------------------------
namespace
{
using neat_torch::HyperTree;
using neat_torch::RayList;
using neat_torch::SampleList;

std::tuple<torch::Tensor, torch::Tensor> op_get_rays(int64_t w, int64_t h, torch::Tensor intrinsics,
                                                     torch::Tensor rotation, torch::Tensor translation,
                                                     torch::Tensor uv, torch::Tensor image_id,
                                                     c10::optional<torch::Tensor> camera_id)
{
    neat_torch::Camera cam;
    cam.w           = (int)w;
    cam.h           = (int)h;
    cam.intrinsics  = intrinsics;
    cam.rotation    = rotation;
    cam.translation = translation;
    auto r          = neat_torch::GetRays(cam, uv, image_id, camera_id.value_or(torch::Tensor()));
    return {r.origin, r.direction};
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, int64_t>
op_create_samples(torch::Tensor node_position_min, torch::Tensor node_position_max, torch::Tensor active_node_ids,
                  int64_t max_depth, int64_t seed, int64_t step, torch::Tensor origin, torch::Tensor direction,
                  int64_t max_samples_per_node, bool interval_jitter)
{
    HyperTree tree(node_position_min, node_position_max, active_node_ids, (int)max_depth, (uint64_t)seed);
    tree.step = (uint32_t)step;
    RayList rays{origin, direction};
    SampleList s = tree.CreateSamplesForRays(rays, (int)max_samples_per_node, interval_jitter);
    return {s.global_coordinate, s.ray_t, s.weight, s.ray_index, s.local_index_in_ray, s.node_id,
            s.max_samples_per_ray};
}

torch::Tensor op_local_samples(torch::Tensor node_position_min, torch::Tensor node_position_max,
                               torch::Tensor active_node_ids, int64_t max_depth, torch::Tensor global_samples,
                               torch::Tensor node_indices)
{
    HyperTree tree(node_position_min, node_position_max, active_node_ids, (int)max_depth);
    return tree.ComputeLocalSamples(global_samples, node_indices);
}

torch::Tensor op_compute_image(torch::Tensor node_position_min, torch::Tensor node_position_max,
                               torch::Tensor active_node_ids, int64_t max_depth, torch::Tensor global_coordinate,
                               torch::Tensor weight, torch::Tensor ray_index, torch::Tensor node_id,
                               torch::Tensor grid, torch::Tensor decoder, int64_t num_channels, int64_t num_pixels,
                               double softplus_beta)
{
    HyperTree tree(node_position_min, node_position_max, active_node_ids, (int)max_depth);
    SampleList s;
    s.global_coordinate = global_coordinate;
    s.weight            = weight;
    s.ray_index         = ray_index;
    s.node_id           = node_id;
    return neat_torch::ComputeImage(s, tree, grid, decoder, (int)num_channels, (int)num_pixels, softplus_beta);
}

// num_steps Adam steps over param groups (group_of[i] = group of params[i],
// lrs[group]); grads holds num_steps x params.size() gradients, step-major.
void op_adam_steps(std::vector<torch::Tensor> params, std::vector<torch::Tensor> grads, std::vector<int64_t> group_of,
                   std::vector<double> lrs, int64_t num_steps, double beta1, double beta2, double eps)
{
    TORCH_CHECK(group_of.size() == params.size(), "adam_steps: one group index per parameter");
    TORCH_CHECK((int64_t)grads.size() == num_steps * (int64_t)params.size(), "adam_steps: num_steps x params grads");
    std::vector<neat_torch::Adam::Group> groups(lrs.size());
    for (size_t g = 0; g < lrs.size(); ++g) groups[g].lr = lrs[g];
    for (size_t i = 0; i < params.size(); ++i)
    {
        TORCH_CHECK(group_of[i] >= 0 && group_of[i] < (int64_t)lrs.size(), "adam_steps: bad group index");
        groups[group_of[i]].params.push_back(params[i]);
    }
    neat_torch::Adam opt(groups, beta1, beta2, eps);
    for (int64_t s = 0; s < num_steps; ++s)
    {
        for (size_t i = 0; i < params.size(); ++i) params[i].mutable_grad() = grads[s * params.size() + i];
        opt.step();
        opt.zero_grad();
    }
}
}  // namespace

TORCH_LIBRARY(neat, m)
{
    m.def("IndirectGridSample3D(Tensor multi_grid, Tensor index, Tensor uv) -> Tensor",
          &neat_torch::IndirectGridSample3D);
    m.def("GetRays(int w, int h, Tensor intrinsics, Tensor rotation, Tensor translation, Tensor uv, Tensor image_id, "
          "Tensor? camera_id) -> (Tensor, Tensor)",
          &op_get_rays);
    m.def("CreateSamplesForRays(Tensor node_position_min, Tensor node_position_max, Tensor active_node_ids, "
          "int max_depth, int seed, int step, Tensor origin, Tensor direction, int max_samples_per_node, "
          "bool interval_jitter) -> (Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, int)",
          &op_create_samples);
    m.def("ComputeLocalSamples(Tensor node_position_min, Tensor node_position_max, Tensor active_node_ids, "
          "int max_depth, Tensor global_samples, Tensor node_indices) -> Tensor",
          &op_local_samples);
    m.def("ComputeImage(Tensor node_position_min, Tensor node_position_max, Tensor active_node_ids, int max_depth, "
          "Tensor global_coordinate, Tensor weight, Tensor ray_index, Tensor node_id, Tensor grid, Tensor decoder, "
          "int num_channels, int num_pixels, float softplus_beta) -> Tensor",
          &op_compute_image);
    m.def("AdamSteps(Tensor[] params, Tensor[] grads, int[] group_of, float[] lrs, int num_steps, float beta1, "
          "float beta2, float eps) -> ()",
          &op_adam_steps);
}
