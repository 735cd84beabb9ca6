// neat_internal.h -- launchers shared between the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/neat_b200.h"

namespace neat
{

// Node-major segment record of the fused step (one ray crossing one node).
// It carries the ray and the node box so that a sample needs one record load.
struct __align__(16) SegRec
{
    int32_t ray;
    int32_t local_base;  // index in ray of the segment's first sample
    float tmin, tmax;
    int32_t n;           // samples in the segment
    int32_t rm;          // ray-major (canonical) segment index
    int32_t row;         // active (local) node id = grid row
    float step;          // (tmax - tmin) / n, rounded as the sampler rounds it
    float o[3], d[3];    // the ray (f32, as GetRays returns it)
    float mn[3], mx[3];  // the node box
};
static_assert(sizeof(SegRec) == 80, "SegRec must be 80 bytes");

// Pass 1 of the step: rays from (uv, image), one octree walk per ray, the
// canonical hit list of ray r at ray_hits[r * cap_ray ...], per-node counts.
cudaError_t launch_step_rays(const float* uv, const int32_t* image_id, int64_t R, int w, int h, const double* intr,
                             const double* rot, const double* trans, const void* table, int D, int M, int cap_ray,
                             float* origin, float* direction, SegRec* ray_hits, int* ray_nseg, int* node_nseg,
                             int64_t* counters, int* status, cudaStream_t st,
                             const int32_t* cell_node = nullptr);

// Pass 2: place the per-ray lists into node-major buckets.
cudaError_t launch_step_place(const SegRec* ray_hits, const int* ray_nseg, const int* ray_seg_off, int64_t R,
                              int cap_ray, const int* node_seg_off, SegRec* segs, int* seg_n,
                              int64_t* counters, int64_t cap, double* partial, int* status, cudaStream_t st);

int sm_count();

// CTAs per SM a kernel can keep resident, from its registers, static and
// dynamic shared memory and the device limits (cap: extra limit, e.g. TMEM).
int resident_ctas(const void* kernel, int threads, size_t dyn_smem, int cap);

// Arguments of the node-major sample-tile kernels of the fused step.
struct StepTileArgs
{
    const SegRec* segs;
    const int* samp_off;
    const int* tile_seg;
    const int64_t* counters;
    const float* origin;
    const float* direction;
    const float* node_min;
    const float* node_max;
    const float* grid;
    const uint16_t* grid_bf16;  // when set: BF16 copy of the grid the gathers read
    float* grid_grad;
    const float* decoder;
    float* dec_part;
    const float* dpred;
    double* partial;  // per-segment projection sums (ray-major segment index)
    int* status;
    uint64_t seed;
    uint32_t step;
    const int* step_dev;  // when set, the step number is read here (device-side step counter)
    const float* seg_cdf;  // proposal CDF per node-major segment [8] (null: uniform stratified)
    float* seg_hist;       // per ray-major segment [8]: contribution mass per sub-interval (null: off)
    float* seg_dens;       // per node-major sample: its density (null: off; samples < dens_cap only)
    int64_t dens_cap;
    float* seg_pgrad;      // per node-major segment [6]: sums of dL/d(ix,iy,iz) and t times it (null: off)
    // per-sample records the forward writes for the backward (null: off): SoA
    // [8 + C][rec_cap], fields lu, lv, lw, weight, t (f32), ray, row, seg (i32),
    // then the gathered features x[C]; used while the step's samples fit rec_cap
    float* rec;
    int64_t rec_cap;
    // backward: nonzero when the records backward (k_bwd_rec) runs the step's
    // tiles while its samples fit the records; this kernel then returns at once
    int rec_skip;
    int jitter;  // 0: a = 0.5 (evaluation), else Philox stratified offsets
    int G;
    float beta;
};
using StepTcArgs = StepTileArgs;

// Backward tiles from the forward's per-sample records with a warp that only
// issues the tensor-core work (neat_bwd_rec.cu): three-piece operands, C = 4
// or 8.  Runs while the step's samples fit the records (else returns at once).
bool bwd_rec_supported(int C, int prec);
cudaError_t launch_bwd_rec(int C, int prec, int grid, const StepTileArgs& args, cudaStream_t st);

// Camera pose gradients (neat_pose.cu): per-segment sums -> per-ray dL/do,
// dL/dd -> per-image rotation tangent and translation, camera intrinsics.
cudaError_t launch_pose_grad(const SegRec* segs, const int64_t* counters, const float* seg_pgrad, int G,
                             float* ray_pgrad, const float* uv, const int32_t* image_id, int64_t R, int w, int h,
                             const double* intrinsics, const double* rotation, const neat_pose_grad* pose,
                             cudaStream_t st);

// Learned proposal (neat_proposal.cu).
// CDF of every node-major segment (counters[0] of them) from the proposal MLP
// and, when pr->count_eps > 0, its sample count from the count head (into the
// segment record and seg_n, before the sample offsets are scanned).
cudaError_t launch_proposal_cdf(SegRec* segs, int* seg_n, const int64_t* counters, const neat_proposal* pr,
                                float* seg_cdf, cudaStream_t st);
// Node descriptors from the current grid (channel-last) and decoder.
cudaError_t launch_node_desc(const float* grid, int64_t A, int C, int G, const float* decoder, float beta,
                             float* node_desc, cudaStream_t st);
// Partials of one training iteration over a subset of the segments (iteration it).
int proposal_grad_blocks();
size_t proposal_part_floats();  // workspace floats of the training partials
cudaError_t launch_proposal_train(const SegRec* segs, const int64_t* counters, const float* seg_hist,
                                  const float* seg_tv, const neat_proposal* pr, float* part, int iters,
                                  cudaStream_t st);
// Per segment of a uniformly sampled TRAIN step: (tmax - tmin) times the total
// variation of its samples' densities (seg_dens, node-major samples) into
// seg_tv[rm]; -1 for a segment whose samples lie past dens_cap.
cudaError_t launch_seg_variation(const SegRec* segs, const int* samp_off, const int64_t* counters,
                                 const float* seg_dens, int64_t dens_cap, float* seg_tv, cudaStream_t st);

// tcgen05 tile kernels (neat_tc.cu); prec 0 = BF16 operands, 1 = three-piece BF16 split.
int tc_backward_grid(int C, int prec);
cudaError_t launch_tiles_tc(int C, int prec, bool bwd, const StepTileArgs& args, cudaStream_t st);

}  // namespace neat
