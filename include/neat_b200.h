/*
 * neat_b200.h -- C ABI of the B200-native NeAT forward-projection step.
 *
 * All pointers are DEVICE pointers unless a comment says "host".  Buffers are
 * owned by the caller; no entry point allocates device memory.  Every call is
 * asynchronous on the given stream and returns a neat_status describing the
 * launch; data-dependent failures (capacity overflow, too many hits on one
 * ray, non-dyadic boxes) are reported through a device status word that the
 * caller reads after its own synchronisation (neat_status_* codes, OR-ed).
 *
 * Index types follow the reference: node ids / ray ids / sample indices are
 * int64 ("long" in the reference's torch::kLong tensors), coordinates f32,
 * camera model f64.
 */
#ifndef NEAT_B200_H
#define NEAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* neat_stream_t; /* == cudaStream_t */

typedef enum
{
    NEAT_OK                = 0,
    NEAT_ERR_BAD_INPUT     = 1,  /* invalid sizes / pointers (host check)                    */
    NEAT_ERR_CAPACITY      = 2,  /* output or workspace capacity too small (device flag)     */
    NEAT_ERR_TOO_MANY_HITS = 4,  /* > 256 ray-node intersections on one ray (device flag)    */
    NEAT_ERR_NON_DYADIC    = 8,  /* node box not on the dyadic plane grid (device flag)      */
    NEAT_ERR_CUDA          = 16, /* a CUDA launch failed                                      */
    NEAT_ERR_UNSUPPORTED   = 32, /* configuration the kernels were not built for             */
    NEAT_ERR_TIMEOUT       = 64  /* a bounded wait inside a kernel gave up (device flag)     */
} neat_status;

/* Maximum intersections one ray may have; the reference keeps 256 in shared
 * memory (src/structure/HyperTree.cu:220) and overflows silently. */
#define NEAT_MAX_HITS_PER_RAY 256

/* Human-readable message for a status word. host */
const char* neat_status_string(int status);

/* Library version (host). */
int neat_version(void);

/* ----------------------------------------------------------------------- */
/* Camera rays.                                                             */
/* Replaces SceneBase::GetRays (src/data/SceneBase.cpp:171-193):             */
/*   px = u*(w-1), py = v*(h-1)           (UVToPixel, CameraPose.h:20-36)    */
/*   d_c = ((px-cx)/fx, (py-cy)/fy, 1)/|.|  in f64 (Unproject, CameraPose.cu:262-274) */
/*   d = q (x) d_c  in f64                (RotatePointGPUk, CameraPose.cu:20-33) */
/*   o = translation[image]; both cast to f32.                              */
/* intrinsics: [num_cameras, 5] f64 (fx, fy, cx, cy, skew); camera_id may be */
/* NULL (camera 0).  rotation: [num_images, 4] f64 (x, y, z, w);            */
/* translation: [num_images, 3] f64.  origin/direction: [R, 3] f32.          */
/* ----------------------------------------------------------------------- */
int neat_make_rays(const float* uv, const int32_t* image_id, const int32_t* camera_id, int64_t num_rays, int w, int h,
                   const double* intrinsics, const double* rotation, const double* translation, float* origin,
                   float* direction, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Octree node table.                                                        */
/* The reference keeps node_position_min/max [N,3] and active_node_ids [A]  */
/* (src/structure/HyperTree.h:206-240) for the complete breadth-first tree  */
/* of max_depth (HyperTree.cpp:11-132).  neat_tree_prepare packs, for every */
/* node, its plane indices on the dyadic grid of depth max_depth, its        */
/* diagonal (HyperTree.cu:286), its grid row when active and whether an      */
/* active node lies below it, into a caller buffer of                        */
/* neat_tree_table_bytes(max_depth) bytes.  status: device int, OR-ed flags. */
/* ----------------------------------------------------------------------- */
size_t neat_tree_table_bytes(int max_depth);
int neat_tree_prepare(const float* node_min, const float* node_max, const int64_t* active_ids, int num_active,
                      int max_depth, void* table, int* status, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Ray samples.                                                              */
/* Replaces HyperTreeBaseImpl::CreateSamplesForRays (src/structure/HyperTree.h:157, */
/* kernel ComputeRaySamples, src/structure/HyperTree.cu:206-438).  Outputs   */
/* a SampleList (src/structure/HelperStructs.h:168-234) in canonical order:  */
/* ray-major, segments of one ray ordered by (tmin, node_id).  jitter != 0   */
/* draws the stratified offset a from Philox(seed; ray, index_in_ray, step), */
/* else a = 0.5 (the evaluation setting).  out_count (device int64[2]) gets  */
/* the sample count and the max samples of one ray; samples beyond capacity */
/* are not written and NEAT_ERR_CAPACITY is raised in *status.              */
/* workspace: neat_samples_workspace_bytes(num_rays) bytes.                 */
/* ----------------------------------------------------------------------- */
size_t neat_samples_workspace_bytes(int64_t num_rays);
int neat_create_samples(const void* table, int num_active, int max_depth, const float* origin, const float* direction,
                        int64_t num_rays, int max_samples_per_node, int jitter, uint64_t seed, uint32_t step,
                        int64_t capacity, float* coords, float* ray_t, float* weight, int64_t* ray_index,
                        int64_t* local_index_in_ray, int64_t* node_id, int64_t* out_count, int* status,
                        void* workspace, neat_stream_t stream);

/* Same as neat_create_samples, but the caller passes no workspace: the call
 * allocates nothing.  No counterpart in the reference (its sampler always
 * allocates its outputs and a counter with torch).  It exists for callers that
 * cannot allocate device memory while they run -- a host framework that has
 * reserved the GPU's memory for its own pool, or a loop that must not take the
 * implicit device synchronisation a cudaMalloc costs -- and for bindings that
 * can only hand over input and output arrays.  Its per-ray counts and offsets
 * live in one file-scope device array of the library, sized for at most
 * NEAT_NOALLOC_MAX_RAYS rays (about 3 MB, held on every GPU that loads the
 * library until the process exits); larger batches are rejected with
 * NEAT_ERR_CAPACITY before any kernel is launched (out_count is zeroed
 * first, as on the other paths).  Each call looks up that array's device
 * address in the current context (cudaGetSymbolAddress); the first lookup on
 * a device loads the library's module there, so make the first call before
 * any stream capture.  Every call on a device shares the one array, so calls
 * whose work overlaps on the GPU (different streams or threads without
 * ordering) race and must be serialised by the caller. */
#define NEAT_NOALLOC_MAX_RAYS (1 << 18)
int neat_create_samples_noalloc(const void* table, int num_active, int max_depth, const float* origin,
                                const float* direction, int64_t num_rays, int max_samples_per_node, int jitter,
                                uint64_t seed, uint32_t step, int64_t capacity, float* coords, float* ray_t,
                                float* weight, int64_t* ray_index, int64_t* local_index_in_ray, int64_t* node_id,
                                int64_t* out_count, int* status, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Local coordinates.                                                        */
/* Replaces HyperTreeBaseImpl::ComputeLocalSamples (src/structure/HyperTree.cu:177-192): */
/* local = (g - min[node]) / (max[node] - min[node]) * 2 - 1.                */
/* ----------------------------------------------------------------------- */
int neat_local_samples(const float* global, const int64_t* node_id, int64_t num_samples, const float* node_min,
                       const float* node_max, float* local, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* IndirectGridSample3D.                                                     */
/* Replaces IndirectGridSample3D(multi_grid, index, uv) and its autograd    */
/* Function (src/modules/IndirectGridSample3D.h:18-30, .cu:432-892).        */
/* grid: [N, C, Z, Y, X] f32 (reference layout), index: [S] int64 row,      */
/* uv: [S, 3] f32 (x->X, y->Y, z->Z), out: [S, C].                          */
/* Backward accumulates into grad_grid (same shape) and grad_uv [S,3]        */
/* (may be NULL); both must be zeroed by the caller, as the reference's     */
/* torch::zeros_like (IndirectGridSample3D.cu:848-849).                     */
/* ----------------------------------------------------------------------- */
int neat_igs_forward(const float* grid, int64_t N, int C, int Z, int Y, int X, const int64_t* index, const float* uv,
                     int64_t num_samples, float* out, neat_stream_t stream);
int neat_igs_backward(const float* grid, int64_t N, int C, int Z, int Y, int X, const int64_t* index, const float* uv,
                      int64_t num_samples, const float* grad_out, float* grad_grid, float* grad_uv,
                      neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Adam.                                                                     */
/* Replaces torch::optim::Adam::step as used by NeuralGeometry::OptimizerStep */
/* (src/geometry/geometry.h:66-88): bias-corrected, no weight decay, every  */
/* element updated every step.  step is 1-based.  If zero_grad != 0 the     */
/* gradient is cleared after it is read (optimizer->zero_grad()).           */
/* ----------------------------------------------------------------------- */
int neat_adam(float* param, float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, float lr, float beta1,
              float beta2, float eps, int step, int zero_grad, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Decoder layout.                                                           */
/* FCBlock(C, 1, hidden_layers=1, 64, "silu") (src/geometry/ImplicitNet.h:18-73) */
/* + softplus(beta) (src/geometry/geometry.cpp:133-136).  The parameters are */
/* packed in one f32 buffer of neat_decoder_params(C) floats:               */
/*   W1 [64][C] | b1 [64] | W2 [64][64] | b2 [64] | W3 [64] | b3 [1]         */
/* (torch nn.Linear weight layout: [out][in]).                              */
/* ----------------------------------------------------------------------- */
#define NEAT_HIDDEN 64
int64_t neat_decoder_params(int C);

/* ----------------------------------------------------------------------- */
/* ComputeImage over an explicit SampleList.                                 */
/* Replaces HierarchicalNeuralGeometry::ComputeImage (src/geometry/geometry.cpp:347-389) */
/* for GeometryExEx::SampleVolumeIndirect (src/geometry/geometry_ex_ex.cpp:161-180): */
/* local coords -> IGS -> decoder -> softplus -> * weight -> index_add by ray. */
/* grid: [A, C, G, G, G] (reference layout), local_node_id: active row per  */
/* sample (GlobalNodeIdToLocalActiveId).  image: [R] f32, zeroed by caller. */
/* Backward: grad_image [R] -> grad_grid (same layout, zeroed by caller) and */
/* grad_decoder (neat_decoder_params(C) floats, zeroed by caller).           */
/* ----------------------------------------------------------------------- */
int neat_compute_image_forward(const float* grid, int64_t num_rows, int C, int G, const float* decoder,
                               float softplus_beta, const float* coords, const float* weight,
                               const int64_t* ray_index, const int64_t* node_id, const int64_t* local_node_id,
                               const float* node_min, const float* node_max, int64_t num_samples, float* image,
                               neat_stream_t stream);
int neat_compute_image_backward(const float* grid, int64_t num_rows, int C, int G, const float* decoder,
                                float softplus_beta, const float* coords, const float* weight,
                                const int64_t* ray_index, const int64_t* node_id, const int64_t* local_node_id,
                                const float* node_min, const float* node_max, int64_t num_samples,
                                const float* grad_image, float* grad_grid, float* grad_decoder, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Fused training step.                                                      */
/* Replaces one iteration of Trainer::TrainStep (samples/reconstruct.cpp:362-403): */
/*   GetRays -> CreateSamplesForRays(jitter) -> ComputeImage -> MSE loss ->   */
/*   backward -> OptimizerStep (Adam on grid and decoder),                   */
/* without materialising per-sample tensors: rays are cut into node          */
/* segments, segments are bucketed by node, and node-major sample tiles run */
/* the grid lookup, decoder and its backward in one kernel each way.         */
/* The grid is kept channel-last [A, G, G, G, C] (neat_grid_to_channel_last). */
/* ----------------------------------------------------------------------- */
typedef struct
{
    /* octree */
    const void* tree_table; /* from neat_tree_prepare */
    int num_active;
    int max_depth;
    const float* node_min; /* [N,3] */
    const float* node_max; /* [N,3] */
    /* camera */
    int w, h;
    const double* intrinsics;  /* [1,5] */
    const double* rotation;    /* [num_images,4] */
    const double* translation; /* [num_images,3] */
    /* model */
    int C, G;
    float softplus_beta;
    int max_samples_per_node;
    /* optimizer */
    float lr_grid, lr_decoder, beta1, beta2, eps;
    /* capacity of the per-step segment buffers */
    int64_t seg_capacity;
    /* decoder GEMMs: NEAT_DECODER_* */
    int decoder_path;
    /* nonzero: the workspace also holds the proposal's per-segment CDFs and
     * bins, so that state->proposal may be used */
    int proposal;
    /* nonzero: the workspace also holds the per-segment and per-ray pose
     * gradient accumulators, so that state->pose may be used */
    int pose_grad;
    /* tensor-core paths: the forward keeps each sample's placement and
     * gathered features for the backward, with room for this many samples
     * per ray (0: 4 (max_samples_per_node + 1); negative: no records).  A
     * step with more samples than the room recomputes them in the backward. */
    int record_samples_per_ray;
    /* Optional (may be NULL): for a tree of max_depth <= 5 whose active nodes
     * are disjoint, the global id of the active node holding each finest cell,
     * or -1: int32 [2^D][2^D][2^D] (z, y, x), device memory.  At
     * max_depth 5 the step then finds each ray's hits by a 3-D DDA over these
     * cells (a thread a ray; below depth 5 the walk is faster and stays), the
     * same hits and intervals, each node's slab test unchanged (an entry
     * that is no node of the tree raises NEAT_ERR_BAD_INPUT in the status
     * word and counts as -1); NULL keeps the level-by-level octree walk. */
    const int32_t* cell_node;
} neat_step_desc;

/* Decoder paths of the fused step.
 *   SIMT_FP32:  FP32 FFMA on CUDA cores.
 *   TC_BF16X3:  tcgen05 tensor cores, every operand split into three BF16
 *               pieces (24 significant bits), the six cross products of piece
 *               order <= 2 accumulated in FP32 (FP32-level accuracy, checked
 *               at 1e-5 against the f64 oracle).
 *   TC_BF16:    tcgen05 tensor cores on BF16 operands, FP32 accumulation
 *               (the precision variant; error stated against f64). */
#define NEAT_DECODER_SIMT_FP32 0
#define NEAT_DECODER_TC_BF16X3 1
#define NEAT_DECODER_TC_BF16 2

/* ----------------------------------------------------------------------- */
/* Learned sample proposal (no counterpart in the reference, whose sampler  */
/* is uniform stratified: HyperTree.cu:347-358).  A tiny MLP maps a ray-node */
/* segment -- the node's 6-float descriptor, entry and exit points in      */
/* node-local coordinates, chord length over the node edge, the centroid's */
/* projection onto the chord and its distance from it over the spread, one */
/* zero: 16 inputs -- via 32 -> 32 SiLU units to 8 logits over equal sub-  */
/* intervals */
/* of [tmin,tmax].  The node descriptor is the method's own density in the */
/* node, decoded on a 4^3 lattice at every TRAIN call: density-weighted     */
/* centroid (3, local), spread (RMS distance from it), log mean density,   */
/* log(peak / mean);                                                         */
/* p = (1 - mix) softmax + mix / 8.  In SAMPLE mode the step places its     */
/* samples by inverting that piecewise-linear CDF at (j + a_j) / n (weights */
/* by the reference's midpoint rule on the placed positions).  In TRAIN mode */
/* the step samples uniformly (the fallback and the error yardstick), bins */
/* every sample's contribution density * weight into its segment's 8       */
/* sub-intervals and, after its own update, runs `iters` Adam iterations of */
/* the proposal                                                             */
/* on the cross-entropy between p and where the density changes: bin b's    */
/* target is |m_b - m_b-1| + |m_b+1 - m_b| of the binned masses m, each     */
/* segment weighted by its total variation (the midpoint rule is exact on  */
/* constant and linear stretches; its error sits at changes).               */
/* A linear count head on the last hidden layer and the inputs,            */
/* v = bv + Wv . h2 + Uv . f, predicts log(a + 1e-4) of the segment, a =    */
/* (tmax - tmin) sum_j |rho_j - rho_j-1| over the densities of its TRAIN-  */
/* call samples (the midpoint rule with n samples misses about a / (2 n) of */
/* the integral at density jumps).  TRAIN calls train it on the squared     */
/* error over every segment (its gradient stops at h2; it steps at 10x lr); */
/* with count_eps > 0, SAMPLE calls give a segment                          */
/* n = min(n_ref, max(count_min, ceil(exp(v) / count_eps))) samples, n_ref  */
/* the reference's count at the budget: flat and empty segments get fewer. */
/* params: neat_proposal_params() floats,                                   */
/*   W1 [32][16] | b1 [32] | W2 [32][32] | b2 [32] | W3 [8][32] | b3 [8]    */
/*   | Wv [32] | Uv [16] | bv.                                              */
/* ----------------------------------------------------------------------- */
#define NEAT_PROPOSAL_IN 16
#define NEAT_PROPOSAL_HIDDEN 32
#define NEAT_PROPOSAL_BINS 8
#define NEAT_PROPOSAL_OFF 0
#define NEAT_PROPOSAL_SAMPLE 1
#define NEAT_PROPOSAL_TRAIN 2
int64_t neat_proposal_params(void);

typedef struct
{
    int mode;          /* NEAT_PROPOSAL_* for this call */
    float* params;     /* neat_proposal_params() floats */
    float* m;          /* Adam first moment */
    float* v;          /* Adam second moment */
    float* grad;       /* out: gradient of the last training iteration */
    int* step_counter; /* device int: proposal Adam steps taken (advanced on the device) */
    float* loss;       /* optional device f32[3]: mass-weighted mean cross-entropy of the last
                        * iteration and of its targets' entropy (their difference: the KL),
                        * and the count head's mean squared error / 2 */
    float lr, beta1, beta2, eps;
    float mix;         /* uniform share of the sample density, e.g. 0.1 */
    int iters;         /* Adam iterations per TRAIN call */
    float* node_desc;  /* [num_active][6] node descriptors, written by TRAIN calls */
    float count_eps;   /* > 0: SAMPLE calls take the count head's sample counts (above); 0: n_ref */
    int count_min;     /* fewest samples a segment gets under count_eps (>= 1 when count_eps > 0) */
} neat_proposal;

/* ----------------------------------------------------------------------- */
/* Camera pose and intrinsics gradients of the step's loss: the reference's */
/* autograd through SceneBase::GetRays (src/data/SceneBase.cpp:171-193),    */
/* RotatePoint (src/modules/CameraPose.cu:37-127, left tangent at 0),       */
/* CameraModelModuleImpl::Unproject (CameraPose.cu:262-274) and the sample  */
/* positions o[ray] + d[ray] t with t held constant (HyperTree.cu:426-432),  */
/* IGS's uv gradient and the local coordinates.  Accumulated (added) into:  */
/*   grad_tangent     [num_images, 3] f64: rotation tangent                 */
/*   grad_translation [num_images, 3] f64                                   */
/*   grad_intrinsics  [5] f64: fx, fy, cx, cy, skew (skew's is 0: unused)   */
/* Requires a tensor-core decoder path and desc->pose_grad.                 */
/* ----------------------------------------------------------------------- */
typedef struct
{
    double* grad_tangent;
    double* grad_translation;
    double* grad_intrinsics;
    int num_images;
} neat_pose_grad;

/* The reference's structure optimizer step (SceneBase::OptimizerStep,      */
/* src/data/SceneBase.cpp:103-118, 232-240): plain SGD with lr_pose on the  */
/* rotation tangent and translation (when optimize_pose) and lr_intrinsics  */
/* on the intrinsics (when optimize_intrinsics), then the tangent applied   */
/* to the rotation, q <- exp(tangent) * q (CameraPoseModuleImpl::ApplyTangent, */
/* CameraPose.cu:163-183; the product renormalised), and the gradients      */
/* zeroed (zero_grad).  rotation [num_images, 4] (x, y, z, w), translation  */
/* [num_images, 3], intrinsics [5], all f64 device arrays, updated in place. */
int neat_pose_sgd(double* rotation, double* translation, double* intrinsics, const neat_pose_grad* grad,
                  double lr_pose, double lr_intrinsics, int optimize_pose, int optimize_intrinsics,
                  neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Photometric calibration fused into the loss (PhotometricCalibration,     */
/* src/modules/ToneMapper.cpp:139-223, optimised by SGD in                   */
/* SceneBase::OptimizerStep, src/data/SceneBase.cpp:121-157, 232-263):       */
/*   y = I * exposure_factor[img] (if exposure_mult) + exposure_bias[img]    */
/*       + sensor_bias(uv)  (bilinear, border, align_corners false)          */
/*   y = response(y)  (25-point curve over [0, range], linear interpolation, */
/*       border; + (y - range) above range while training)                  */
/* then the loss compares y with the target.  The step adds the response's  */
/* smoothness loss (CameraResponseNet::ParamLoss) to its gradient, takes one */
/* SGD step per group and clamps the biases at 0 (ApplyConstraints).         */
/* params (packed): exposure_factor [num_images] | exposure_bias            */
/* [num_images] | sensor_bias [bias_h][bias_w] | response [25].             */
/* ----------------------------------------------------------------------- */
#define NEAT_RESPONSE_PARAMS 25
typedef struct
{
    int exposure, exposure_mult, sensor_bias, response; /* enables */
    int num_images, bias_w, bias_h;
    float response_range;                               /* e.g. 2 */
    float lr_exposure, lr_sensor_bias, lr_response;     /* SGD learning rates */
    float* params;                                      /* packed, see above */
    float* grad;                                        /* same layout: zero on entry, left zero */
    float* param_loss;                                  /* optional device f32: ParamLoss of the step */
} neat_tonemap;

typedef struct
{
    float* grid;       /* [A, G,G,G, C] channel-last */
    float* grid_m;     /* Adam first moment, same shape */
    float* grid_v;     /* Adam second moment */
    float* grid_grad;  /* gradient accumulator, same shape: zero on entry, or holding terms to add
                        * (e.g. the regularisers'); the step adds its own, Adam applies the sum
                        * and the step leaves it zero */
    float* decoder;    /* neat_decoder_params(C) */
    float* decoder_m;
    float* decoder_v;
    float* decoder_grad;
    /* optional device int: when set, the step number is (*step_counter + 1),
     * incremented on the device at the start of the step, and the `step`
     * argument is ignored -- a captured CUDA graph of the step then advances
     * by itself on every replay.  NULL: the `step` argument is used. */
    int* step_counter;
    /* optional learned proposal (requires desc->proposal != 0); NULL: off */
    const neat_proposal* proposal;
    /* optional BF16 copy of the grid ([A, G,G,G, C] bf16, 16-byte aligned):
     * when set, the sample gathers read it (the precision variant: BF16
     * feature grids, FP32 accumulation) and Adam refreshes it from the FP32
     * master after every update; gradients stay FP32.  Requires a tensor-core
     * decoder path. */
    uint16_t* grid_bf16;
    /* optional photometric calibration between the line integral and the loss; NULL: identity */
    const neat_tonemap* tonemap;
    /* optional camera pose / intrinsics gradients (requires desc->pose_grad); NULL: off */
    const neat_pose_grad* pose;
} neat_step_state;

typedef struct
{
    const float* uv;         /* [R,2] in [0,1] */
    const int32_t* image_id; /* [R] */
    const float* target;     /* [R] */
    int64_t num_rays;
} neat_step_batch;

typedef struct
{
    float* loss;        /* device f32[1]: mean squared error of the batch */
    int64_t* counters;  /* device int64[4]: segments, samples, max hits per ray, tiles */
    int* status;        /* device int: OR-ed neat_status flags */
    float* prediction;  /* optional [R] predicted projection (may be NULL) */
    /* optional: NEAT_STEP_PHASES cudaEvent_t handles recorded on the step's
     * stream at the phase boundaries: [0] start, [1] segment lists built,
     * [2] forward tiles done, [3] loss done, [4] backward tiles done,
     * [5] Adam done.  NULL disables. */
    void* const* phase_events;
} neat_step_out;

#define NEAT_STEP_PHASES 6

size_t neat_train_step_workspace_bytes(const neat_step_desc* desc, int64_t num_rays);
int neat_train_step(const neat_step_desc* desc, const neat_step_state* state, const neat_step_batch* batch,
                    uint64_t seed, int step, const neat_step_out* out, void* workspace, size_t workspace_bytes,
                    neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Pipelined steps (optional): the next batch's segment lists built while   */
/* the running step's Adam update runs.  The lists depend on the batch and */
/* the octree only, not on any parameter, so the training loop of          */
/* samples/reconstruct.cpp (TrainStep over Dataloader batches) may build   */
/* them one step ahead.                                                     */
/* neat_train_step_segments runs phase [1] of a step (rays, hit lists,      */
/* node-major segments, sample offsets, tile map) for `batch` into          */
/* `workspace` (neat_train_step_workspace_bytes bytes) and `counters` /     */
/* `status` (as neat_step_out); with a learned proposal in SAMPLE mode      */
/* (`proposal`, as the step will pass it in its state) also the segments'   */
/* placement CDF, which depends on the proposal's parameters and node       */
/* descriptors (final once the TRAIN step that updates them has ended).     */
/* neat_train_step_prebuilt is neat_train_step for that batch without       */
/* phase [1] (nor, in SAMPLE mode, the CDF): same arguments, with           */
/* out->counters = the counters neat_train_step_segments filled.            */
/* A step reads the segment buffers up to its phase [4] (backward done),    */
/* or up to [5] when it trains the learned proposal: queue                  */
/* neat_train_step_segments on a second stream behind that phase event of  */
/* the running step (its counters must be another array than the running   */
/* step's), and the prebuilt step behind the segments' completion.         */
/* ----------------------------------------------------------------------- */
int neat_train_step_segments(const neat_step_desc* desc, const neat_proposal* proposal, const neat_step_batch* batch,
                             int64_t* counters, int* status, void* workspace, size_t workspace_bytes,
                             neat_stream_t stream);
int neat_train_step_prebuilt(const neat_step_desc* desc, const neat_step_state* state, const neat_step_batch* batch,
                             uint64_t seed, int step, const neat_step_out* out, void* workspace,
                             size_t workspace_bytes, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Projection (evaluation).                                                  */
/* Replaces the per-batch forward of EvalStepProjection                     */
/* (samples/reconstruct.cpp:551-583): GetRays -> CreateSamplesForRays with   */
/* interval_jitter = false (a = 0.5, HyperTree.cu:347-358) -> ComputeImage, */
/* through the step's segment pipeline and forward tiles; no gradients, no */
/* parameter update.  grid: channel-last [A, G,G,G, C]; decoder packed as   */
/* above.  batch->target may be NULL unless error_sums is given.            */
/* error_sums (optional, device f64[2]): += sum (pred - target)^2 and        */
/* += sum |pred - target| over the batch, added in a fixed order.            */
/* Workspace: neat_train_step_workspace_bytes(desc, num_rays) bytes.         */
/* proposal: NULL (uniform stratified, a = 0.5) or a learned proposal in    */
/* NEAT_PROPOSAL_SAMPLE mode (samples at the CDF inverse of (j + 0.5) / n). */
/* ----------------------------------------------------------------------- */
typedef struct
{
    float* prediction;  /* device [R] */
    double* error_sums; /* optional device f64[2], accumulated */
    int64_t* counters;  /* device int64[4], as neat_step_out */
    int* status;        /* device int, OR-ed neat_status flags */
    /* optional (host struct, may be NULL): the photometric calibration the   */
    /* evaluation applies to the prediction before the error sums, as        */
    /* EvalStepProjection calls tone_mapper->forward (samples/reconstruct.cpp:559); */
    /* uses batch->uv and batch->image_id.                                    */
    const neat_tonemap* tonemap;
} neat_project_out;

int neat_project(const neat_step_desc* desc, const float* grid, const float* decoder, const neat_proposal* proposal,
                 const neat_step_batch* batch, const neat_project_out* out, void* workspace, size_t workspace_bytes,
                 neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Volume regularisers (GeometryExEx::VolumeRegularizer,                    */
/* src/geometry/geometry_ex_ex.cpp:86-156).  Both ADD their gradient into   */
/* grid_grad (channel-last, may be NULL) and their loss into *loss (device  */
/* f32): run them on the step's stream right before neat_train_step, whose  */
/* Adam applies the summed gradient.  workspace:                             */
/* neat_regularizer_workspace_bytes() bytes.                                 */
/* TV (TVLoss, geometry_ex_ex.h:18-58): weight * C * sum over the 3 grid     */
/* axes of mean_node mean_{c,cells} |neighbour difference|.                  */
/* Edge (NodeNeighborSamples, src/structure/HyperTree.cu:830-928): on each  */
/* face of each active node a G x G lattice of points; where the point      */
/* moved by epsilon outwards lies in another active node, the pair's error  */
/* is mean_c |f_node - f_other| * r, r uniform in [0,1) (Philox keyed on    */
/* (node, face point, step) with seed; torch::rand_like in the reference);  */
/* loss = weight * C * mean over pairs.                                      */
/* ----------------------------------------------------------------------- */
size_t neat_regularizer_workspace_bytes(void);
int neat_tv_loss(const float* grid, int64_t A, int C, int G, float weight, float* loss, float* grid_grad,
                 void* workspace, neat_stream_t stream);
int neat_edge_loss(const void* tree_table, int max_depth, const float* node_min, const float* node_max,
                   const int64_t* active_ids, int64_t A, const float* grid, int C, int G, float epsilon, float weight,
                   uint64_t seed, uint32_t step, float* loss, float* grid_grad, void* workspace, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Structure updates (the decisions stay on the host).                       */
/* neat_node_max_density: ComputeMaxDensity (samples/reconstruct.cpp:254-286): */
/* per active node the max decoded density over its G^3 lattice (cell       */
/* (x,y,z) at local (x,y,z)/(G-1) * size + min, UniformGlobalSamples,       */
/* src/structure/HyperTree.cu:781-815), points outside every image masked   */
/* to 0 when num_images > 0 (PointInAnyImage, src/data/SceneBase.cu:13-45). */
/* grid channel-last; out_max [num_active] f32.                              */
/* neat_interpolate_grid: InterpolateInactiveNodes                          */
/* (src/geometry/geometry_ex_ex.cpp:182-209): the new tree's grid rows from */
/* the old grid at the new nodes' lattice points (old node by the top-down  */
/* descent in the old tree's table; outside every old active node the first */
/* old active node, as NodeIdForPositionGPU returns).  Both grids channel-  */
/* last; node_min/max of the complete tree (shared by old and new).         */
/* ----------------------------------------------------------------------- */
int neat_node_max_density(const int64_t* active_ids, int64_t num_active, const float* node_min, const float* node_max,
                          const float* grid, int C, int G, const float* decoder, float softplus_beta, int num_images,
                          int w, int h, const double* intrinsics, const double* rotation, const double* translation,
                          float* out_max, neat_stream_t stream);
int neat_interpolate_grid(const int64_t* new_active_ids, int64_t new_num_active, const float* node_min,
                          const float* node_max, const void* old_tree_table, int max_depth, int64_t old_first_active,
                          const float* old_grid, int C, int G, float* new_grid, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Volume export.                                                            */
/* Replaces HierarchicalNeuralGeometry::UniformSampledVolume                */
/* (src/geometry/geometry.cpp:166-248) with VolumeSamples / NodeIdForPositionGPU */
/* (src/structure/HyperTree.cu:546-672): voxel (x,y,z) of an nx*ny*nz volume */
/* sits at p = (c / (n-1)) * 2 - 1 per axis and takes the decoded density   */
/* (softplus output) of the active node that the top-down descent finds;    */
/* voxels outside every active node get value 0, node 0, valid 0.           */
/* grid: channel-last [A,G,G,G,C] (channel_last != 0, 16-byte aligned) or   */
/* the reference layout [A,C,G,G,G].  out: [nz][ny][nx] f32 (x fastest);    */
/* out_node [nz][ny][nx] int64 and out_valid f32 are optional.              */
/* ----------------------------------------------------------------------- */
int neat_sample_volume(const void* tree_table, int max_depth, const float* node_min, const float* node_max,
                       const float* grid, int channel_last, int C, int G, const float* decoder, float softplus_beta,
                       int nx, int ny, int nz, float* out, int64_t* out_node, float* out_valid,
                       neat_stream_t stream);

/* Grid layout conversion between the reference's [A, C, G,G,G] and the     */
/* step's channel-last [A, G,G,G, C].                                        */
int neat_grid_to_channel_last(const float* src, float* dst, int64_t A, int C, int G, neat_stream_t stream);
int neat_grid_from_channel_last(const float* src, float* dst, int64_t A, int C, int G, neat_stream_t stream);

/* ----------------------------------------------------------------------- */
/* Synthetic scans (stand-in for the reference's measured projections).     */
/* objects: [n, 17] f64 = centre(3), semi-axes(3), R(9, local = R^T (p-c)),  */
/* density, kind (0 additive ellipsoid, 1 void).  Projection [n_img, h, w]   */
/* f32 of line integrals through pixel centres; density volume [n^3] at     */
/* voxel-corner positions -1 + 2 i/(n-1), x fastest.                         */
/* ----------------------------------------------------------------------- */
int neat_synth_project(const double* objects, int num_objects, int num_images, int w, int h,
                       const double* intrinsics, const double* rotation, const double* translation, float* out,
                       neat_stream_t stream);
int neat_synth_density(const double* objects, int num_objects, const double* points, int64_t num_points,
                       double* out, neat_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* NEAT_B200_H */
