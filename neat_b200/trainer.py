"""Fused training step: one C-ABI call per Trainer::TrainStep iteration
(samples/reconstruct.cpp:362-403: GetRays -> CreateSamplesForRays(jitter) ->
ComputeImage -> MSE -> backward -> OptimizerStep).

FusedTrainer owns the device state (grid in channel-last layout, decoder,
Adam moments, gradient scratch, step workspace) and issues neat_train_step on
the current stream.  Nothing is synchronised inside a step; the loss stays on
the device until the caller reads it.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from .api import CameraModel, decoder_init, grid_init
from .proposal import proposal_init
from .scene import pixel_to_uv
from .tree import HyperTreeBase


class FusedTrainer:
    def __init__(self, tree: HyperTreeBase, camera: CameraModel, num_features=4, grid_size=17,
                 max_samples_per_node=32, lr_grid=1e-2, lr_decoder=5e-5, softplus_beta=2.0, seed=0, grid=None,
                 decoder=None, seg_capacity_per_ray=None, decoder_path=_lib.NEAT_DECODER_TC_BF16X3, device="cuda",
                 proposal=False, proposal_budget=12, proposal_every=50, proposal_lr=1e-2, proposal_iters=10,
                 proposal_mix=0.25, proposal_count_eps=0.0, proposal_count_min=2, grid_bf16=False, loss_tv=0.0, loss_edge=0.0, edge_epsilon=0.001,
                 tonemap=None, pose_grad=False, optimize_pose=False, optimize_intrinsics=False, lr_pose=1e-3,
                 lr_intrinsics=100.0, record_samples_per_ray=0, cell_map=True):
        self.dev = torch.device(device)
        self.tree, self.camera = tree, camera
        self.C, self.G, self.M = int(num_features), int(grid_size), int(max_samples_per_node)
        self.seed = int(seed)
        A = tree.NumActiveNodes()
        self.A = A
        gen = torch.Generator().manual_seed(seed)
        if grid is None:
            grid = grid_init(A, self.C, self.G, gen)
        if decoder is None:
            decoder = decoder_init(self.C, gen)
        lib = _lib.load()
        self.lib = lib
        grid = grid.to(self.dev, torch.float32).contiguous()
        if tuple(grid.shape) != (A, self.C, self.G, self.G, self.G):
            raise ValueError("grid must be [num_active, C, G, G, G]")
        self.grid = torch.empty((A, self.G, self.G, self.G, self.C), dtype=torch.float32, device=self.dev)
        _lib.check(lib.neat_grid_to_channel_last(grid.data_ptr(), self.grid.data_ptr(), A, self.C, self.G,
                                                 self._stream()), "neat_grid_to_channel_last")
        self.grid_m = torch.zeros_like(self.grid)
        self.grid_v = torch.zeros_like(self.grid)
        self.grid_grad = torch.zeros_like(self.grid)
        self.decoder = decoder.to(self.dev, torch.float32).contiguous().clone()
        if self.decoder.numel() != lib.neat_decoder_params(self.C):
            raise ValueError("decoder has the wrong number of parameters")
        self.decoder_m = torch.zeros_like(self.decoder)
        self.decoder_v = torch.zeros_like(self.decoder)
        self.decoder_grad = torch.zeros_like(self.decoder)
        self.tables = tree.device_tables(self.dev)
        # a line crosses at most 3 * 2^D - 2 cells of a 2^D grid
        self.seg_per_ray = seg_capacity_per_ray or min(_lib.NEAT_MAX_HITS_PER_RAY, 3 * (1 << tree.max_depth))
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.counters = torch.zeros(4, dtype=torch.int64, device=self.dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.desc = _lib.StepDesc(
            tree_table=self.tables["table"].data_ptr(), num_active=A, max_depth=tree.max_depth,
            node_min=self.tables["min"].data_ptr(), node_max=self.tables["max"].data_ptr(), w=camera.w, h=camera.h,
            intrinsics=camera.intrinsics.data_ptr(), rotation=camera.rotation.data_ptr(),
            translation=camera.translation.data_ptr(), C=self.C, G=self.G, softplus_beta=float(softplus_beta),
            max_samples_per_node=self.M, lr_grid=float(lr_grid), lr_decoder=float(lr_decoder), beta1=0.9,
            beta2=0.999, eps=1e-8, seg_capacity=0, decoder_path=int(decoder_path),
            record_samples_per_ray=int(record_samples_per_ray))
        # hits by a DDA over the finest cells when the tree allows (depth <= 5,
        # disjoint active nodes); cell_map=False keeps the level-by-level walk
        self.cell_map = bool(cell_map)
        self.desc.cell_node = self._cell_node_ptr(self.tables)
        # step number kept on the device: a captured graph of the step advances it on replay
        self.step_counter = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.state = _lib.StepState(
            grid=self.grid.data_ptr(), grid_m=self.grid_m.data_ptr(), grid_v=self.grid_v.data_ptr(),
            grid_grad=self.grid_grad.data_ptr(), decoder=self.decoder.data_ptr(),
            decoder_m=self.decoder_m.data_ptr(), decoder_v=self.decoder_v.data_ptr(),
            decoder_grad=self.decoder_grad.data_ptr(), step_counter=self.step_counter.data_ptr())
        self.ws = None
        self.ws_rays = 0
        self._stage = None  # device staging of host batches (see _stage_host)
        self._pf = None     # the next batch's segment lists, built ahead (see step)
        self._cnt = [self.counters, torch.zeros_like(self.counters)]
        self._ci = 0
        self.step_id = 0
        self._graph = None
        self._graphs = {}
        # volume regularisers (GeometryExEx::VolumeRegularizer): their gradients go into
        # grid_grad before the step, whose Adam applies the sum
        self.loss_tv, self.loss_edge, self.edge_epsilon = float(loss_tv), float(loss_edge), float(edge_epsilon)
        self.reg_loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.reg_ws = torch.empty(lib.neat_regularizer_workspace_bytes(), dtype=torch.uint8, device=self.dev)
        # photometric calibration (PhotometricCalibration): tonemap = dict of
        # PhotometricCalibrationParams fields (response_enable, response_range,
        # response_lr, exposure_enable, exposure_mult, exposure_lr,
        # sensor_bias_enable, sensor_bias_size_w, sensor_bias_lr) or None
        self.tonemap = None
        if tonemap is not None:
            self.tonemap = PhotometricCalibration(camera.rotation.shape[0], camera.w, camera.h, self.dev, **tonemap)
            self.state.tonemap = ctypes.addressof(self.tonemap.struct)
        # precision variant: the sample gathers read a BF16 copy of the grid that
        # Adam refreshes from the FP32 master after every update
        self.grid_bf16 = None
        if grid_bf16:
            if decoder_path == _lib.NEAT_DECODER_SIMT_FP32:
                raise ValueError("BF16 grids run with the tensor-core decoder paths")
            self.grid_bf16 = self.grid.to(torch.bfloat16).contiguous()
            self.state.grid_bf16 = self.grid_bf16.data_ptr()
        # learned sample proposal: SAMPLE-mode steps place proposal_budget samples per
        # node segment by the proposal's CDF (with proposal_count_eps > 0: fewer,
        # down to proposal_count_min, where the count head predicts little density
        # variation); every proposal_every-th step (the first included) samples
        # uniformly with max_samples_per_node, bins the contributions and trains
        # the proposal on them
        self.proposal = bool(proposal)
        self.desc.proposal = 1 if self.proposal else 0
        if self.proposal:
            if decoder_path == _lib.NEAT_DECODER_SIMT_FP32:
                raise ValueError("the learned proposal runs with the tensor-core decoder paths")
            self.prop = proposal_init(gen).to(self.dev)
            self.prop_m = torch.zeros_like(self.prop)
            self.prop_v = torch.zeros_like(self.prop)
            self.prop_grad = torch.zeros_like(self.prop)
            self.prop_steps = torch.zeros(1, dtype=torch.int32, device=self.dev)
            # cross-entropy, target entropy, count head's mean squared error / 2
            self.prop_loss = torch.zeros(3, dtype=torch.float32, device=self.dev)
            self.prop_node_desc = torch.zeros((A, 6), dtype=torch.float32, device=self.dev)
            self.prop_every = int(proposal_every)
            self.prop_struct = _lib.Proposal(
                mode=_lib.NEAT_PROPOSAL_OFF, params=self.prop.data_ptr(), m=self.prop_m.data_ptr(),
                v=self.prop_v.data_ptr(), grad=self.prop_grad.data_ptr(), step_counter=self.prop_steps.data_ptr(),
                loss=self.prop_loss.data_ptr(), lr=float(proposal_lr), beta1=0.9, beta2=0.999, eps=1e-8,
                mix=float(proposal_mix), iters=int(proposal_iters), node_desc=self.prop_node_desc.data_ptr(),
                count_eps=float(proposal_count_eps), count_min=int(proposal_count_min))
            self.state.proposal = ctypes.addressof(self.prop_struct)
            self.desc_budget = _lib.StepDesc.from_buffer_copy(self.desc)
            self.desc_budget.max_samples_per_node = int(proposal_budget)
        # camera pose / intrinsics gradients (the reference's structure
        # parameters: rotation tangent, translation, intrinsics), accumulated by
        # every step into pose_grad_*; with optimize_pose / optimize_intrinsics
        # the step is followed by the reference's SGD on them (lr_pose,
        # lr_intrinsics; SceneBase::OptimizerStep), which also zeroes them
        self.optimize_pose, self.optimize_intrinsics = bool(optimize_pose), bool(optimize_intrinsics)
        self.lr_pose, self.lr_intrinsics = float(lr_pose), float(lr_intrinsics)
        self.pose = None
        if pose_grad or self.optimize_pose or self.optimize_intrinsics:
            if decoder_path == _lib.NEAT_DECODER_SIMT_FP32:
                raise ValueError("pose gradients run with the tensor-core decoder paths")
            n_img = camera.rotation.shape[0]
            self.pose_grad_tangent = torch.zeros((n_img, 3), dtype=torch.float64, device=self.dev)
            self.pose_grad_translation = torch.zeros((n_img, 3), dtype=torch.float64, device=self.dev)
            self.pose_grad_intrinsics = torch.zeros(5, dtype=torch.float64, device=self.dev)
            self.pose = _lib.PoseGrad(grad_tangent=self.pose_grad_tangent.data_ptr(),
                                      grad_translation=self.pose_grad_translation.data_ptr(),
                                      grad_intrinsics=self.pose_grad_intrinsics.data_ptr(), num_images=n_img)
            self.desc.pose_grad = 1
            if self.proposal:
                self.desc_budget.pose_grad = 1
            self.state.pose = ctypes.addressof(self.pose)

    def _cell_node_ptr(self, tables):
        cells = tables.get("cell_node")
        return cells.data_ptr() if (self.cell_map and cells is not None) else None

    def _stream(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def reserve(self, num_rays):
        """Allocate the step workspace for batches of up to num_rays rays."""
        if self.ws is not None and num_rays <= self.ws_rays:
            return
        self._drain_prefetch()
        self.desc.seg_capacity = int(num_rays) * self.seg_per_ray
        if self.proposal:
            self.desc_budget.seg_capacity = self.desc.seg_capacity
        nbytes = self.lib.neat_train_step_workspace_bytes(ctypes.byref(self.desc), int(num_rays))
        if nbytes == 0:
            raise _lib.NeatError(_lib.NEAT_ERR_UNSUPPORTED, "neat_train_step_workspace_bytes")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
        self.ws_rays = int(num_rays)

    def _stage_host(self, uv, image_id, target):
        """A host batch (the reference's Dataloader hands the step host tensors,
        src/utils/Dataloader.cpp:8-49) into device staging buffers.  Two buffer
        sets alternate.  A set's copy runs on a copy stream once the step that
        last read the set has finished (an event), and the step waits for its
        own copy (another event), so the copy of the next batch overlaps this
        step's kernels when the caller queues steps ahead.  Pinned host memory
        makes the copies asynchronous; pageable memory is copied by CUDA
        synchronously.  Returns the device views, the set index and the event
        that marks the copies done (the caller's stream waits on it)."""
        R = uv.shape[0]
        if uv.dtype != torch.float32 or image_id.dtype != torch.int32 or target.dtype != torch.float32:
            raise TypeError("host batches: uv float32 [R, 2], image_id int32 [R], target float32 [R]")
        if tuple(uv.shape) != (R, 2) or tuple(image_id.shape) != (R,) or tuple(target.shape) != (R,):
            raise ValueError("host batches: uv [R, 2], image_id [R], target [R]")
        if self._stage is None or self._stage["rays"] < R:
            dev = self.dev
            self._stage = {"rays": R, "next": 0, "stream": torch.cuda.Stream(dev), "used": [None, None],
                           "bufs": [(torch.empty((R, 2), dtype=torch.float32, device=dev),
                                     torch.empty(R, dtype=torch.int32, device=dev),
                                     torch.empty(R, dtype=torch.float32, device=dev)) for _ in range(2)]}
        st = self._stage
        b = st["next"]
        st["next"] = b ^ 1
        cs, cur = st["stream"], torch.cuda.current_stream(self.dev)
        if st["used"][b] is not None:
            cs.wait_event(st["used"][b])
        d_uv, d_img, d_tgt = (t[:R] for t in st["bufs"][b])
        with torch.cuda.stream(cs):
            d_uv.copy_(uv.contiguous(), non_blocking=True)
            d_img.copy_(image_id.contiguous(), non_blocking=True)
            d_tgt.copy_(target.contiguous(), non_blocking=True)
        ready = torch.cuda.Event()
        ready.record(cs)
        return d_uv, d_img, d_tgt, b, ready

    def host_copy_stream(self):
        """The stream that copies host batches in (None before the first one)."""
        return None if self._stage is None else self._stage["stream"]

    def step(self, uv, image_id, target, prediction=None, phase_events=None, next=None):
        """One fused forward+backward+Adam step on a ray batch; returns the
        device loss tensor (mean squared projection error of the batch).
        The batch may be device tensors or host tensors (pinned for an
        asynchronous copy that overlaps the previous step: _stage_host).
        phase_events: optional list of NEAT_STEP_PHASES torch.cuda.Event
        (enable_timing) recorded at the step's phase boundaries.
        next: optional (uv, image_id, target) of the batch that the following
        call takes.  Its segment lists (rays, hit lists, node-major segments,
        tile map: they depend on the batch and the octree only) are then built
        on a side stream while this step's Adam update runs
        (neat_train_step_segments, queued behind the step's phase [4], or [5]
        on a proposal TRAIN step), and that call skips building them
        (neat_train_step_prebuilt).  The following call is recognised by its
        tensors, so their contents must stay as passed until it runs (a loop
        that refills one buffer in place passes next=None).  Ignored while
        poses or intrinsics are optimised (the pose update after the step moves
        the next rays)."""
        cur = torch.cuda.current_stream(self.dev)
        pf, self._pf = self._pf, None
        staged = None
        if not uv.is_cuda:
            key = (uv.data_ptr(), image_id.data_ptr(), target.data_ptr(), uv.shape[0])
            if pf is not None and pf["host_key"] == key:
                uv, image_id, target = pf["dev"]
                staged = pf["set"]
            else:
                uv, image_id, target, staged, ready = self._stage_host(uv, image_id, target)
                cur.wait_event(ready)
        if pf is not None:
            # the workspace's segment buffers and the staged batch, before anything
            # (a reserve() below included) touches them
            cur.wait_event(pf["done"])
        R = uv.shape[0]
        self.reserve(R)
        self.step_id += 1
        train = self.proposal and (self.step_id - 1) % self.prop_every == 0
        prebuilt = (pf is not None and pf["key"] == (uv.data_ptr(), image_id.data_ptr(), R)
                    and pf["train"] == train)
        if prebuilt:
            self._ci = pf["ci"]
        self.counters = self._cnt[self._ci]
        batch = _lib.StepBatch(uv=uv.data_ptr(), image_id=image_id.data_ptr(), target=target.data_ptr(), num_rays=R)
        prefetch = next is not None and not (self.optimize_pose or self.optimize_intrinsics)
        handles = [None] * _lib.NEAT_STEP_PHASES
        if phase_events is not None:
            if len(phase_events) != _lib.NEAT_STEP_PHASES:
                raise ValueError("phase_events needs NEAT_STEP_PHASES events")
            handles = [e.cuda_event for e in phase_events]
            if not all(handles):
                raise ValueError("phase_events must be created (record them once) before use")
        free_phase = 5 if train else 4  # the step's last read of its segment buffers
        free_ev = None
        if prefetch:
            if phase_events is not None:
                free_ev = phase_events[free_phase]
            else:
                free_ev = torch.cuda.Event()
                free_ev.record(cur)  # creates the handle; recorded again by the step
                handles[free_phase] = free_ev.cuda_event
        ev = None
        if any(h is not None for h in handles):
            self._ev_arr = (ctypes.c_void_p * _lib.NEAT_STEP_PHASES)(*handles)
            ev = ctypes.cast(self._ev_arr, ctypes.c_void_p)
        out = _lib.StepOut(loss=self.loss.data_ptr(), counters=self.counters.data_ptr(),
                           status=self.status.data_ptr(),
                           prediction=prediction.data_ptr() if prediction is not None else None,
                           phase_events=ev)
        if self.loss_tv > 0 or self.loss_edge > 0:
            self.regularize()
        desc = self._step_desc(self.step_id)
        fn = self.lib.neat_train_step_prebuilt if prebuilt else self.lib.neat_train_step
        rc = fn(ctypes.byref(desc), ctypes.byref(self.state), ctypes.byref(batch), self.seed, self.step_id,
                ctypes.byref(out), self.ws.data_ptr(), self.ws.numel(), self._stream())
        _lib.check(rc, "neat_train_step_prebuilt" if prebuilt else "neat_train_step")
        if staged is not None:
            done = torch.cuda.Event()
            done.record(cur)
            self._stage["used"][staged] = done  # the set's next copy waits for this step
        if self.optimize_pose or self.optimize_intrinsics:
            self.pose_step()
        if prefetch:
            self._prefetch(next, free_ev)
        return self.loss

    def _drain_prefetch(self):
        """Order a pending look-ahead segment build before whatever follows on
        the current stream (before the workspace is freed or replaced), and
        drop it: the next step builds its own lists."""
        if self._pf is not None:
            torch.cuda.current_stream(self.dev).wait_event(self._pf["done"])
            self._pf = None

    def _step_desc(self, step_id):
        """The step descriptor of step number step_id (with the learned
        proposal: uniform TRAIN steps and budget SAMPLE steps)."""
        if not self.proposal:
            return self.desc
        train = (step_id - 1) % self.prop_every == 0
        self.prop_struct.mode = _lib.NEAT_PROPOSAL_TRAIN if train else _lib.NEAT_PROPOSAL_SAMPLE
        return self.desc if train else self.desc_budget

    def _prefetch(self, nxt, free_ev):
        """The segment lists of the next step's batch nxt on a side stream,
        behind free_ev (the running step's last read of its segment buffers),
        into the workspace and the other counters array (see step)."""
        uv, image_id, target = nxt
        R = uv.shape[0]
        if R > self.ws_rays:
            return  # the next step re-reserves and builds its own lists
        if getattr(self, "_pf_stream", None) is None:
            self._pf_stream = torch.cuda.Stream(self.dev)
        ps = self._pf_stream
        host_key, set_idx = None, None
        if not uv.is_cuda:
            host_key = (uv.data_ptr(), image_id.data_ptr(), target.data_ptr(), R)
            uv, image_id, target, set_idx, ready = self._stage_host(uv, image_id, target)
            ps.wait_event(ready)
        ps.wait_event(free_ev)
        step_id = self.step_id + 1
        train = self.proposal and (step_id - 1) % self.prop_every == 0
        desc = self.desc if (not self.proposal or train) else self.desc_budget
        ci = self._ci ^ 1
        batch = _lib.StepBatch(uv=uv.data_ptr(), image_id=image_id.data_ptr(), target=target.data_ptr(), num_rays=R)
        prop = None
        if self.proposal:
            # the next step's mode; the running step read the struct when it was queued
            self.prop_struct.mode = _lib.NEAT_PROPOSAL_TRAIN if train else _lib.NEAT_PROPOSAL_SAMPLE
            prop = ctypes.addressof(self.prop_struct)
        rc = self.lib.neat_train_step_segments(ctypes.byref(desc), prop, ctypes.byref(batch),
                                               self._cnt[ci].data_ptr(), self.status.data_ptr(), self.ws.data_ptr(),
                                               self.ws.numel(), ps.cuda_stream)
        _lib.check(rc, "neat_train_step_segments")
        done = torch.cuda.Event()
        done.record(ps)
        self._pf = {"key": (uv.data_ptr(), image_id.data_ptr(), R), "host_key": host_key,
                    "dev": (uv, image_id, target), "set": set_idx, "done": done, "ci": ci, "train": train}

    def pose_step(self):
        """The reference's structure optimizer step on the accumulated pose
        gradients (SGD, rotation <- exp(tangent) rotation), which zeroes them."""
        cam = self.camera
        _lib.check(self.lib.neat_pose_sgd(cam.rotation.data_ptr(), cam.translation.data_ptr(),
                                          cam.intrinsics.data_ptr(), ctypes.byref(self.pose), self.lr_pose,
                                          self.lr_intrinsics, int(self.optimize_pose),
                                          int(self.optimize_intrinsics), self._stream()), "neat_pose_sgd")

    def regularize(self):
        """VolumeRegularizer (src/geometry/geometry_ex_ex.cpp:86-156): TV and edge
        losses into self.reg_loss, their gradients into grid_grad."""
        self.reg_loss.zero_()
        st = self._stream()
        if self.loss_tv > 0:
            _lib.check(self.lib.neat_tv_loss(self.grid.data_ptr(), self.A, self.C, self.G, self.loss_tv,
                                             self.reg_loss.data_ptr(), self.grid_grad.data_ptr(),
                                             self.reg_ws.data_ptr(), st), "neat_tv_loss")
        if self.loss_edge > 0:
            t = self.tables
            _lib.check(self.lib.neat_edge_loss(t["table"].data_ptr(), self.tree.max_depth, t["min"].data_ptr(),
                                               t["max"].data_ptr(), t["active"].data_ptr(), self.A,
                                               self.grid.data_ptr(), self.C, self.G, self.edge_epsilon,
                                               self.loss_edge, self.seed, self.step_id, self.reg_loss.data_ptr(),
                                               self.grid_grad.data_ptr(), self.reg_ws.data_ptr(), st),
                       "neat_edge_loss")
        return self.reg_loss

    def graph_step(self, uv, image_id, target):
        """step() replayed from a CUDA graph: the first call for a batch size
        runs the step eagerly and captures it; later calls copy the batch into
        the captured input buffers and replay (one graph launch instead of the
        step's ~20 kernel launches).  Same results as step()."""
        self._drain_prefetch()
        R = uv.shape[0]
        train = self.proposal and self.step_id % self.prop_every == 0
        key = (R, train)
        if getattr(self, "_graph_rays", None) != R:
            self._graphs = {}
            self.reserve(R)
            self._g_uv = uv.detach().clone().contiguous()
            self._g_img = image_id.detach().clone().contiguous()
            self._g_tgt = target.detach().clone().contiguous()
            self._graph_rays = R
        if key not in self._graphs:
            self._g_uv.copy_(uv)
            self._g_img.copy_(image_id)
            self._g_tgt.copy_(target)
            self.step(self._g_uv, self._g_img, self._g_tgt)  # eager: also initialises per-kernel attributes
            torch.cuda.synchronize(self.dev)
            g = torch.cuda.CUDAGraph()
            self.step_id -= 1
            with torch.cuda.graph(g):
                self.step(self._g_uv, self._g_img, self._g_tgt)  # captured for this step's mode, not run
            self._graphs[key] = g
            return self.loss
        self._g_uv.copy_(uv, non_blocking=True)
        self._g_img.copy_(image_id, non_blocking=True)
        self._g_tgt.copy_(target, non_blocking=True)
        self._graphs[key].replay()
        self.step_id += 1
        return self.loss

    def project(self, uv, image_id, target=None, error_sums=None, prediction=None, use_proposal=False,
                samples_per_node=None):
        """Deterministic projection (a = 0.5) of a ray batch with the current
        parameters: the forward of EvalStepProjection
        (samples/reconstruct.cpp:551-559), the trainer's photometric
        calibration applied when it has one (tone_mapper->forward, :559).
        error_sums: optional device f64[2] that receives += sum (pred-target)^2
        and += sum |pred-target|."""
        self._drain_prefetch()  # this call rewrites the workspace's segment buffers
        R = uv.shape[0]
        self.reserve(R)
        if prediction is None:
            prediction = torch.empty(R, dtype=torch.float32, device=self.dev)
        if error_sums is not None and target is None:
            raise ValueError("error_sums needs a target")
        batch = _lib.StepBatch(uv=uv.data_ptr(), image_id=image_id.data_ptr(),
                               target=target.data_ptr() if target is not None else None, num_rays=R)
        out = _lib.ProjectOut(prediction=prediction.data_ptr(),
                              error_sums=error_sums.data_ptr() if error_sums is not None else None,
                              counters=self.counters.data_ptr(), status=self.status.data_ptr(),
                              tonemap=ctypes.addressof(self.tonemap.struct) if self.tonemap is not None else None)
        desc = _lib.StepDesc.from_buffer_copy(self.desc)
        prop = None
        if use_proposal:
            if not self.proposal:
                raise ValueError("this trainer has no proposal")
            prop = _lib.Proposal.from_buffer_copy(self.prop_struct)
            prop.mode = _lib.NEAT_PROPOSAL_SAMPLE
            desc.max_samples_per_node = self.desc_budget.max_samples_per_node
        if samples_per_node is not None:
            if samples_per_node > self.desc.max_samples_per_node:
                raise ValueError("samples_per_node above the workspace's max_samples_per_node")
            desc.max_samples_per_node = int(samples_per_node)
        rc = self.lib.neat_project(ctypes.byref(desc), self.grid.data_ptr(), self.decoder.data_ptr(),
                                   ctypes.byref(prop) if prop is not None else None, ctypes.byref(batch),
                                   ctypes.byref(out), self.ws.data_ptr(), self.ws.numel(), self._stream())
        _lib.check(rc, "neat_project")
        return prediction

    def eval_projection(self, image_ids, projections, rows_per_batch=None):
        """EvalStepProjection (samples/reconstruct.cpp:504-707) at eval_scale 1:
        every pixel of each listed image, row batches of rows_per_batch rows
        (default: as many as fit the reserved workspace), uv = (x/(w-1),
        y/(h-1)) (CoordinatesRow, src/data/SceneBase.cpp:40-58).  Per image
        MSE and L1 are means over its pixels; the results average them over the
        images and PSNR = 10 log10(1 / MSE) (reconstruct.cpp:686-688).
        projections: device [num_images, h, w] f32 targets.  Returns dict(mse,
        l1, psnr, images) with images the predicted [len(image_ids), h, w]."""
        w, h = self.camera.w, self.camera.h
        if rows_per_batch is None:
            rows_per_batch = max(1, min(h, max(self.ws_rays, 1 << 16) // w))
        xs = pixel_to_uv(torch.arange(w, device=self.dev), w)
        out_imgs = torch.empty((len(image_ids), h, w), dtype=torch.float32, device=self.dev)
        sums = torch.zeros((len(image_ids), 2), dtype=torch.float64, device=self.dev)
        for k, img in enumerate(image_ids):
            for r0 in range(0, h, rows_per_batch):
                r1 = min(h, r0 + rows_per_batch)
                ys = pixel_to_uv(torch.arange(r0, r1, device=self.dev), h)
                uv = torch.stack([xs.repeat(r1 - r0), ys.repeat_interleave(w)], 1).contiguous()
                ids = torch.full((uv.shape[0],), int(img), dtype=torch.int32, device=self.dev)
                tgt = projections[int(img), r0:r1].reshape(-1).contiguous()
                self.project(uv, ids, tgt, sums[k], out_imgs[k, r0:r1].view(-1))
        self.check_status()
        per = (sums / float(w * h)).cpu().numpy()
        mse = float(per[:, 0].mean())
        l1 = float(per[:, 1].mean())
        psnr = 10.0 * math.log10(1.0 / mse) if mse > 0 else float("inf")
        return dict(mse=mse, l1=l1, psnr=psnr, images=out_imgs)

    def ComputeMaxDensity(self, image_mask=True):
        """ComputeMaxDensity (samples/reconstruct.cpp:254-286): per active node the
        max decoded density over its G^3 lattice, points outside every image
        masked out (PointInAnyImage) when image_mask.  Writes the tree's
        node_max_density and returns the per-active-node values [A] (device)."""
        out = torch.empty(self.A, dtype=torch.float32, device=self.dev)
        cam = self.camera
        n_img = cam.rotation.shape[0] if image_mask else 0
        t = self.tables
        _lib.check(self.lib.neat_node_max_density(
            t["active"].data_ptr(), self.A, t["min"].data_ptr(), t["max"].data_ptr(), self.grid.data_ptr(), self.C,
            self.G, self.decoder.data_ptr(), float(self.desc.softplus_beta), n_img, cam.w, cam.h,
            cam.intrinsics.data_ptr(), cam.rotation.data_ptr(), cam.translation.data_ptr(), out.data_ptr(),
            self._stream()), "neat_node_max_density")
        self.tree.node_max_density[self.tree.active_node_ids] = out.cpu().numpy()
        return out

    def restructure(self, new_tree):
        """Move to a new active-node structure: InterpolateInactiveNodes
        (src/geometry/geometry_ex_ex.cpp:182-209) fills the new grid rows from
        the current grid, then the optimizer state restarts
        (ResetGeometryOptimizer)."""
        if new_tree.max_depth != self.tree.max_depth:
            raise ValueError("the new tree must have the same max_depth")
        old_tables, old_grid, old_first = self.tables, self.grid, int(self.tree.active_node_ids[0])
        new_tables = new_tree.device_tables(self.dev)
        A = new_tree.NumActiveNodes()
        grid = torch.empty((A, self.G, self.G, self.G, self.C), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.neat_interpolate_grid(
            new_tables["active"].data_ptr(), A, new_tables["min"].data_ptr(), new_tables["max"].data_ptr(),
            old_tables["table"].data_ptr(), self.tree.max_depth, old_first, old_grid.data_ptr(), self.C, self.G,
            grid.data_ptr(), self._stream()), "neat_interpolate_grid")
        self._adopt_tree(new_tree, grid)

    def _adopt_tree(self, new_tree, grid):
        """Point the step at new_tree with `grid` ([A, G, G, G, C]) as its grid:
        fresh Adam moments and gradient buffers, descriptors and workspace
        rebuilt for the new active-node count."""
        new_tables = new_tree.device_tables(self.dev)
        A = new_tree.NumActiveNodes()
        self.tree, self.tables, self.A, self.grid = new_tree, new_tables, A, grid
        self.grid_m = torch.zeros_like(grid)
        self.grid_v = torch.zeros_like(grid)
        self.grid_grad = torch.zeros_like(grid)
        self.decoder_m.zero_()
        self.decoder_v.zero_()
        self.step_counter.zero_()
        for desc in [self.desc] + ([self.desc_budget] if self.proposal else []):
            desc.tree_table = new_tables["table"].data_ptr()
            desc.num_active = A
            desc.cell_node = self._cell_node_ptr(new_tables)
        self.state.grid, self.state.grid_m = grid.data_ptr(), self.grid_m.data_ptr()
        self.state.grid_v, self.state.grid_grad = self.grid_v.data_ptr(), self.grid_grad.data_ptr()
        if self.grid_bf16 is not None:
            self.grid_bf16 = grid.to(torch.bfloat16).contiguous()
            self.state.grid_bf16 = self.grid_bf16.data_ptr()
        if self.proposal:
            self.prop_node_desc = torch.zeros((A, 6), dtype=torch.float32, device=self.dev)
            self.prop_struct.node_desc = self.prop_node_desc.data_ptr()
        self._drain_prefetch()
        self.ws, self.ws_rays, self._graphs = None, 0, {}
        if hasattr(self, "_graph_rays"):
            del self._graph_rays

    def UniformSampledVolume(self, shape):
        """UniformSampledVolume (src/geometry/geometry.cpp:166-248): the decoded
        density on an nx*ny*nz voxel-corner grid of [-1,1]^3, shape = (nx, ny,
        nz).  Returns (volume [1, nz, ny, nx], node_id [nz, ny, nx] int64,
        valid [nz, ny, nx] f32) on the device; voxels outside every active
        node are 0 / node 0 / invalid."""
        nx, ny, nz = (int(v) for v in shape)
        vol = torch.empty((1, nz, ny, nx), dtype=torch.float32, device=self.dev)
        node = torch.empty((nz, ny, nx), dtype=torch.int64, device=self.dev)
        valid = torch.empty((nz, ny, nx), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.neat_sample_volume(
            self.tables["table"].data_ptr(), self.tree.max_depth, self.tables["min"].data_ptr(),
            self.tables["max"].data_ptr(), self.grid.data_ptr(), 1, self.C, self.G, self.decoder.data_ptr(),
            float(self.desc.softplus_beta), nx, ny, nz, vol.data_ptr(), node.data_ptr(), valid.data_ptr(),
            self._stream()), "neat_sample_volume")
        return vol, node, valid

    # ---- checkpoint / resume -------------------------------------------------
    # The reference saves the geometry module, tree and camera per epoch
    # (samples/reconstruct.cpp:36-62, 153-199) but not the optimizer.  This state
    # also holds the Adam moments and the step number (the jitter of a step is
    # keyed on it), so a restored trainer takes the same next step.  The tree is
    # saved as its depth and active-node ids (the node boxes follow from the
    # depth: HyperTreeBase builds them deterministically), so the grid rows are
    # restored onto the nodes they belong to after any restructure().
    def _state_tensors(self):
        names = ["grid", "grid_m", "grid_v", "grid_grad", "decoder", "decoder_m", "decoder_v", "step_counter"]
        if getattr(self, "grid_bf16", None) is not None:
            names.append("grid_bf16")
        if self.proposal:
            # node descriptors: formed on the proposal's TRAIN steps, read by the SAMPLE steps between
            names += ["prop", "prop_m", "prop_v", "prop_steps", "prop_node_desc"]
        t = {n: getattr(self, n) for n in names}
        if self.tonemap is not None:
            t["tonemap_params"] = self.tonemap.params
        if self.optimize_pose or self.optimize_intrinsics:
            t["camera_rotation"] = self.camera.rotation
            t["camera_translation"] = self.camera.translation
            t["camera_intrinsics"] = self.camera.intrinsics
        return t

    def state_dict(self):
        """Copies (on the host) of everything a step reads and updates, plus the
        step number and the seed."""
        torch.cuda.synchronize(self.dev)
        sd = {n: v.detach().cpu().clone() for n, v in self._state_tensors().items()}
        sd["tree_max_depth"] = int(self.tree.max_depth)
        sd["tree_active_node_ids"] = torch.from_numpy(self.tree.active_node_ids.copy())
        sd["step_id"] = int(self.step_id)
        sd["seed"] = int(self.seed)
        return sd

    def load_state_dict(self, sd):
        """Restores a state_dict() of a trainer built with the same tree depth,
        model sizes and options.  When the saved active-node set differs from
        this trainer's (a checkpoint taken after restructure()), the trainer
        first moves to the saved structure; then every value is copied into the
        trainer's buffers, whose device addresses the step descriptors hold."""
        self._drain_prefetch()  # the restored cameras may move the next rays
        if int(sd["seed"]) != self.seed:
            raise ValueError("state was saved by a trainer with another seed")
        if "tree_max_depth" not in sd or "tree_active_node_ids" not in sd:
            raise KeyError("state has no tree (tree_max_depth, tree_active_node_ids)")
        if int(sd["tree_max_depth"]) != self.tree.max_depth:
            raise ValueError(f"state was saved with a depth-{int(sd['tree_max_depth'])} tree, "
                             f"this trainer's tree has depth {self.tree.max_depth}")
        ids = sd["tree_active_node_ids"].cpu().numpy().astype(np.int64)
        if not np.array_equal(ids, self.tree.active_node_ids):
            if ids.size == 0 or ids.min() < 0 or ids.max() >= self.tree.NumNodes() or np.any(np.diff(ids) <= 0):
                raise ValueError("state holds an invalid active-node set")
            tree = self.tree.copy()
            tree.SetActiveNodes(ids)
            self._adopt_tree(tree, torch.empty((tree.NumActiveNodes(), self.G, self.G, self.G, self.C),
                                               dtype=torch.float32, device=self.dev))
        for n, v in self._state_tensors().items():
            if n not in sd:
                raise KeyError(f"state has no {n}")
            if tuple(sd[n].shape) != tuple(v.shape) or sd[n].dtype != v.dtype:
                raise ValueError(f"state {n} has shape {tuple(sd[n].shape)} {sd[n].dtype}, "
                                 f"expected {tuple(v.shape)} {v.dtype}")
            v.copy_(sd[n].to(v.device))
        self.step_id = int(sd["step_id"])
        torch.cuda.synchronize(self.dev)

    def check_status(self):
        st = int(self.status.item())
        if st:
            self.status.zero_()
            raise _lib.NeatError(st, "neat_train_step")

    def grid_reference_layout(self):
        out = torch.empty((self.A, self.C, self.G, self.G, self.G), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.neat_grid_from_channel_last(self.grid.data_ptr(), out.data_ptr(), self.A, self.C, self.G,
                                                        self._stream()), "neat_grid_from_channel_last")
        return out

    def grad_reference_layout(self, t):
        out = torch.empty((self.A, self.C, self.G, self.G, self.G), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.neat_grid_from_channel_last(t.data_ptr(), out.data_ptr(), self.A, self.C, self.G,
                                                        self._stream()), "neat_grid_from_channel_last")
        return out


class PhotometricCalibration:
    """Parameters of the photometric calibration the fused step applies between
    the line integral and the loss (PhotometricCalibrationImpl,
    src/modules/ToneMapper.cpp:139-223; defaults of PhotometricCalibrationParams,
    src/modules/ToneMapper.h:36-47).  Packed exposure_factor [n] | exposure_bias
    [n] | sensor_bias [bias_h][bias_w] | response [25]; the response starts as
    the identity on [0, range] (a gamma-1 curve normalised to the range)."""

    def __init__(self, num_images, w, h, device, response_enable=True, response_range=2.0, response_lr=0.1,
                 exposure_enable=True, exposure_mult=False, exposure_lr=0.01, sensor_bias_enable=True,
                 sensor_bias_size_w=32, sensor_bias_lr=0.05):
        n = int(num_images)
        bw = int(sensor_bias_size_w)
        bh = int(math.ceil(bw * (float(h) / w)))
        P = _lib.NEAT_RESPONSE_PARAMS
        self.num_images, self.bias_w, self.bias_h = n, bw, bh
        self.params = torch.cat([torch.ones(n), torch.zeros(n), torch.zeros(bh * bw),
                                 torch.arange(P, dtype=torch.float32) / (P - 1) * float(response_range)]).to(device)
        self.grad = torch.zeros_like(self.params)
        self.param_loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.struct = _lib.ToneMap(
            exposure=int(bool(exposure_enable)), exposure_mult=int(bool(exposure_mult)),
            sensor_bias=int(bool(sensor_bias_enable)), response=int(bool(response_enable)), num_images=n, bias_w=bw,
            bias_h=bh, response_range=float(response_range), lr_exposure=float(exposure_lr),
            lr_sensor_bias=float(sensor_bias_lr), lr_response=float(response_lr), params=self.params.data_ptr(),
            grad=self.grad.data_ptr(), param_loss=self.param_loss.data_ptr())

    def split(self):
        n, b = self.num_images, self.bias_w * self.bias_h
        p = self.params
        return p[:n], p[n:2 * n], p[2 * n:2 * n + b].reshape(self.bias_h, self.bias_w), p[2 * n + b:]
