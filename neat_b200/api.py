"""Reference-facing API of the hot path, on libneat_b200.

Names, argument meaning, layouts and error behaviour mirror darglein/NeAT's
libtorch modules so a caller of the reference can switch:

  SceneBase::GetRays                     -> GetRays            (src/data/SceneBase.cpp:171-193)
  HyperTreeBaseImpl::CreateSamplesForRays -> CreateSamplesForRays (src/structure/HyperTree.cu:393-438)
  HyperTreeBaseImpl::ComputeLocalSamples -> ComputeLocalSamples (src/structure/HyperTree.cu:116-199)
  IndirectGridSample3D (+ autograd)      -> IndirectGridSample3D (src/modules/IndirectGridSample3D.cu:804-892)
  GeometryExEx / ComputeImage            -> GeometryExEx.ComputeImage (src/geometry/geometry.cpp:347-389)
  NeuralGeometry::OptimizerStep          -> GeometryExEx.OptimizerStep (src/geometry/geometry.h:66-88)

The reference aborts through glog CHECKs on bad input; here the same
conditions raise ValueError / NeatError.  Every op runs on CUDA tensors
through the C ABI; there is no CPU path.
"""
from dataclasses import dataclass

import torch

from . import _lib
from .tree import HyperTreeBase


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


def _need_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("libneat_b200 ops take CUDA tensors only (no CPU fallback)")


@dataclass
class RayList:
    """src/structure/HelperStructs.h:92-164: origin/direction float [R, 3]."""
    origin: torch.Tensor
    direction: torch.Tensor

    def size(self):
        return self.origin.shape[0]


@dataclass
class SampleList:
    """src/structure/HelperStructs.h:168-234."""
    global_coordinate: torch.Tensor  # float [S, 3]
    ray_t: torch.Tensor              # float [S]
    weight: torch.Tensor             # float [S]
    ray_index: torch.Tensor          # long [S]
    local_index_in_ray: torch.Tensor # long [S]
    node_id: torch.Tensor            # long [S]
    max_samples_per_ray: int = 0

    def size(self):
        return self.global_coordinate.shape[0]


class CameraModel:
    """Pinhole camera + per-image poses (CameraModelModule / CameraPoseModule)."""

    def __init__(self, w, h, intrinsics, rotation, translation, device="cuda"):
        self.w, self.h = int(w), int(h)
        dev = torch.device(device)
        self.intrinsics = torch.as_tensor(intrinsics, dtype=torch.float64).reshape(-1, 5).to(dev).contiguous()
        self.rotation = torch.as_tensor(rotation, dtype=torch.float64).reshape(-1, 4).to(dev).contiguous()
        self.translation = torch.as_tensor(translation, dtype=torch.float64).reshape(-1, 3).to(dev).contiguous()

    @classmethod
    def from_scene(cls, scene):
        return cls(scene.w, scene.h, scene.intr_t, scene.rot_t, scene.trans_t, scene.device)


def GetRays(camera, uv, image_id, camera_id=None):
    """RayList for pixels uv [R,2] in [0,1] of images image_id [R] (int32)."""
    _need_cuda(uv, image_id)
    if uv.dim() != 2 or uv.shape[1] != 2 or image_id.shape[0] != uv.shape[0]:
        raise ValueError("GetRays: uv must be [R,2] and image_id [R]")
    uv = uv.float().contiguous()
    image_id = image_id.to(torch.int32).contiguous()
    cid = camera_id.to(torch.int32).contiguous() if camera_id is not None else None
    R = uv.shape[0]
    o = torch.empty((R, 3), dtype=torch.float32, device=uv.device)
    d = torch.empty((R, 3), dtype=torch.float32, device=uv.device)
    lib = _lib.load()
    _lib.check(lib.neat_make_rays(uv.data_ptr(), image_id.data_ptr(), cid.data_ptr() if cid is not None else None, R,
                                  camera.w, camera.h, camera.intrinsics.data_ptr(), camera.rotation.data_ptr(),
                                  camera.translation.data_ptr(), o.data_ptr(), d.data_ptr(), _stream(uv)),
               "neat_make_rays")
    return RayList(o, d)


def CreateSamplesForRays(tree: HyperTreeBase, rays: RayList, max_samples_per_node: int, interval_jitter: bool,
                         seed: int = 0, step: int = 1):
    """Stratified samples of every ray in every active node it crosses.

    Like the reference this synchronises once to learn the sample count.  The
    capacity is the reference's estimate R * M * A^(1/3) (HyperTree.cu:398),
    grown and retried if a scene needs more."""
    _need_cuda(rays.origin, rays.direction)
    if max_samples_per_node < 1:
        raise ValueError("max_samples_per_node must be >= 1")
    dev = rays.origin.device
    t = tree.device_tables(dev)
    R = rays.size()
    A = tree.NumActiveNodes()
    o = rays.origin.float().contiguous()
    d = rays.direction.float().contiguous()
    lib = _lib.load()
    ws = torch.empty(max(lib.neat_samples_workspace_bytes(R), 16), dtype=torch.uint8, device=dev)
    cap = int(-(-R * max_samples_per_node * (A ** (1.0 / 3.0)) // 1)) + 1
    while True:
        out = SampleList(torch.empty((cap, 3), dtype=torch.float32, device=dev),
                         torch.empty(cap, dtype=torch.float32, device=dev),
                         torch.empty(cap, dtype=torch.float32, device=dev),
                         torch.empty(cap, dtype=torch.int64, device=dev),
                         torch.empty(cap, dtype=torch.int64, device=dev),
                         torch.empty(cap, dtype=torch.int64, device=dev))
        count = torch.zeros(2, dtype=torch.int64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(lib.neat_create_samples(t["table"].data_ptr(), A, tree.max_depth, o.data_ptr(), d.data_ptr(), R,
                                           max_samples_per_node, int(bool(interval_jitter)), seed & (2 ** 64 - 1),
                                           step, cap, out.global_coordinate.data_ptr(), out.ray_t.data_ptr(),
                                           out.weight.data_ptr(), out.ray_index.data_ptr(),
                                           out.local_index_in_ray.data_ptr(), out.node_id.data_ptr(),
                                           count.data_ptr(), status.data_ptr(), ws.data_ptr(), _stream(o)),
                   "neat_create_samples")
        cnt = count.cpu()
        st = int(status.item())
        S = int(cnt[0])
        if st & _lib.NEAT_ERR_CAPACITY and S > cap:
            cap = S
            continue
        if st:
            raise _lib.NeatError(st, "CreateSamplesForRays")
        out.global_coordinate = out.global_coordinate[:S]
        out.ray_t = out.ray_t[:S]
        out.weight = out.weight[:S]
        out.ray_index = out.ray_index[:S]
        out.local_index_in_ray = out.local_index_in_ray[:S]
        out.node_id = out.node_id[:S]
        out.max_samples_per_ray = int(cnt[1])
        return out


def ComputeLocalSamples(tree: HyperTreeBase, global_samples, node_indices):
    """local = (g - min[node]) / (max[node] - min[node]) * 2 - 1, [S,3]."""
    _need_cuda(global_samples, node_indices)
    g = global_samples.float().contiguous().reshape(-1, 3)
    nid = node_indices.to(torch.int64).contiguous().reshape(-1)
    if nid.shape[0] != g.shape[0]:
        raise ValueError("ComputeLocalSamples: one node id per sample")
    t = tree.device_tables(g.device)
    out = torch.empty_like(g)
    _lib.check(_lib.load().neat_local_samples(g.data_ptr(), nid.data_ptr(), g.shape[0], t["min"].data_ptr(),
                                              t["max"].data_ptr(), out.data_ptr(), _stream(g)),
               "neat_local_samples")
    return out.reshape(global_samples.shape)


class _IndirectGridSample3DFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, multi_grid, index, uv):
        N, C, Z, Y, X = multi_grid.shape
        S = index.shape[0]
        out = torch.zeros((S, C), dtype=torch.float32, device=multi_grid.device)
        _lib.check(_lib.load().neat_igs_forward(multi_grid.data_ptr(), N, C, Z, Y, X, index.data_ptr(),
                                                uv.data_ptr(), S, out.data_ptr(), _stream(multi_grid)),
                   "neat_igs_forward")
        ctx.save_for_backward(multi_grid, index, uv)
        return out

    @staticmethod
    def backward(ctx, grad_output):
        multi_grid, index, uv = ctx.saved_tensors
        N, C, Z, Y, X = multi_grid.shape
        go = grad_output.float().contiguous()
        grad_grid = torch.zeros_like(multi_grid)
        grad_uv = torch.zeros_like(uv)
        _lib.check(_lib.load().neat_igs_backward(multi_grid.data_ptr(), N, C, Z, Y, X, index.data_ptr(),
                                                 uv.data_ptr(), index.shape[0], go.data_ptr(),
                                                 grad_grid.data_ptr(), grad_uv.data_ptr(), _stream(multi_grid)),
                   "neat_igs_backward")
        return grad_grid, None, grad_uv


def IndirectGridSample3D(multi_grid, index, uv):
    """out[i, c] = trilinear(multi_grid[index[i], c], uv[i]) with align_corners
    and index-clamped border; multi_grid [N,C,Z,Y,X] f32, index [S] long,
    uv [S,3] f32 (x, y, z)."""
    if multi_grid is None or index is None or uv is None:
        raise ValueError("IndirectGridSample3D: undefined tensor")
    if multi_grid.dim() != 5 or index.dim() != 1 or uv.dim() != 2 or uv.shape[1] != 3:
        raise ValueError("IndirectGridSample3D: expected grid [N,C,Z,Y,X], index [S], uv [S,3]")
    _need_cuda(multi_grid, index, uv)
    if multi_grid.dtype != torch.float32 or uv.dtype != torch.float32 or index.dtype != torch.int64:
        raise ValueError("IndirectGridSample3D: grid/uv float32, index int64")
    return _IndirectGridSample3DFn.apply(multi_grid.contiguous(), index.contiguous(), uv.contiguous())


# --------------------------------------------------------------------------
# model
# --------------------------------------------------------------------------
def decoder_init(C, generator=None, hidden=_lib.NEAT_HIDDEN):
    """FCBlock(C, 1, hidden_layers=1, 64) init (src/geometry/ImplicitNet.h:25-31):
    kaiming_normal_(fan_in, relu) weights, nn.Linear default bias
    U(-1/sqrt(fan_in), 1/sqrt(fan_in)).  Packed W1|b1|W2|b2|W3|b3, f32 (CPU)."""
    g = generator
    parts = []
    for fin, fout in ((C, hidden), (hidden, hidden), (hidden, 1)):
        w = torch.randn((fout, fin), generator=g, dtype=torch.float32) * (2.0 / fin) ** 0.5
        b = (torch.rand((fout,), generator=g, dtype=torch.float32) * 2 - 1) / fin ** 0.5
        parts += [w.reshape(-1), b]
    return torch.cat(parts)


def grid_init(rows, C, G, generator=None, init="uniform"):
    """ExplicitFeatureGrid init (src/geometry/ImplicitNet.h:92-107)."""
    if init in ("uniform", "random"):
        return torch.rand((rows, C, G, G, G), generator=generator, dtype=torch.float32) * 2 - 1
    if init == "minus":
        return -torch.ones((rows, C, G, G, G))
    if init == "zero":
        return torch.zeros((rows, C, G, G, G))
    raise ValueError(f"Unknown grid init: {init}. Expected: uniform, minus, zero")


def split_decoder(dec, C, hidden=_lib.NEAT_HIDDEN):
    """Packed decoder -> (W1 [64,C], b1, W2 [64,64], b2, W3 [1,64], b3)."""
    sizes = [hidden * C, hidden, hidden * hidden, hidden, hidden, 1]
    ws = torch.split(dec, sizes)
    return ws[0].reshape(hidden, C), ws[1], ws[2].reshape(hidden, hidden), ws[3], ws[4].reshape(1, hidden), ws[5]


class _ComputeImageFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, grid, decoder, geom, samples_t, num_pixels):
        coords, weight, ray_index, node_id, local_id = samples_t
        rows, C, G = grid.shape[0], grid.shape[1], grid.shape[2]
        t = geom.tree.device_tables(grid.device)
        image = torch.zeros(num_pixels, dtype=torch.float32, device=grid.device)
        _lib.check(_lib.load().neat_compute_image_forward(
            grid.data_ptr(), rows, C, G, decoder.data_ptr(), geom.softplus_beta, coords.data_ptr(),
            weight.data_ptr(), ray_index.data_ptr(), node_id.data_ptr(), local_id.data_ptr(), t["min"].data_ptr(),
            t["max"].data_ptr(), coords.shape[0], image.data_ptr(), _stream(grid)), "neat_compute_image_forward")
        ctx.geom = geom
        ctx.save_for_backward(grid, decoder, coords, weight, ray_index, node_id, local_id)
        return image.reshape(1, num_pixels)

    @staticmethod
    def backward(ctx, grad_image):
        grid, decoder, coords, weight, ray_index, node_id, local_id = ctx.saved_tensors
        geom = ctx.geom
        rows, C, G = grid.shape[0], grid.shape[1], grid.shape[2]
        t = geom.tree.device_tables(grid.device)
        gi = grad_image.reshape(-1).float().contiguous()
        grad_grid = torch.zeros_like(grid)
        grad_dec = torch.zeros_like(decoder)
        _lib.check(_lib.load().neat_compute_image_backward(
            grid.data_ptr(), rows, C, G, decoder.data_ptr(), geom.softplus_beta, coords.data_ptr(),
            weight.data_ptr(), ray_index.data_ptr(), node_id.data_ptr(), local_id.data_ptr(), t["min"].data_ptr(),
            t["max"].data_ptr(), coords.shape[0], gi.data_ptr(), grad_grid.data_ptr(), grad_dec.data_ptr(),
            _stream(grid)), "neat_compute_image_backward")
        return grad_grid, grad_dec, None, None, None


class GeometryExEx:
    """Explicit per-node feature grids + decoder (GeometryExEx,
    src/geometry/geometry_ex_ex.cpp:10-50) with the two Adam groups of
    NeuralGeometry (grid lr_exex_grid_adam, decoder decoder_lr)."""

    def __init__(self, tree, num_features=4, grid_size=17, max_active_nodes=None, softplus_beta=2.0,
                 lr_grid=1e-2, lr_decoder=5e-5, seed=0, grid_init_mode="uniform", device="cuda"):
        self.tree = tree
        self.C, self.G = int(num_features), int(grid_size)
        self.softplus_beta = float(softplus_beta)
        self.lr_grid, self.lr_decoder = float(lr_grid), float(lr_decoder)
        rows = max_active_nodes or tree.NumActiveNodes()
        gen = torch.Generator().manual_seed(seed)
        dev = torch.device(device)
        self.grid_data = grid_init(rows, self.C, self.G, gen, grid_init_mode).to(dev).requires_grad_(True)
        self.decoder = decoder_init(self.C, gen).to(dev).requires_grad_(True)
        self._adam = {}
        self.step_count = 0

    def ComputeImage(self, all_samples: SampleList, num_channels: int, num_pixels: int):
        if num_channels != 1:
            raise ValueError("ComputeImage: the X-ray decoder has one output channel")
        local_id = self.tree.GlobalNodeIdToLocalActiveId(all_samples.node_id).contiguous()
        samples_t = (all_samples.global_coordinate.contiguous(), all_samples.weight.contiguous(),
                     all_samples.ray_index.contiguous(), all_samples.node_id.contiguous(), local_id)
        return _ComputeImageFn.apply(self.grid_data, self.decoder, self, samples_t, int(num_pixels))

    def parameters(self):
        return [self.grid_data, self.decoder]

    def zero_grad(self):
        for p in self.parameters():
            if p.grad is not None:
                p.grad.zero_()

    def OptimizerStep(self, epoch_id=0):
        """torch::optim::Adam step on both groups, then zero_grad."""
        self.step_count += 1
        lib = _lib.load()
        for p, lr in ((self.grid_data, self.lr_grid), (self.decoder, self.lr_decoder)):
            if p.grad is None:
                continue
            if id(p) not in self._adam:
                self._adam[id(p)] = (torch.zeros_like(p), torch.zeros_like(p))
            m, v = self._adam[id(p)]
            with torch.no_grad():
                _lib.check(lib.neat_adam(p.data_ptr(), p.grad.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), lr,
                                         0.9, 0.999, 1e-8, self.step_count, 1, _stream(p)), "neat_adam")
