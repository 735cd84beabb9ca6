"""CPU execution of the reference's training step -- baseline only.

TEST AND CPU-BASELINE INFRASTRUCTURE: used by bench.py's cpu_baseline leg and its
--impl reference arm, never by the product.

The reference (darglein/NeAT) has no CPU training path for the whole step:
ComputeRaySamples is CUDA-only (src/structure/HyperTree.cu:206-438).  The CPU
arm therefore runs, with all host threads:
  * GetRays + CreateSamplesForRays: the oracle's OpenMP C restatement;
  * IndirectGridSample3D forward/backward: the reference's own CPU code
    (src/modules/IndirectGridSample3D.cu:27-429) compiled from its source into
    oracle/_ref (make -C oracle ref); the oracle's bit-identical restatement
    when that library is absent;
  * FCBlock, softplus(beta=2), index_add_, MSE, autograd, torch.optim.Adam:
    libtorch CPU, as the reference's geometry code calls them
    (src/geometry/geometry.cpp:102-163, :393-424, samples/reconstruct.cpp:378-396,
    src/geometry/geometry.h:66-88).
"""
import ctypes
import os

import numpy as np
import torch

from oracle import oracle as O

_REF_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libneat_ref.so")
_ref = None


def reference_igs():
    """The reference's compiled CPU IGS (None when oracle/_ref is not built)."""
    global _ref
    if _ref is None and os.path.exists(_REF_SO):
        lib = ctypes.CDLL(_REF_SO)
        P, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
        lib.ref_igs_forward.argtypes = [P, L, I, I, I, I, P, P, L, P]
        lib.ref_igs_backward.argtypes = [P, L, I, I, I, I, P, P, L, P, P, P]
        _ref = lib
    return _ref


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def igs_forward(grid, index, uv):
    ref = reference_igs()
    if ref is None:
        return O.igs_forward(grid, index, uv)
    N, C, Z, Y, X = grid.shape
    out = np.zeros((index.shape[0], C), np.float32)
    ref.ref_igs_forward(_p(grid), N, C, Z, Y, X, _p(index), _p(uv), index.shape[0], _p(out))
    return out


def igs_backward(grid, index, uv, grad_out):
    ref = reference_igs()
    if ref is None:
        return O.igs_backward(grid, index, uv, grad_out)[0]
    N, C, Z, Y, X = grid.shape
    gg = np.zeros_like(grid)
    gu = np.zeros((index.shape[0], 3), np.float32)
    ref.ref_igs_backward(_p(grid), N, C, Z, Y, X, _p(index), _p(uv), index.shape[0], _p(grad_out), _p(gg), _p(gu))
    return gg


class _IGS(torch.autograd.Function):
    @staticmethod
    def forward(ctx, grid, index, uv):
        g = np.ascontiguousarray(grid.detach().numpy())
        i = np.ascontiguousarray(index.numpy())
        u = np.ascontiguousarray(uv.numpy())
        ctx.save_for_backward(grid, index, uv)
        return torch.from_numpy(igs_forward(g, i, u))

    @staticmethod
    def backward(ctx, go):
        grid, index, uv = ctx.saved_tensors
        gg = igs_backward(np.ascontiguousarray(grid.detach().numpy()), np.ascontiguousarray(index.numpy()),
                          np.ascontiguousarray(uv.numpy()), np.ascontiguousarray(go.numpy()))
        return torch.from_numpy(gg), None, None


def _decoder(C, gen):
    seq = torch.nn.Sequential(torch.nn.Linear(C, 64), torch.nn.SiLU(), torch.nn.Linear(64, 64), torch.nn.SiLU(),
                              torch.nn.Linear(64, 1))
    with torch.no_grad():
        for m in seq:
            if isinstance(m, torch.nn.Linear):
                torch.nn.init.kaiming_normal_(m.weight, 0, "fan_in", "relu", generator=gen)
    return seq


class CpuReferenceStep:
    def __init__(self, objects, tree, cfg, seed=0):
        from neat_b200 import scene as SC
        self.objects = np.ascontiguousarray(objects, np.float64)
        self.tree = tree
        self.cfg = cfg
        self.w, self.h, self.n_img = cfg["w"], cfg["h"], cfg["n_angles"]
        self.intr, self.rot, self.trans = SC.cone_beam_geometry(self.n_img, self.w, self.h)
        A = tree.NumActiveNodes()
        C, G = cfg["C"], cfg["G"]
        gen = torch.Generator().manual_seed(seed)
        self.grid = torch.nn.Parameter(torch.rand((A, C, G, G, G), generator=gen) * 2 - 1)
        self.dec = _decoder(C, gen)
        self.opt = torch.optim.Adam([{"params": [self.grid], "lr": 1e-2},
                                     {"params": list(self.dec.parameters()), "lr": 5e-5}])
        self.rng = np.random.default_rng(seed + 1)
        self.last_samples = 0

    def batch(self, R):
        img = self.rng.integers(0, self.n_img, R).astype(np.int32)
        x = self.rng.integers(0, self.w, R).astype(np.int32)
        y = self.rng.integers(0, self.h, R).astype(np.int32)
        uv = np.stack([x.astype(np.float32) / np.float32(self.w - 1), y.astype(np.float32) / np.float32(self.h - 1)],
                      1)
        target = O.project_pixels(self.objects, img, x, y, self.intr, self.rot, self.trans)
        ph = self.cfg.get("photons")
        if ph:
            counts = np.maximum(self.rng.poisson(ph * np.exp(-target.astype(np.float64))), 1)
            target = (-np.log(counts / ph)).astype(np.float32)
        return uv, img, target

    def run(self, uv, img, target, step):
        T = self.tree
        o, d = O.make_rays(uv, img, self.w, self.h, self.intr, self.rot, self.trans)
        s = O.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, self.cfg["M"], True,
                             seed=7, step=step)
        self.last_samples = s["ray_t"].shape[0]
        local = O.local_samples(s["coords"], s["node_id"], T.node_position_min, T.node_position_max)
        row = torch.from_numpy(T.node_active_prefix_sum[s["node_id"]])
        feat = _IGS.apply(self.grid, row, torch.from_numpy(local))
        dens = torch.nn.functional.softplus(self.dec(feat), beta=2.0)[:, 0]
        val = dens * torch.from_numpy(s["weight"])
        pred = torch.zeros(uv.shape[0]).index_add(0, torch.from_numpy(s["ray_index"]), val)
        loss = ((pred - torch.from_numpy(target)) ** 2).mean()
        self.opt.zero_grad()
        loss.backward()
        self.opt.step()
        return float(loss.detach())

    def step(self, R, step):
        uv, img, target = self.batch(R)
        return self.run(uv, img, target, step + 1)
