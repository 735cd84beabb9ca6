"""Seeded test cases shared by the CPU and GPU tests (small configurations
the oracle finishes in seconds)."""
import numpy as np
import torch

from neat_b200 import scene as SC
from neat_b200.api import decoder_init, grid_init
from neat_b200.tree import HyperTreeBase


class Case:
    pass


def cfg1_case(R=4096, seed=0, n_angles=32, w=128, h=128, depth=2, C=4, G=11, M=16, oracle=None, adaptive=None):
    """Config-1 shapes: 8 ellipsoids, 32 angles of 128^2, depth-2 octree
    (64 leaves), C=4, G=11, M=16, R=4096 rays."""
    c = Case()
    c.R, c.C, c.G, c.M, c.w, c.h, c.n_img = R, C, G, M, w, h, n_angles
    c.objects = SC.ellipsoid_phantom(8, 0, seed=seed + 1)
    c.intr, c.rot, c.trans = SC.cone_beam_geometry(n_angles, w, h)
    c.tree = HyperTreeBase(3, depth)
    if adaptive:
        c.tree.RefineByVariance(lambda p: oracle.phantom_density(c.objects, p), adaptive, samples_per_axis=3)
    else:
        c.tree.SetActive(depth)
    c.A = c.tree.NumActiveNodes()
    rng = np.random.default_rng(seed)
    c.img = rng.integers(0, n_angles, R).astype(np.int32)
    c.x = rng.integers(0, w, R)
    c.y = rng.integers(0, h, R)
    c.uv = np.stack([c.x.astype(np.float32) / np.float32(w - 1), c.y.astype(np.float32) / np.float32(h - 1)], 1)
    if oracle is not None:
        c.proj = oracle.project(c.objects, n_angles, w, h, c.intr, c.rot, c.trans)
        c.target = c.proj[c.img, c.y, c.x].astype(np.float32)
    gen = torch.Generator().manual_seed(seed + 7)
    c.grid = grid_init(c.A, C, G, gen).numpy()
    c.dec = decoder_init(C, gen).numpy()
    return c


def workload_case(name, R=4096, seed=0):
    """A slice of a measured workload (neat_b200.workloads): the very scene,
    scan geometry and octree the benchmark trains on, R rays drawn from its
    projections by the benchmark's batch sampler, and a seeded initial grid
    and decoder of the workload's sizes.  Needs CUDA (the device projector
    makes the scans)."""
    from neat_b200.workloads import WORKLOADS, build_workload
    cfg = WORKLOADS[name]
    scene, tree, cam = build_workload(cfg, "cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    uv, img, tgt = scene.sample_batch(R, gen)
    c = Case()
    c.name, c.cfg, c.scene = name, cfg, scene
    c.R, c.C, c.G, c.M = R, cfg["C"], cfg["G"], cfg["M"]
    c.w, c.h, c.n_img = scene.w, scene.h, scene.n_img
    c.objects = scene.objects
    c.intr, c.rot, c.trans = scene.intrinsics, scene.rotation, scene.translation
    c.tree = tree
    c.A = tree.NumActiveNodes()
    c.uv = uv.cpu().numpy()
    c.img = img.cpu().numpy()
    c.target = tgt.cpu().numpy()
    g = torch.Generator().manual_seed(seed + 7)
    c.grid = grid_init(c.A, c.C, c.G, g).numpy()
    c.dec = decoder_init(c.C, g).numpy()
    return c
