"""The reference-API entry points a maintainer binds one by one (besides the
fused step): ComputeLocalSamples, the optimizer step, and the batch sampler's
semantics.

Bars: bit-exact for the local coordinates (float32 arithmetic written as the
reference writes it) and for the batch's pixel coordinates and targets;
parameters after Adam within float32 rounding (half an ulp per step) plus
1e-6 of each step's update of float64 torch.optim.Adam.
"""
import numpy as np
import pytest
import torch

from tests.cases import cfg1_case

pytestmark = pytest.mark.gpu


def _rel2(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("boxes", ["tree", "arbitrary"])
def test_compute_local_samples_bit_exact(neat, oracle, boxes):
    """HyperTreeBaseImpl::ComputeLocalSamples (src/structure/HyperTree.cu:177-192):
    (g - min[node]) / (max[node] - min[node]) * 2 - 1 in float32, against the
    oracle and against the reference's own torch expression evaluated on the
    CPU.  Dyadic tree boxes (the power-of-two scale fast path) and arbitrary
    boxes (true division)."""
    from neat_b200.api import ComputeLocalSamples
    from neat_b200.tree import HyperTreeBase
    rng = np.random.default_rng(3)
    T = HyperTreeBase(3, 3)
    T.SetActive(3)
    if boxes == "arbitrary":
        lo = rng.uniform(-1, 0.5, (T.NumNodes(), 3)).astype(np.float32)
        T.node_position_min = lo
        T.node_position_max = (lo + rng.uniform(1e-3, 0.7, lo.shape)).astype(np.float32)
    S = 50000
    nid = rng.choice(T.active_node_ids, S)
    mn, mx = T.node_position_min[nid], T.node_position_max[nid]
    g = (mn + rng.uniform(-0.05, 1.05, (S, 3)) * (mx - mn)).astype(np.float32)
    g[:4] = mn[:4]  # on the min faces
    g[4:8] = mx[4:8]  # on the max faces
    if boxes == "tree":  # the reference-facing wrapper (device tables of the octree)
        out = ComputeLocalSamples(T, torch.from_numpy(g).cuda(), torch.from_numpy(nid).cuda()).cpu().numpy()
    else:  # any boxes: the C ABI takes just the node min/max tables
        gd, nd = torch.from_numpy(g).cuda(), torch.from_numpy(nid).cuda()
        mn_d, mx_d = torch.from_numpy(T.node_position_min).cuda(), torch.from_numpy(T.node_position_max).cuda()
        od = torch.empty_like(gd)
        assert neat.neat_local_samples(gd.data_ptr(), nd.data_ptr(), S, mn_d.data_ptr(), mx_d.data_ptr(),
                                       od.data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
        out = od.cpu().numpy()
    np.testing.assert_array_equal(out, oracle.local_samples(g, nid, T.node_position_min, T.node_position_max))
    tg = torch.from_numpy(g)
    tmin = torch.from_numpy(T.node_position_min).index_select(0, torch.from_numpy(nid))
    tmax = torch.from_numpy(T.node_position_max).index_select(0, torch.from_numpy(nid))
    np.testing.assert_array_equal(out, ((tg - tmin) / (tmax - tmin) * 2 - 1).numpy())
    if boxes == "tree":
        assert ComputeLocalSamples(T, torch.zeros((0, 3), device="cuda"),
                                   torch.zeros(0, dtype=torch.int64, device="cuda")).shape == (0, 3)


def test_optimizer_step_matches_torch_adam(neat):
    """GeometryExEx.OptimizerStep (NeuralGeometry::OptimizerStep,
    src/geometry/geometry.h:66-88): Adam on the grid group (lr_grid) and the
    decoder group (lr_decoder) followed by zero_grad, over three steps with
    fresh gradients, against torch.optim.Adam in float64."""
    from neat_b200.api import GeometryExEx
    from neat_b200.tree import HyperTreeBase
    T = HyperTreeBase(3, 2)
    T.SetActive(2)
    geom = GeometryExEx(T, num_features=4, grid_size=9, lr_grid=1e-2, lr_decoder=5e-5, seed=4)
    ref = [p.detach().cpu().double().clone().requires_grad_(True) for p in geom.parameters()]
    opt = torch.optim.Adam([{"params": [ref[0]], "lr": 1e-2}, {"params": [ref[1]], "lr": 5e-5}],
                           betas=(0.9, 0.999), eps=1e-8)
    p0 = [p.detach().cpu().double().clone() for p in geom.parameters()]
    # per element and step: one float32 rounding of the parameter (half an ulp
    # of its magnitude after the step) plus 1e-6 of the step's update (the
    # float32 moments, square root and division); summed over the steps
    bound = [torch.zeros_like(q) for q in p0]
    prev = [q.clone() for q in p0]
    rng = np.random.default_rng(9)
    for _ in range(3):
        grads = [rng.normal(0, 1, tuple(p.shape)).astype(np.float32) for p in geom.parameters()]
        grads[0][0] = 0.0  # a zero-gradient row still moves with its moments, as in torch
        for p, g, r in zip(geom.parameters(), grads, ref):
            p.grad = torch.from_numpy(g).cuda()
            r.grad = torch.from_numpy(g).double()
        geom.OptimizerStep()
        opt.step()
        torch.cuda.synchronize()
        for p in geom.parameters():
            assert float(p.grad.abs().max()) == 0.0  # zero_grad after the step
        for k, r in enumerate(ref):
            now = r.detach().clone()
            half_ulp = 0.5 * np.spacing(np.abs(now.numpy()).astype(np.float32)).astype(np.float64)
            bound[k] += torch.from_numpy(half_ulp) + 1e-6 * (now - prev[k]).abs()
            prev[k] = now
    for p, r, q0, b in zip(geom.parameters(), ref, p0, bound):
        got, want = p.detach().cpu().double(), r.detach()
        diff = (got - want).abs()
        print("Adam: max |p - p64|", float(diff.max()), "max ratio to bound", float((diff / (b + 1e-30)).max()))
        assert bool((diff <= b).all())
        assert _rel2((got - q0).numpy(), (want - q0).numpy()) < 1e-3


def test_sample_batch_semantics(neat):
    """RandomMultiSceneDataset::get_batch (src/data/Dataloader.cpp:8-49) with
    CoordinatesRandomNoInterpolate and SampleProjection (src/data/SceneBase.cpp:
    32-39, 59-76): a uniform image (from the training split when one is given),
    a uniform integer pixel, uv = (x / (w - 1), y / (h - 1)) in float32 and the
    target = that pixel's value."""
    from neat_b200 import scene as SC
    objs = SC.ellipsoid_phantom(4, 0, seed=2)
    sc = SC.SyntheticScene(objs, 12, 40, 30)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    split = [1, 4, 5, 9]
    R = 200000
    uv, img, tgt = sc.sample_batch(R, gen, images=split)
    uv, img, tgt = uv.cpu().numpy(), img.cpu().numpy(), tgt.cpu().numpy()
    assert uv.dtype == np.float32 and img.dtype == np.int32 and tgt.dtype == np.float32
    x = np.rint(uv[:, 0] * (sc.w - 1)).astype(np.int64)
    y = np.rint(uv[:, 1] * (sc.h - 1)).astype(np.int64)
    assert x.min() == 0 and x.max() == sc.w - 1 and y.min() == 0 and y.max() == sc.h - 1
    np.testing.assert_array_equal(uv[:, 0], x.astype(np.float32) / np.float32(sc.w - 1))
    np.testing.assert_array_equal(uv[:, 1], y.astype(np.float32) / np.float32(sc.h - 1))
    proj = sc.projection.cpu().numpy()
    np.testing.assert_array_equal(tgt, proj[img, y, x])
    assert set(np.unique(img).tolist()) == set(split)
    # uniform over the split's images and the pixel columns (loose chi-square bounds)
    for counts in (np.bincount(img, minlength=12)[split], np.bincount(x, minlength=sc.w)):
        e = counts.sum() / len(counts)
        chi2 = float(((counts - e) ** 2 / e).sum())
        assert chi2 < 3 * len(counts) + 30
    # without a split every image can be drawn
    _, img_all, _ = sc.sample_batch(20000, gen)
    assert np.unique(img_all.cpu().numpy()).size == 12
