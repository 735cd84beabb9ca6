"""The libtorch shim (neat_b200/shim/neat_torch.{h,cpp}, libneat_torch.so):
the reference's C++ module API -- IndirectGridSample3D as a
torch::autograd::Function, GetRays, HyperTree::CreateSamplesForRays /
ComputeLocalSamples, ComputeImage with autograd, the Adam optimizer step --
compiled against libtorch and driven through its registered torch operators.

Bars as for the C ABI underneath: bit-exact for rays, SampleLists, local
coordinates, the IGS forward and grad_uv (the reference's own CPU IGS golden);
grad_grid to float-add order (1e-6); ComputeImage projection and gradients
1e-5 of the f64 oracle; Adam within float32 rounding of f64 torch.optim.Adam.
"""
import os

import numpy as np
import pytest
import torch

from tests.cases import cfg1_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops(neat):
    from neat_b200 import _lib
    return _lib.load_torch_ops()


@pytest.fixture(scope="module")
def case(oracle):
    return cfg1_case(R=2048, seed=3, depth=4, G=9, M=16, oracle=oracle, adaptive=400)


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def _rel2(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def _tree(c):
    T = c.tree
    return _dev(T.node_position_min), _dev(T.node_position_max), _dev(T.active_node_ids), T.max_depth


def test_shim_igs_matches_reference_cpu_golden(ops):
    """IndirectGridSample3D through the C++ autograd Function against the
    reference's own CPU IGS (golden fixture)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "igs_reference_cpu.npz"))
    g = _dev(z["grid"]).requires_grad_(True)
    p = _dev(z["uv"]).requires_grad_(True)
    out = ops.IndirectGridSample3D(g, _dev(z["index"]), p)
    np.testing.assert_array_equal(out.detach().cpu().numpy(), z["out"])
    out.backward(_dev(z["grad_out"]))
    np.testing.assert_array_equal(p.grad.cpu().numpy(), z["grad_uv"])
    np.testing.assert_allclose(g.grad.cpu().numpy(), z["grad_grid"], rtol=0, atol=1e-6)
    with pytest.raises(RuntimeError, match="multi_grid"):
        ops.IndirectGridSample3D(g.detach()[0], _dev(z["index"]), p.detach())


def test_shim_rays_samples_and_local_coordinates(ops, oracle, case):
    """GetRays, CreateSamplesForRays (with jitter) and ComputeLocalSamples of
    the C++ API, bit for bit against the oracle on an adaptive depth-4 tree."""
    c = case
    o, d = ops.GetRays(c.w, c.h, _dev(c.intr), _dev(c.rot), _dev(c.trans), _dev(c.uv), _dev(c.img), None)
    oo, dd = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    np.testing.assert_array_equal(o.cpu().numpy(), oo)
    np.testing.assert_array_equal(d.cpu().numpy(), dd)
    nmin, nmax, act, depth = _tree(c)
    coords, ray_t, weight, ray_index, local, node_id, mx = ops.CreateSamplesForRays(nmin, nmax, act, depth, 11, 3, o, d,
                                                                                     c.M, True)
    T = c.tree
    ref = oracle.create_samples(oo, dd, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                seed=11, step=3)
    for got, key in ((coords, "coords"), (ray_t, "ray_t"), (weight, "weight"), (ray_index, "ray_index"),
                     (local, "local_index"), (node_id, "node_id")):
        np.testing.assert_array_equal(got.cpu().numpy(), ref[key], err_msg=key)
    assert mx == ref["max_per_ray"]
    lc = ops.ComputeLocalSamples(nmin, nmax, act, depth, coords, node_id)
    np.testing.assert_array_equal(lc.cpu().numpy(), oracle.local_samples(ref["coords"], ref["node_id"],
                                                                         T.node_position_min, T.node_position_max))


def test_shim_compute_image_autograd_matches_f64(ops, oracle, case):
    """ComputeImage through the C++ autograd Function: projection, MSE loss and
    the grid and decoder gradients of loss.backward() against the f64 oracle."""
    c = case
    T = c.tree
    oo, dd = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    s = oracle.create_samples(oo, dd, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                              seed=5, step=1)
    nmin, nmax, act, depth = _tree(c)
    grid = _dev(c.grid).requires_grad_(True)
    dec = _dev(c.dec).requires_grad_(True)
    img = ops.ComputeImage(nmin, nmax, act, depth, _dev(s["coords"]), _dev(s["weight"]), _dev(s["ray_index"]),
                           _dev(s["node_id"]), grid, dec, 1, c.R, 2.0)
    assert tuple(img.shape) == (1, c.R)
    loss = ((img[0] - _dev(c.target)) ** 2).mean()
    loss.backward()
    ref = oracle.step_f64(s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                          T.node_active_prefix_sum)
    assert _rel2(img[0].detach().cpu().numpy(), ref["pred"]) < 1e-5
    assert abs(float(loss.detach()) - ref["loss"]) < 1e-5 * ref["loss"]
    assert _rel2(grid.grad.cpu().numpy(), ref["grad_grid"]) < 1e-5
    assert _rel2(dec.grad.cpu().numpy(), ref["grad_dec"]) < 1e-5


def test_shim_adam_matches_torch_adam(ops):
    """neat_torch::Adam (two groups, lr 1e-2 and 5e-5, three steps with fresh
    gradients, zero_grad after each) against torch.optim.Adam in float64:
    per element within one float32 rounding of the parameter per step plus
    1e-6 of each step's update."""
    rng = np.random.default_rng(2)
    shapes = [(64, 4, 9, 9, 9), (4673,)]
    p0 = [rng.uniform(-1, 1, s).astype(np.float32) for s in shapes]
    grads = [[rng.normal(0, 1, s).astype(np.float32) for s in shapes] for _ in range(3)]
    params = [_dev(p.copy()) for p in p0]
    ops.AdamSteps(params, [_dev(g) for step in grads for g in step], [0, 1], [1e-2, 5e-5], 3, 0.9, 0.999, 1e-8)
    torch.cuda.synchronize()
    ref = [torch.from_numpy(p.astype(np.float64)).requires_grad_(True) for p in p0]
    opt = torch.optim.Adam([{"params": [ref[0]], "lr": 1e-2}, {"params": [ref[1]], "lr": 5e-5}], betas=(0.9, 0.999),
                           eps=1e-8)
    bound = [np.zeros(s) for s in shapes]
    prev = [p.astype(np.float64) for p in p0]
    for step in grads:
        for r, g in zip(ref, step):
            r.grad = torch.from_numpy(g.astype(np.float64))
        opt.step()
        for k, r in enumerate(ref):
            now = r.detach().numpy().copy()
            bound[k] += 0.5 * np.spacing(np.abs(now).astype(np.float32)).astype(np.float64) + 1e-6 * np.abs(now - prev[k])
            prev[k] = now
    for p, r, b in zip(params, ref, bound):
        diff = np.abs(p.cpu().numpy().astype(np.float64) - r.detach().numpy())
        assert np.all(diff <= b), float((diff / (b + 1e-30)).max())
        assert float(p.grad.abs().max()) == 0.0  # zero_grad after each step
