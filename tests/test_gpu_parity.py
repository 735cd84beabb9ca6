"""GPU parity: every CUDA entry point against the oracle on the same inputs.

Bars: bit-exact for rays, hit lists, sample counts, sample positions/weights,
node indexing (the decisions are integer/ordering work) and for the IGS
forward and grad_uv (same fma order); FP32 tolerances stated per test for
everything that sums in a different order than the f64 oracle:
  projection / loss:  1e-5 relative (the FP32 bar)
  gradients:          1e-5 relative in the 2-norm (||g - g64|| / ||g64||);
                      elementwise checks would flag cancellation noise.
"""
import ctypes

import numpy as np
import pytest
import torch

from tests.cases import cfg1_case

pytestmark = pytest.mark.gpu


def _dev(a, dt=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dt is not None:
        t = t.to(dt)
    return t.cuda()


def _rel2(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.fixture(scope="module")
def case(oracle):
    return cfg1_case(R=4096, oracle=oracle)


@pytest.fixture(scope="module")
def adaptive_case(oracle):
    # depth-4 tree refined by density variance (mixed node sizes)
    return cfg1_case(R=2048, seed=3, depth=4, G=9, M=16, oracle=oracle, adaptive=400)


@pytest.fixture(scope="module")
def c8_case(oracle):
    # C=8, G=17 grids (the full-size model) on a depth-3 refined tree
    return cfg1_case(R=2048, seed=5, depth=3, C=8, G=17, M=32, oracle=oracle, adaptive=200)


@pytest.fixture(scope="module")
def c8_long_case(oracle):
    # 16 k rays of the C=8 model: ~3.3 k tiles, ~22 per CTA of the backward's
    # one-CTA-per-SM grid (long tile loops in every kernel)
    return cfg1_case(R=16384, seed=7, depth=3, C=8, G=17, M=32, oracle=oracle, adaptive=200)


def _camera(c):
    from neat_b200.api import CameraModel
    return CameraModel(c.w, c.h, c.intr, c.rot, c.trans)


# ---------------------------------------------------------------- rays
def test_make_rays_bit_exact(neat, oracle, case):
    from neat_b200.api import GetRays
    rays = GetRays(_camera(case), _dev(case.uv), _dev(case.img))
    o, d = oracle.make_rays(case.uv, case.img, case.w, case.h, case.intr, case.rot, case.trans)
    np.testing.assert_array_equal(rays.origin.cpu().numpy(), o)
    np.testing.assert_array_equal(rays.direction.cpu().numpy(), d)


# ---------------------------------------------------------------- samples
@pytest.mark.parametrize("which", ["cfg1", "adaptive"])
@pytest.mark.parametrize("jitter", [False, True])
def test_create_samples_bit_exact(neat, oracle, case, adaptive_case, which, jitter):
    from neat_b200.api import CreateSamplesForRays, GetRays
    c = case if which == "cfg1" else adaptive_case
    rays = GetRays(_camera(c), _dev(c.uv), _dev(c.img))
    s = CreateSamplesForRays(c.tree, rays, c.M, jitter, seed=11, step=3)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    ref = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, jitter,
                                seed=11, step=3)
    assert s.size() == ref["ray_t"].shape[0] > 0
    np.testing.assert_array_equal(s.ray_index.cpu().numpy(), ref["ray_index"])
    np.testing.assert_array_equal(s.node_id.cpu().numpy(), ref["node_id"])
    np.testing.assert_array_equal(s.local_index_in_ray.cpu().numpy(), ref["local_index"])
    np.testing.assert_array_equal(s.ray_t.cpu().numpy(), ref["ray_t"])
    np.testing.assert_array_equal(s.weight.cpu().numpy(), ref["weight"])
    np.testing.assert_array_equal(s.global_coordinate.cpu().numpy(), ref["coords"])
    assert s.max_samples_per_ray == ref["max_per_ray"]


def test_create_samples_edge_cases(neat, oracle, case):
    from neat_b200.api import CreateSamplesForRays, RayList
    T = case.tree
    # rays that miss the volume, an axis-parallel ray on a node face, a ray
    # starting inside the volume, an empty batch
    o = np.array([[5, 5, 5], [-3, 0.0, 0.0], [0.1, 0.2, 0.3], [-3, 0.5, -0.5]], np.float32)
    d = np.array([[1, 0, 0], [1, 0, 0], [0, 0, 1], [1, 0, 0]], np.float32)
    s = CreateSamplesForRays(T, RayList(_dev(o), _dev(d)), case.M, False)
    ref = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, case.M, False)
    np.testing.assert_array_equal(s.ray_t.cpu().numpy(), ref["ray_t"])
    np.testing.assert_array_equal(s.node_id.cpu().numpy(), ref["node_id"])
    assert not np.any(s.ray_index.cpu().numpy() == 0)  # the first ray misses
    empty = CreateSamplesForRays(T, RayList(_dev(np.zeros((0, 3), np.float32)), _dev(np.zeros((0, 3), np.float32))),
                                 case.M, True)
    assert empty.size() == 0


def test_create_samples_capacity_status(neat, case):
    from neat_b200 import _lib
    from neat_b200.api import GetRays
    rays = GetRays(_camera(case), _dev(case.uv), _dev(case.img))
    t = case.tree.device_tables("cuda")
    R = rays.size()
    ws = torch.empty(neat.neat_samples_workspace_bytes(R), dtype=torch.uint8, device="cuda")
    cap = 10
    bufs = [torch.empty((cap, 3), device="cuda"), torch.empty(cap, device="cuda"), torch.empty(cap, device="cuda")] + \
           [torch.empty(cap, dtype=torch.int64, device="cuda") for _ in range(3)]
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = neat.neat_create_samples(t["table"].data_ptr(), case.A, case.tree.max_depth, rays.origin.data_ptr(),
                                  rays.direction.data_ptr(), R, case.M, 0, 0, 1, cap, *[b.data_ptr() for b in bufs],
                                  cnt.data_ptr(), st.data_ptr(), ws.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(st.item()) & _lib.NEAT_ERR_CAPACITY
    assert int(cnt[0]) > cap


def test_non_dyadic_tree_rejected(neat):
    from neat_b200 import _lib
    from neat_b200.tree import HyperTreeBase
    T = HyperTreeBase(3, 2)
    T.SetActive(2)
    T.node_position_max = T.node_position_max.copy()
    T.node_position_max[T.active_node_ids[0], 0] += np.float32(0.01)
    with pytest.raises(_lib.NeatError) as e:
        T.device_tables("cuda")
    assert e.value.status & _lib.NEAT_ERR_NON_DYADIC


def test_bad_input_is_reported(neat):
    from neat_b200 import _lib
    assert neat.neat_make_rays(None, None, None, 5, 1, 1, None, None, None, None, None, None) == \
        _lib.NEAT_ERR_BAD_INPUT
    assert neat.neat_igs_forward(None, 1, 1, 1, 1, 1, None, None, 3, None, None) == _lib.NEAT_ERR_BAD_INPUT


# ---------------------------------------------------------------- IGS
def test_igs_forward_backward(neat, oracle):
    from neat_b200.api import IndirectGridSample3D
    rng = np.random.default_rng(4)
    grid = rng.uniform(-1, 1, (7, 5, 11, 9, 13)).astype(np.float32)
    S = 20000
    idx = rng.integers(0, 7, S)
    uv = rng.uniform(-1.05, 1.05, (S, 3)).astype(np.float32)
    uv[:6] = [[-1, -1, -1], [1, 1, 1], [1, -1, 1], [0, 0, 0], [-1, 1, -1], [1, 1, -1]]
    go = rng.normal(size=(S, 5)).astype(np.float32)
    g = _dev(grid).requires_grad_(True)
    p = _dev(uv).requires_grad_(True)
    out = IndirectGridSample3D(g, _dev(idx), p)
    np.testing.assert_array_equal(out.detach().cpu().numpy(), oracle.igs_forward(grid, idx, uv))
    out.backward(_dev(go))
    gg, gu = oracle.igs_backward(grid, idx, uv, go)
    np.testing.assert_array_equal(p.grad.cpu().numpy(), gu)
    assert _rel2(g.grad.cpu().numpy(), gg) < 1e-6
    # empty batch
    e = IndirectGridSample3D(g.detach(), _dev(np.zeros(0, np.int64)), _dev(np.zeros((0, 3), np.float32)))
    assert e.shape == (0, 5)


def test_igs_matches_reference_cpu_golden(neat):
    """The CUDA IGS against the reference's own CPU IGS (golden fixture):
    forward and grad_uv bit-exact, grad_grid to summation order."""
    import os
    from neat_b200.api import IndirectGridSample3D
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "igs_reference_cpu.npz"))
    g = _dev(z["grid"]).requires_grad_(True)
    p = _dev(z["uv"]).requires_grad_(True)
    out = IndirectGridSample3D(g, _dev(z["index"]), p)
    np.testing.assert_array_equal(out.detach().cpu().numpy(), z["out"])
    out.backward(_dev(z["grad_out"]))
    np.testing.assert_array_equal(p.grad.cpu().numpy(), z["grad_uv"])
    np.testing.assert_allclose(g.grad.cpu().numpy(), z["grad_grid"], rtol=0, atol=1e-6)


# ---------------------------------------------------------------- ComputeImage
def test_compute_image_forward_backward(neat, oracle, case):
    from neat_b200.api import CreateSamplesForRays, GeometryExEx, GetRays
    c = case
    rays = GetRays(_camera(c), _dev(c.uv), _dev(c.img))
    s = CreateSamplesForRays(c.tree, rays, c.M, True, seed=5, step=1)
    geom = GeometryExEx(c.tree, c.C, c.G)
    with torch.no_grad():
        geom.grid_data.copy_(_dev(c.grid))
        geom.decoder.copy_(_dev(c.dec))
    img = geom.ComputeImage(s, 1, c.R)
    loss = ((img[0] - _dev(c.target)) ** 2).mean()
    loss.backward()
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True, seed=5,
                                  step=1)
    ref = oracle.step_f64(ref_s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                          T.node_active_prefix_sum)
    pred = img[0].detach().cpu().numpy()
    assert _rel2(pred, ref["pred"]) < 1e-5
    assert abs(float(loss.detach()) - ref["loss"]) < 1e-5 * ref["loss"]
    assert _rel2(geom.grid_data.grad.cpu().numpy(), ref["grad_grid"]) < 1e-5
    assert _rel2(geom.decoder.grad.cpu().numpy(), ref["grad_dec"]) < 1e-5


# ---------------------------------------------------------------- fused step
# decoder paths and their tolerances against the f64 oracle:
#   simt / bf16x3: the FP32 bar (1e-5 relative); Adam-updated parameters 1e-6
#   bf16: BF16 operands with FP32 accumulation -- stated bound 1e-2 on the
#   projection, 5e-2 on gradients (2-norm relative)
PATHS = {"simt": (0, 1e-5, 1e-5, 1e-6), "bf16x3": (1, 1e-5, 1e-5, 1e-6), "bf16": (2, 1e-2, 5e-2, 5e-3)}


def _trainer(c, path="bf16x3", **kw):
    from neat_b200.trainer import FusedTrainer
    return FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                        grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec),
                        decoder_path=PATHS[path][0], **kw)


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("which", ["cfg1", "adaptive", "c8"])
def test_fused_step_matches_f64(neat, oracle, case, adaptive_case, c8_case, which, path):
    c = {"cfg1": case, "adaptive": adaptive_case, "c8": c8_case}[which]
    _check_fused_step(oracle, c, which, path)


@pytest.mark.parametrize("path", ["bf16", "bf16x3"])
@pytest.mark.parametrize("records", [-1, 1])
@pytest.mark.parametrize("which", ["cfg1", "c8"])
def test_fused_step_recomputes_without_records(neat, oracle, case, c8_case, which, records, path):
    """The backward recomputes placement and gather when the forward kept no
    records (-1) or the step has more samples than their room (1 per ray)."""
    c = {"cfg1": case, "c8": c8_case}[which]
    _check_fused_step(oracle, c, which, path, record_samples_per_ray=records)


@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
def test_fused_step_long_tile_loops(neat, oracle, c8_long_case, path):
    """~22 tiles per CTA: the pipelined tile loops (records, deferred dX and
    scatter, weight gradients under the next tile) over many iterations."""
    _check_fused_step(oracle, c8_long_case, "c8_long", path)


def _oracle_step(oracle, c):
    """The oracle's samples, segments and f64 step for the case's batch (seed
    99, step 1: what _trainer's first step draws), computed once per case."""
    if getattr(c, "_oracle_step", None) is None:
        o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
        T = c.tree
        ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                      seed=99, step=1)
        seg = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M)
        ref = oracle.step_f64(ref_s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                              T.node_active_prefix_sum, lr_grid=1e-2, lr_decoder=5e-5, step=1)
        c._oracle_step = (ref_s, seg, ref)
    return c._oracle_step


def _check_fused_step(oracle, c, which, path, **kw):
    _, tol_p, tol_g, tol_w = PATHS[path]
    tr = _trainer(c, path, **kw)
    pred = torch.zeros(c.R, device="cuda")
    loss = tr.step(_dev(c.uv), _dev(c.img), _dev(c.target), prediction=pred)
    torch.cuda.synchronize()
    tr.check_status()
    ref_s, seg, ref = _oracle_step(oracle, c)
    cnt = tr.counters.cpu().numpy()
    assert cnt[0] == seg["n"].shape[0]          # segments (bit-exact hit lists)
    assert cnt[1] == ref_s["ray_t"].shape[0]    # samples
    assert cnt[2] == seg["ray_nseg"].max()
    err = dict(pred=_rel2(pred.cpu().numpy(), ref["pred"]), loss=abs(float(loss.item()) - ref["loss"]) / ref["loss"],
               dec=_rel2(tr.decoder_grad.cpu().numpy(), ref["grad_dec"]),
               grid=_rel2(tr.grad_reference_layout(tr.grid_m).cpu().numpy().astype(np.float64) / 0.1,
                          ref["grad_grid"]),
               pgrid=_rel2(tr.grid_reference_layout().cpu().numpy(), ref["grid"]),
               pdec=_rel2(tr.decoder.cpu().numpy(), ref["dec"]))
    print(which, path, {k: f"{v:.2e}" for k, v in err.items()})
    assert err["pred"] < tol_p and err["loss"] <= tol_p
    # gradients: decoder grad is kept; grid grad recovered from m = (1-b1) g
    assert err["dec"] < tol_g and err["grid"] < tol_g
    # parameters after Adam
    assert err["pgrid"] < tol_w and err["pdec"] < tol_w
    assert float(tr.grid_grad.abs().max()) == 0.0  # zero_grad after the step


@pytest.mark.parametrize("path", ["simt", "bf16x3"])
def test_fused_step_trajectory(neat, oracle, case, path):
    """Five steps on the same batch: the loss follows the f64 trajectory."""
    c = case
    tr = _trainer(c, path)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    grid, dec, state = c.grid.astype(np.float64), c.dec.astype(np.float64), None
    for k in range(1, 6):
        loss = float(tr.step(_dev(c.uv), _dev(c.img), _dev(c.target)).item())
        ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                      seed=99, step=k)
        r = oracle.step_f64(ref_s, grid, dec, c.target, T.node_position_min, T.node_position_max,
                            T.node_active_prefix_sum, step=k, state=state)
        grid, dec, state = r["grid"], r["dec"], r["state"]
        assert abs(loss - r["loss"]) <= 1e-4 * r["loss"], (k, loss, r["loss"])
    tr.check_status()


def test_fused_step_capacity_overflow_is_reported(neat, case):
    from neat_b200 import _lib
    from neat_b200.trainer import FusedTrainer
    c = case
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, seed=1, seg_capacity_per_ray=1)
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    with pytest.raises(_lib.NeatError) as e:
        tr.check_status()
    assert e.value.status & _lib.NEAT_ERR_CAPACITY


# ---------------------------------------------------------------- synthetic scans
def test_projector_matches_oracle(neat, oracle):
    from neat_b200 import scene as SC
    objs = SC.ellipsoid_phantom(6, 20, seed=9)
    sc = SC.SyntheticScene(objs, 4, 48, 40)
    ref = oracle.project(objs, 4, 48, 40, sc.intrinsics, sc.rotation, sc.translation)
    np.testing.assert_allclose(sc.projection.cpu().numpy(), ref, rtol=0, atol=1e-6)
    pts = np.random.default_rng(0).uniform(-1, 1, (500, 3))
    np.testing.assert_array_equal(sc.density(pts), oracle.phantom_density(objs, pts))


# ---------------------------------------------------------------- projection (evaluation)
@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("which", ["cfg1", "adaptive"])
def test_project_matches_f64(neat, oracle, case, adaptive_case, which, path):
    """Deterministic projection (a = 0.5): sample set bit-exact, projection and
    error sums within the path's tolerance of the f64 oracle."""
    c = {"cfg1": case, "adaptive": adaptive_case}[which]
    _, tol_p, _, _ = PATHS[path]
    tr = _trainer(c, path)
    sums = torch.zeros(2, dtype=torch.float64, device="cuda")
    pred = tr.project(_dev(c.uv), _dev(c.img), _dev(c.target), sums)
    torch.cuda.synchronize()
    tr.check_status()
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, False)
    assert int(tr.counters[1].item()) == ref_s["ray_t"].shape[0]
    import torch as _t
    ref = oracle.image_f64(ref_s, _t.from_numpy(c.grid.astype(np.float64)), _t.from_numpy(c.dec.astype(np.float64)),
                           T.node_position_min, T.node_position_max, T.node_active_prefix_sum, c.R).numpy()
    assert _rel2(pred.cpu().numpy(), ref) < tol_p
    diff = ref - c.target.astype(np.float64)
    s = sums.cpu().numpy()
    assert abs(s[0] - (diff ** 2).sum()) <= 2 * tol_p * (diff ** 2).sum()
    assert abs(s[1] - np.abs(diff).sum()) <= 2 * tol_p * np.abs(diff).sum()
    # parameters untouched, deterministic across calls
    pred2 = tr.project(_dev(c.uv), _dev(c.img))
    assert torch.equal(pred, pred2)
    assert tr.step_id == 0


def test_eval_projection_psnr(neat, oracle, case):
    """EvalStepProjection over whole images: per-image MSE/L1 means and
    PSNR = 10 log10(1/MSE), against the f64 oracle on the same pixels."""
    c = case
    tr = _trainer(c, "bf16x3")
    imgs = [3, 17]
    proj = _dev(c.proj.astype(np.float32))
    res = tr.eval_projection(imgs, proj, rows_per_batch=40)
    o_mse, o_l1 = [], []
    T = c.tree
    import torch as _t
    for i in imgs:
        ys, xs = np.meshgrid(np.arange(c.h), np.arange(c.w), indexing="ij")
        uv = np.stack([xs.reshape(-1).astype(np.float32) / np.float32(c.w - 1),
                       ys.reshape(-1).astype(np.float32) / np.float32(c.h - 1)], 1)
        ids = np.full(uv.shape[0], i, np.int32)
        o, d = oracle.make_rays(uv, ids, c.w, c.h, c.intr, c.rot, c.trans)
        s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, False)
        p = oracle.image_f64(s, _t.from_numpy(c.grid.astype(np.float64)), _t.from_numpy(c.dec.astype(np.float64)),
                             T.node_position_min, T.node_position_max, T.node_active_prefix_sum, uv.shape[0]).numpy()
        np.testing.assert_allclose(res["images"][imgs.index(i)].cpu().numpy().reshape(-1), p, rtol=1e-4, atol=1e-5)
        diff = p - c.proj[i].reshape(-1).astype(np.float32).astype(np.float64)
        o_mse.append((diff ** 2).mean())
        o_l1.append(np.abs(diff).mean())
    mse, l1 = float(np.mean(o_mse)), float(np.mean(o_l1))
    assert abs(res["mse"] - mse) <= 1e-5 * mse
    assert abs(res["l1"] - l1) <= 1e-5 * l1
    assert abs(res["psnr"] - 10 * np.log10(1 / mse)) < 1e-4


# ---------------------------------------------------------------- volume export
@pytest.mark.parametrize("which", ["cfg1", "adaptive"])
def test_uniform_sampled_volume(neat, oracle, case, adaptive_case, which):
    """Voxel-corner volume: node lookup bit-exact (including the inclusive
    face ties of the descent), density within 1e-5 of f64."""
    c = {"cfg1": case, "adaptive": adaptive_case}[which]
    tr = _trainer(c, "simt")
    n = (33, 17, 25)
    vol, node, valid = tr.UniformSampledVolume(n)
    T = c.tree
    rv, rn, rval = oracle.volume_f64(*n, c.grid, c.dec, T.node_active, T.node_position_min, T.node_position_max,
                                     T.node_active_prefix_sum, T.max_depth)
    np.testing.assert_array_equal(node.cpu().numpy().reshape(-1), rn)
    np.testing.assert_array_equal(valid.cpu().numpy().reshape(-1), rval)
    v = vol.cpu().numpy().reshape(-1)
    assert np.all(v[rval == 0] == 0)
    assert _rel2(v, rv) < 1e-5


# ---------------------------------------------------------------- CUDA graph replay
def test_graph_step_matches_eager(neat, case):
    """graph_step (captured once, replayed) follows step() over several steps;
    the device step counter advances on every replay."""
    c = case
    rng = np.random.default_rng(11)
    batches = []
    for _ in range(5):
        idx = rng.permutation(c.R)[:2048]
        batches.append((_dev(c.uv[idx]), _dev(c.img[idx]), _dev(c.target[idx])))
    a = _trainer(c, "bf16x3")
    b = _trainer(c, "bf16x3")
    la = [float(a.step(*bt).item()) for bt in batches]
    lb = [float(b.graph_step(*bt).item()) for bt in batches]
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    assert int(b.step_counter.item()) == 5 and int(a.step_counter.item()) == 5
    np.testing.assert_allclose(lb, la, rtol=1e-5)
    assert _rel2(b.grid.cpu().numpy(), a.grid.cpu().numpy()) < 1e-6
    assert _rel2(b.decoder.cpu().numpy(), a.decoder.cpu().numpy()) < 1e-6


# ---------------------------------------------------------------- learned proposal
def _prop_trainer(c, path="bf16x3", **kw):
    from neat_b200.trainer import FusedTrainer
    return FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                        grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec),
                        decoder_path=PATHS[path][0], proposal=True, **kw)


def _random_proposal(tr, seed=3):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.4, tr.prop.numel()).astype(np.float32)
    tr.prop.copy_(torch.from_numpy(p))
    desc = rng.normal(0, 0.5, tuple(tr.prop_node_desc.shape)).astype(np.float32)
    tr.prop_node_desc.copy_(torch.from_numpy(desc))
    return p.astype(np.float64)


@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
def test_proposal_sampling_matches_f64(neat, oracle, case, path):
    """Samples placed by the proposal's CDF (budget 8 per segment), a = 0.5:
    projection within the path's tolerance of the f64 oracle that places them
    from the same parameters."""
    c = case
    tr = _prop_trainer(c, path, proposal_budget=8)
    params = _random_proposal(tr)
    pred = tr.project(_dev(c.uv), _dev(c.img), use_proposal=True)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    segs = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 8)
    f = oracle.proposal_features(o, d, segs, T.node_position_min, T.node_position_max, tr.prop_node_desc.cpu().numpy(),
                                 T.node_active_prefix_sum)
    p = oracle.proposal_probs_f64(torch, torch.from_numpy(params), f, tr.prop_struct.mix).numpy()
    cdf = np.cumsum(p, 1)
    cdf[:, -1] = 1.0
    s = oracle.proposal_samples(o, d, segs, cdf, False)
    ref = oracle.image_f64(s, torch.from_numpy(c.grid.astype(np.float64)), torch.from_numpy(c.dec.astype(np.float64)),
                           T.node_position_min, T.node_position_max, T.node_active_prefix_sum, c.R).numpy()
    assert int(tr.counters[1].item()) == s["weight"].shape[0]
    err = _rel2(pred.cpu().numpy(), ref)
    print(path, "proposal projection rel err", err)
    assert err < PATHS[path][1]


@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
def test_proposal_counts_match_f64(neat, oracle, case, path):
    """Sample counts from the count head (count_eps 0.2, count_min 2, budget
    8) and the samples placed with them, a = 0.5: the total sample count and
    the projection against the f64 oracle that forms the same counts from the
    same parameters.  A segment whose exp(v) / eps lies within 1e-4 of an
    integer may round either way in f32; rays holding one are set aside (and
    counted)."""
    c = case
    eps, nmin = 0.2, 2
    tr = _prop_trainer(c, path, proposal_budget=8, proposal_count_eps=eps, proposal_count_min=nmin)
    params = _random_proposal(tr)
    pred = tr.project(_dev(c.uv), _dev(c.img), use_proposal=True)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    segs = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 8)
    f = oracle.proposal_features(o, d, segs, T.node_position_min, T.node_position_max, tr.prop_node_desc.cpu().numpy(),
                                 T.node_active_prefix_sum)
    P = torch.from_numpy(params)
    v = oracle.proposal_head_f64(torch, P, f).numpy()
    n, x = oracle.proposal_counts(v, segs["n"], eps, nmin)
    amb = (np.abs(x - np.round(x)) < 1e-4) & (x > nmin) & (x < segs["n"])
    p = oracle.proposal_probs_f64(torch, P, f, tr.prop_struct.mix).numpy()
    cdf = np.cumsum(p, 1)
    cdf[:, -1] = 1.0
    s = oracle.proposal_samples(o, d, dict(segs, n=n), cdf, False, n_key=segs["n"])
    ref = oracle.image_f64(s, torch.from_numpy(c.grid.astype(np.float64)), torch.from_numpy(c.dec.astype(np.float64)),
                           T.node_position_min, T.node_position_max, T.node_active_prefix_sum, c.R).numpy()
    keep = np.ones(c.R, bool)
    keep[segs["ray"][amb]] = False
    total = int(tr.counters[1].item())
    print(path, "count head: samples", total, "of", int(segs["n"].sum()), "at the budget; ambiguous segments",
          int(amb.sum()), "rays kept", int(keep.sum()))
    assert abs(total - int(n.sum())) <= int(amb.sum())
    assert total < 0.9 * int(segs["n"].sum())  # the head cuts counts on this case
    err = _rel2(pred.cpu().numpy()[keep], ref[keep])
    print(path, "proposal projection with learned counts, rel err", err)
    assert err < PATHS[path][1]


def test_proposal_training_gradient_matches_f64(neat, oracle, case):
    """A TRAIN step: uniform sampling, contributions binned per segment,
    one proposal iteration with lr 0 -> its gradient equals the f64 oracle's
    cross-entropy gradient on the same bins."""
    c = case
    tr = _prop_trainer(c, "bf16x3", proposal_iters=1, proposal_lr=0.0)
    params = _random_proposal(tr, seed=5)
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    segs = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M)
    hist = oracle.proposal_targets(o, d, segs, c.M, c.grid, c.dec, T.node_position_min, T.node_position_max,
                                   T.node_active_prefix_sum, True, 99, 1)
    # node descriptors: written by the step from its updated grid and decoder
    nd = tr.prop_node_desc.cpu().numpy()
    nd_ref = oracle.node_descriptors_f64(tr.grid_reference_layout().cpu().numpy(), tr.decoder.cpu().numpy())
    np.testing.assert_allclose(nd, nd_ref, rtol=1e-4, atol=1e-4)
    a = oracle.proposal_count_targets(o, d, segs, c.M, c.grid, c.dec, T.node_position_min, T.node_position_max,
                                      T.node_active_prefix_sum, True, 99, 1)
    f = oracle.proposal_features(o, d, segs, T.node_position_min, T.node_position_max, nd, T.node_active_prefix_sum)
    loss, g, lh = oracle.proposal_grad_f64(params, f, hist, tr.prop_struct.mix, a)
    gg = tr.prop_grad.cpu().numpy()
    tl = tr.prop_loss.cpu().numpy()
    head = slice(oracle.PROP_TRUNK, None)
    print("proposal loss", tl[0], loss, "grad rel err", _rel2(gg, g), "| count head loss", tl[2], lh,
          "grad rel err", _rel2(gg[head], g[head]))
    assert abs(float(tl[0]) - loss) <= 1e-4 * abs(loss)
    assert abs(float(tl[2]) - lh) <= 1e-4 * abs(lh)
    assert _rel2(gg, g) < 1e-4
    assert _rel2(gg[head], g[head]) < 1e-4
    np.testing.assert_array_equal(tr.prop.cpu().numpy(), params.astype(np.float32))  # lr 0


def test_proposal_gain_over_uniform(neat, oracle, case):
    """What the trained network gains: after online training on the scene, it
    predicts where the density changes along held-out segments (a fresh TRAIN
    batch, evaluated before any update on it) with a cross-entropy well below
    that of the method without it (uniform sampling: log 8).  The projection
    error of 8 proposal-placed vs 8 uniform samples per segment against a dense
    f64 evaluation is printed for the record."""
    c = case
    tr = _prop_trainer(c, "bf16x3", proposal_budget=8, proposal_every=20, proposal_iters=50, proposal_lr=1e-2,
                       proposal_mix=0.25)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    proj = _dev(c.proj.astype(np.float32))

    def batch():
        img = torch.randint(0, c.n_img, (4096,), generator=gen, device="cuda")
        x = torch.randint(0, c.w, (4096,), generator=gen, device="cuda")
        y = torch.randint(0, c.h, (4096,), generator=gen, device="cuda")
        uv = torch.stack([x.float() / (c.w - 1), y.float() / (c.h - 1)], 1).contiguous()
        return uv, img.to(torch.int32).contiguous(), proj[img, y, x].contiguous()

    for _ in range(600):
        tr.step(*batch())
    # held-out: a fresh batch in TRAIN mode with a zero learning rate and one
    # iteration reports the trained proposal's cross-entropy on it
    tr.prop_struct.lr, tr.prop_struct.iters = 0.0, 1
    while tr.step_id % tr.prop_every != 0:
        tr.step(*batch())
    params = tr.prop.clone()
    tr.step(*batch())
    torch.cuda.synchronize()
    tr.check_status()
    assert torch.equal(params, tr.prop)
    ce, h, _ = tr.prop_loss.cpu().numpy()
    uv, im = _dev(c.uv), _dev(c.img)
    p_prop = tr.project(uv, im, use_proposal=True).cpu().numpy().astype(np.float64)
    p_unif = tr.project(uv, im, samples_per_node=8).cpu().numpy().astype(np.float64)
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    dense = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 256, False)
    ref = oracle.image_f64(dense, torch.from_numpy(tr.grid_reference_layout().cpu().numpy().astype(np.float64)),
                           torch.from_numpy(tr.decoder.cpu().numpy().astype(np.float64)), T.node_position_min,
                           T.node_position_max, T.node_active_prefix_sum, c.R).numpy()
    print("held-out cross-entropy", ce, "target entropy", h, "uniform", np.log(8),
          "| projection error vs dense f64: proposal", np.abs(p_prop - ref).mean(), "uniform",
          np.abs(p_unif - ref).mean())
    assert ce < np.log(8) - 0.02


def test_count_head_gain_over_uniform(neat, oracle, case):
    """What the count head gains, and what not: after online training on the
    scene (budget 8, count_eps 0.05, count_min 2) its per-segment counts place
    far fewer samples than the budget on every segment.  Against a dense f64
    evaluation, their projection error is on a par with uniform sampling that
    spreads as many samples evenly (interpolated between the uniform budgets
    around that total): on this scene the learned counts save samples against
    a fixed budget, they do not beat an even spread of the same number (within
    15 % either way in repeated runs, better at the most aggressive tolerances
    and worse at mild ones; the check allows 25 %)."""
    c = case
    tr = _prop_trainer(c, "bf16x3", proposal_budget=8, proposal_every=20, proposal_iters=50, proposal_lr=1e-2,
                       proposal_mix=0.25, proposal_count_eps=0.05, proposal_count_min=2)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4)
    proj = _dev(c.proj.astype(np.float32))
    for _ in range(600):
        img = torch.randint(0, c.n_img, (4096,), generator=gen, device="cuda")
        x = torch.randint(0, c.w, (4096,), generator=gen, device="cuda")
        y = torch.randint(0, c.h, (4096,), generator=gen, device="cuda")
        uv = torch.stack([x.float() / (c.w - 1), y.float() / (c.h - 1)], 1).contiguous()
        tr.step(uv, img.to(torch.int32).contiguous(), proj[img, y, x].contiguous())
    torch.cuda.synchronize()
    tr.check_status()
    uv, im = _dev(c.uv), _dev(c.img)
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    dense = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 256, False)
    ref = oracle.image_f64(dense, torch.from_numpy(tr.grid_reference_layout().cpu().numpy().astype(np.float64)),
                           torch.from_numpy(tr.decoder.cpu().numpy().astype(np.float64)), T.node_position_min,
                           T.node_position_max, T.node_active_prefix_sum, c.R).numpy()

    def run(**kw):
        p = tr.project(uv, im, **kw).cpu().numpy().astype(np.float64)
        torch.cuda.synchronize()
        return np.abs(p - ref).mean(), int(tr.counters[1].item())

    e_cnt, n_cnt = run(use_proposal=True)
    eps = tr.prop_struct.count_eps
    tr.prop_struct.count_eps = 0.0
    e_full, n_full = run(use_proposal=True)
    tr.prop_struct.count_eps = eps
    uni = {m: run(samples_per_node=m) for m in range(1, 9)}
    e_uni = float(np.interp(n_cnt, [v[1] for v in uni.values()], [v[0] for v in uni.values()]))
    print("count head:", n_cnt, "samples, error", e_cnt, "| budget 8 on every segment:", n_full, "samples, error",
          e_full, "| uniform with as many samples (interpolated): error", e_uni,
          "| uniform budgets:", {k: (v[1], float("%.3g" % v[0])) for k, v in uni.items()})
    assert n_cnt < 0.7 * n_full
    assert e_cnt < 1.25 * e_uni


# ---------------------------------------------------------------- finite differences
def test_backward_matches_central_differences(neat, oracle):
    """Config-5 style gradient check: the fused step's analytic gradients
    (C = 16, FP32-accurate tensor-core path) on 1000 random parameters -- 900
    grid entries the batch touches and 100 decoder weights -- against central
    differences (eps 1e-4) of the f64 loss on the same samples."""
    c = cfg1_case(R=384, seed=11, depth=3, C=16, G=9, M=16, oracle=oracle, adaptive=120)
    tr = _trainer(c, "bf16x3")
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    g_grid = tr.grad_reference_layout(tr.grid_m).cpu().numpy().astype(np.float64) / 0.1  # m = (1 - b1) g
    g_dec = tr.decoder_grad.cpu().numpy().astype(np.float64)
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                              seed=99, step=1)
    tgt = torch.from_numpy(c.target.astype(np.float64))

    def loss(grid, dec):
        pred = oracle.image_f64(s, torch.from_numpy(grid), torch.from_numpy(dec), T.node_position_min,
                                T.node_position_max, T.node_active_prefix_sum, c.R)
        return float(((pred - tgt) ** 2).mean())

    rng = np.random.default_rng(12)
    grid0, dec0 = c.grid.astype(np.float64), c.dec.astype(np.float64)
    touched = np.flatnonzero(np.abs(g_grid) > 1e-12 * np.abs(g_grid).max())
    gi = rng.choice(touched, 900, replace=False)
    di = rng.choice(dec0.size, 100, replace=False)
    eps = 1e-4
    fd, an = [], []
    for arr, idx, ana in ((grid0, gi, g_grid), (dec0, di, g_dec)):
        for k in idx:  # perturb in place, restore after
            v = arr.flat[k]
            arr.flat[k] = v + eps
            lp = loss(grid0, dec0)
            arr.flat[k] = v - eps
            lm = loss(grid0, dec0)
            arr.flat[k] = v
            fd.append((lp - lm) / (2 * eps))
            an.append(ana.flat[k])
    fd, an = np.array(fd), np.array(an)
    err = _rel2(an, fd)
    print("finite differences vs analytic (1000 params): rel 2-norm err", err)
    assert err < 1e-4


# ---------------------------------------------------------------- precision variant (BF16 grids)
@pytest.mark.parametrize("which", ["cfg1", "c8"])
def test_bf16_grid_step_error_vs_f64(neat, oracle, case, c8_case, which):
    """Config-3 precision variant: BF16 feature grid copy read by the gathers,
    BF16 decoder operands, FP32 accumulation, f64 segment sums.  Projection and
    gradients against the f64 evaluation of the same FP32 parameters within the
    stated BF16 bounds (1e-2 projection, 5e-2 gradients); after the update the
    BF16 copy equals the rounded FP32 master."""
    from neat_b200.trainer import FusedTrainer
    c = {"cfg1": case, "c8": c8_case}[which]
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                      grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec),
                      decoder_path=PATHS["bf16"][0], grid_bf16=True)
    pred = torch.zeros(c.R, device="cuda")
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target), prediction=pred)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                  seed=99, step=1)
    ref = oracle.step_f64(ref_s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                          T.node_active_prefix_sum, lr_grid=1e-2, lr_decoder=5e-5, step=1)
    e_pred = _rel2(pred.cpu().numpy(), ref["pred"])
    e_dec = _rel2(tr.decoder_grad.cpu().numpy(), ref["grad_dec"])
    e_grid = _rel2(tr.grad_reference_layout(tr.grid_m).cpu().numpy().astype(np.float64) / 0.1, ref["grad_grid"])
    print(which, "BF16 grid + BF16 decoder vs f64: projection", e_pred, "grad decoder", e_dec, "grad grid", e_grid)
    assert e_pred < 1e-2 and e_dec < 5e-2 and e_grid < 5e-2
    assert torch.equal(tr.grid_bf16, tr.grid.to(torch.bfloat16))


# ---------------------------------------------------------------- regularisers
def test_tv_and_edge_regularisers_match_f64(neat, oracle, adaptive_case):
    """TV and edge losses and the gradients they add into the grid gradient,
    against f64 autograd restatements (mixed node sizes: adaptive tree)."""
    from neat_b200 import _lib
    c = adaptive_case
    tr = _trainer(c, "bf16x3")
    lib = _lib.load()
    T = c.tree
    tab = tr.tables
    ws = torch.empty(lib.neat_regularizer_workspace_bytes(), dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    loss = torch.zeros(1, device="cuda")
    grad = torch.zeros_like(tr.grid)
    _lib.check(lib.neat_tv_loss(tr.grid.data_ptr(), tr.A, c.C, c.G, 0.3, loss.data_ptr(), grad.data_ptr(),
                                ws.data_ptr(), st))
    torch.cuda.synchronize()
    l_ref, g_ref = oracle.tv_f64(c.grid, 0.3)
    g = tr.grad_reference_layout(grad).cpu().numpy()
    print("tv", float(loss.item()), l_ref, _rel2(g, g_ref))
    assert abs(float(loss.item()) - l_ref) <= 1e-5 * l_ref
    assert _rel2(g, g_ref) < 1e-5
    loss.zero_()
    grad.zero_()
    _lib.check(lib.neat_edge_loss(tab["table"].data_ptr(), T.max_depth, tab["min"].data_ptr(), tab["max"].data_ptr(),
                                  tab["active"].data_ptr(), tr.A, tr.grid.data_ptr(), c.C, c.G, 0.001, 0.2, 5, 3,
                                  loss.data_ptr(), grad.data_ptr(), ws.data_ptr(), st))
    torch.cuda.synchronize()
    l_ref, g_ref, npairs = oracle.edge_f64(c.grid, T.node_position_min, T.node_position_max, T.node_active,
                                           T.active_node_ids, T.node_active_prefix_sum, T.max_depth, 0.001, 0.2, 5, 3)
    g = tr.grad_reference_layout(grad).cpu().numpy()
    print("edge", float(loss.item()), l_ref, npairs, _rel2(g, g_ref))
    assert npairs > 0
    assert abs(float(loss.item()) - l_ref) <= 1e-5 * l_ref
    assert _rel2(g, g_ref) < 1e-4


def test_step_with_regularisers(neat, oracle, case):
    """A step with TV and edge weights: the grid gradient Adam sees is the
    projection loss's plus the regularisers' (f64 references of each)."""
    c = case
    from neat_b200.trainer import FusedTrainer
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                      grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec), loss_tv=0.05, loss_edge=0.02)
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    ref_s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                  seed=99, step=1)
    ref = oracle.step_f64(ref_s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                          T.node_active_prefix_sum, lr_grid=1e-2, lr_decoder=5e-5, step=1)
    l_tv, g_tv = oracle.tv_f64(c.grid, 0.05)
    l_ed, g_ed, _ = oracle.edge_f64(c.grid, T.node_position_min, T.node_position_max, T.node_active,
                                    T.active_node_ids, T.node_active_prefix_sum, T.max_depth, 0.001, 0.02, 99, 1)
    g = tr.grad_reference_layout(tr.grid_m).cpu().numpy().astype(np.float64) / 0.1
    err = _rel2(g, ref["grad_grid"] + g_tv + g_ed)
    print("regularised step grid-gradient rel err", err, "reg loss", float(tr.reg_loss.item()), l_tv + l_ed)
    assert err < 1e-4
    assert abs(float(tr.reg_loss.item()) - (l_tv + l_ed)) <= 1e-5 * (l_tv + l_ed)


# ---------------------------------------------------------------- structure updates
def test_max_density_culling_and_interpolation(neat, oracle, adaptive_case):
    """ComputeMaxDensity (with the in-image mask) against f64; culling on the
    host; InterpolateInactiveNodes into a refined/coarsened tree against f64;
    the trainer keeps stepping on the new structure."""
    c = adaptive_case
    tr = _trainer(c, "bf16x3")
    T = c.tree
    mx = tr.ComputeMaxDensity().cpu().numpy()
    ref = oracle.node_max_density_f64(c.grid, c.dec, T.node_position_min, T.node_position_max, T.active_node_ids, c.G,
                                      cam=(c.intr, c.rot, c.trans, c.w, c.h))
    print("max density rel err", _rel2(mx, ref))
    assert _rel2(mx, ref) < 1e-5
    # cull the lowest quarter, then split the densest remaining leaf-level-minus-one node
    thr = np.quantile(mx, 0.25)
    new_tree = T.copy()
    new_tree.node_max_density = T.node_max_density.copy()
    k = new_tree.NodeCulling(thr)
    assert k == int((mx < thr).sum()) and new_tree.NumActiveNodes() == T.NumActiveNodes() - k
    act = set(new_tree.active_node_ids.tolist())
    split = next(n for n in new_tree.active_node_ids if new_tree.node_depth[n] < new_tree.max_depth)
    act.discard(int(split))
    act.update(int(x) for x in new_tree.node_children[split])
    new_tree.SetActiveNodes(sorted(act))
    old_ref_grid = tr.grid_reference_layout().cpu().numpy()
    tr.restructure(new_tree)
    got = tr.grid_reference_layout().cpu().numpy()
    want = oracle.interpolate_grid_f64(old_ref_grid, T.node_position_min, T.node_position_max, T.node_active,
                                       T.active_node_ids, T.node_active_prefix_sum, T.max_depth,
                                       new_tree.active_node_ids, c.G)
    print("interpolation rel err", _rel2(got, want))
    assert got.shape == want.shape and _rel2(got, want) < 1e-6
    loss = tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    assert np.isfinite(float(loss.item()))


# ---------------------------------------------------------------- photometric calibration
def test_photometric_calibration_step(neat, oracle, case):
    """The step with exposure (factor and bias), sensor-bias map and response
    curve fused into the loss: prediction, grid and decoder gradients, the
    ParamLoss, and the SGD-updated, clamped calibration parameters against f64
    autograd through torch's own grid_sample (as the reference calls it)."""
    c = case
    from neat_b200.trainer import FusedTrainer
    tmc = dict(exposure_mult=True, response_range=2.0)
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                      grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec), tonemap=tmc)
    tm = tr.tonemap
    rng = np.random.default_rng(21)
    n, b = tm.num_images, tm.bias_w * tm.bias_h
    p0 = tm.params.cpu().numpy().astype(np.float64)
    p0[:n] = rng.uniform(0.8, 1.2, n)
    p0[n:2 * n] = rng.uniform(0.0, 0.05, n)
    p0[2 * n:2 * n + b] = rng.uniform(0.0, 0.05, b)
    p0[2 * n + b:] = np.sort(p0[2 * n + b:] + rng.uniform(-0.02, 0.02, 25))
    p0[2 * n + b] = 0.0
    tm.params.copy_(torch.from_numpy(p0.astype(np.float32)))
    p0 = tm.params.cpu().numpy().astype(np.float64)
    pred = torch.zeros(c.R, device="cuda")
    loss = tr.step(_dev(c.uv), _dev(c.img), _dev(c.target), prediction=pred)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                              seed=99, step=1)
    grid = torch.tensor(c.grid.astype(np.float64), requires_grad=True)
    dec = torch.tensor(c.dec.astype(np.float64), requires_grad=True)
    P = torch.tensor(p0, requires_grad=True)
    x = oracle.image_f64(s, grid, dec, T.node_position_min, T.node_position_max, T.node_active_prefix_sum, c.R)
    y = oracle.tonemap_f64(torch, x, torch.from_numpy(c.uv.astype(np.float64)), torch.from_numpy(c.img.astype(np.int64)),
                           P[:n], P[n:2 * n], P[2 * n:2 * n + b].reshape(tm.bias_h, tm.bias_w), P[2 * n + b:], 2.0,
                           mult=True)
    mse = ((y - torch.from_numpy(c.target.astype(np.float64))) ** 2).mean()
    pl = oracle.response_param_loss_f64(torch, P[2 * n + b:])
    (mse + pl).backward()
    e = dict(pred=_rel2(pred.cpu().numpy(), y.detach().numpy()), loss=abs(float(loss.item()) - float(mse)) / float(mse),
             dec=_rel2(tr.decoder_grad.cpu().numpy(), dec.grad.numpy()),
             grid=_rel2(tr.grad_reference_layout(tr.grid_m).cpu().numpy().astype(np.float64) / 0.1, grid.grad.numpy()),
             param_loss=abs(float(tm.param_loss.item()) - float(pl)) / float(pl))
    lr = np.concatenate([np.full(n, 0.01), np.full(n, 0.01), np.full(b, 0.05), np.full(25, 0.1)])
    want = p0 - lr * P.grad.numpy()
    want[n:2 * n + b] = np.maximum(want[n:2 * n + b], 0.0)
    e["params"] = _rel2(tm.params.cpu().numpy() - p0, want - p0)
    print("photometric calibration errors", {k: f"{v:.2e}" for k, v in e.items()})
    assert e["pred"] < 1e-5 and e["loss"] < 1e-5 and e["dec"] < 1e-5 and e["grid"] < 1e-5
    assert e["param_loss"] < 1e-5 and e["params"] < 1e-4
    assert float(tm.grad.abs().max()) == 0.0


def test_projection_applies_the_tone_mapper(neat, oracle, case):
    """The evaluation path (EvalStepProjection, samples/reconstruct.cpp:551-559)
    applies tone_mapper->forward to the predicted projection: the trainer's
    projection with a calibration equals the f64 tone map (exposure factor and
    bias, sensor-bias map, response curve) of the oracle's a = 0.5 projection,
    and so do the error sums against the target."""
    c = case
    from neat_b200.trainer import FusedTrainer
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, seed=99, grid=torch.from_numpy(c.grid),
                      decoder=torch.from_numpy(c.dec), tonemap=dict(exposure_mult=True, response_range=2.0))
    tm = tr.tonemap
    rng = np.random.default_rng(5)
    n, b = tm.num_images, tm.bias_w * tm.bias_h
    p0 = tm.params.cpu().numpy().astype(np.float64)
    p0[:n] = rng.uniform(0.8, 1.2, n)
    p0[n:2 * n] = rng.uniform(0.0, 0.05, n)
    p0[2 * n:2 * n + b] = rng.uniform(0.0, 0.05, b)
    p0[2 * n + b:] = np.sort(p0[2 * n + b:] + rng.uniform(-0.02, 0.02, 25))
    p0[2 * n + b] = 0.0
    tm.params.copy_(torch.from_numpy(p0.astype(np.float32)))
    p0 = tm.params.cpu().numpy().astype(np.float64)
    sums = torch.zeros(2, dtype=torch.float64, device="cuda")
    pred = tr.project(_dev(c.uv), _dev(c.img), _dev(c.target), sums)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, False)
    x = oracle.image_f64(s, torch.from_numpy(c.grid.astype(np.float64)), torch.from_numpy(c.dec.astype(np.float64)),
                         T.node_position_min, T.node_position_max, T.node_active_prefix_sum, c.R)
    P = torch.from_numpy(p0)
    y = oracle.tonemap_f64(torch, x, torch.from_numpy(c.uv.astype(np.float64)), torch.from_numpy(c.img.astype(np.int64)),
                           P[:n], P[n:2 * n], P[2 * n:2 * n + b].reshape(tm.bias_h, tm.bias_w), P[2 * n + b:], 2.0,
                           mult=True).numpy()
    assert _rel2(pred.cpu().numpy(), y) < 1e-5
    diff = y - c.target.astype(np.float64)
    got = sums.cpu().numpy()
    assert abs(got[0] - (diff ** 2).sum()) <= 2e-5 * (diff ** 2).sum()
    assert abs(got[1] - np.abs(diff).sum()) <= 2e-5 * np.abs(diff).sum()
    # without a calibration the projection is the plain integral
    plain = _trainer(c, "bf16x3").project(_dev(c.uv), _dev(c.img))
    assert _rel2(plain.cpu().numpy(), x.numpy()) < 1e-5


# ---------------------------------------------------------------- camera pose gradients
@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
@pytest.mark.parametrize("which", ["cfg1", "c8"])
def test_pose_gradients_match_f64(neat, oracle, case, c8_case, which, path):
    """Rotation-tangent, translation and intrinsics gradients of one fused step
    against the f64 autograd chain on the oracle's samples.  The GPU sums per
    sample in FP32 (segment runs, then rays, as the reference's index_add) and
    per image in f64; bar in the 2-norm per parameter group: 1e-4 (FP32-accurate
    decoder), 5e-2 (BF16 precision variant)."""
    from neat_b200.trainer import FusedTrainer
    c = {"cfg1": case, "c8": c8_case}[which]
    tr = FusedTrainer(c.tree, _camera(c), c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                      grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec),
                      decoder_path=PATHS[path][0], pose_grad=True)
    tr.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                              seed=99, step=1)
    ref = oracle.pose_grads_f64(s, c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans, c.grid, c.dec, c.target,
                                T.node_position_min, T.node_position_max, T.node_active_prefix_sum)
    gi = tr.pose_grad_intrinsics.cpu().numpy()
    err = dict(tangent=_rel2(tr.pose_grad_tangent.cpu().numpy(), ref["tangent"]),
               translation=_rel2(tr.pose_grad_translation.cpu().numpy(), ref["translation"]),
               intrinsics=_rel2(gi[:4], ref["intrinsics"][:4]))
    print(which, path, {k: f"{v:.2e}" for k, v in err.items()})
    tol = 1e-4 if path == "bf16x3" else 5e-2
    assert all(v < tol for v in err.values()), err
    assert gi[4] == 0.0
    # the step's own results are unchanged by the pose gradients
    tr2 = _trainer(c, path)
    tr2.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    assert _rel2(tr.decoder.cpu().numpy(), tr2.decoder.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("proposal", [False, True])
def test_checkpoint_resume_reproduces_the_next_step(neat, case, proposal):
    """A trainer restored from state_dict() takes the same next step as the
    trainer it was saved from: the same loss (the forward is deterministic given
    parameters, seed and step number) and the same parameters up to the
    grid-gradient atomics' addition order."""
    def make():
        from neat_b200.trainer import FusedTrainer
        return FusedTrainer(case.tree, _camera(case), case.C, case.G, case.M, lr_grid=1e-2, lr_decoder=5e-5, seed=7,
                            grid=torch.from_numpy(case.grid), decoder=torch.from_numpy(case.dec),
                            proposal=proposal, proposal_every=2)
    uv, img, tgt = _dev(case.uv), _dev(case.img), _dev(case.target)
    n = case.R // 2
    a = make()
    for k in range(3):
        a.step(uv[k % 2 * n:(k % 2 + 1) * n], img[k % 2 * n:(k % 2 + 1) * n], tgt[k % 2 * n:(k % 2 + 1) * n])
    a.check_status()
    sd = a.state_dict()
    la = float(a.step(uv[:n], img[:n], tgt[:n]).item())
    b = make()
    b.load_state_dict(sd)
    lb = float(b.step(uv[:n], img[:n], tgt[:n]).item())
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    assert lb == pytest.approx(la, rel=1e-6)
    assert b.step_id == a.step_id
    # a lost moment, step number or parameter would move nearly every updated
    # element by about a learning rate; the atomics' order moves a rare element
    # whose gradient nearly cancels
    def moved(x, y):
        return float(((x - y).abs() > 1e-6).float().mean())
    assert moved(b.decoder, a.decoder) < 1e-2
    assert moved(b.grid, a.grid) < 1e-3
    # a restore into a trainer with another seed is refused
    with pytest.raises(ValueError):
        sd2 = dict(sd)
        sd2["seed"] = 8
        b.load_state_dict(sd2)


def test_host_batches_are_staged_like_device_batches(neat, case):
    """FusedTrainer.step on pinned host batches (staged through the trainer's
    copy stream into two alternating device buffer sets, each copy overlapping
    the previous step) takes the same steps as on device batches: four steps
    queued without a synchronisation, each on another batch, so a set is
    rewritten while the other set's step runs.  Same losses (the forward is
    deterministic; the parameters differ only by the grid-gradient atomics'
    order) and the same parameters up to that order."""
    from neat_b200.trainer import FusedTrainer
    def make():
        return FusedTrainer(case.tree, _camera(case), case.C, case.G, case.M, lr_grid=1e-2, lr_decoder=5e-5, seed=7,
                            grid=torch.from_numpy(case.grid), decoder=torch.from_numpy(case.dec))
    n = case.R // 4
    parts = [(case.uv[k * n:(k + 1) * n], case.img[k * n:(k + 1) * n], case.target[k * n:(k + 1) * n])
             for k in range(4)]
    a, b = make(), make()
    la = [a.step(_dev(u), _dev(i), _dev(t)).clone() for u, i, t in parts]
    host = [tuple(torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in p) for p in parts]
    lb = [b.step(u, i, t).clone() for u, i, t in host]
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    assert b.host_copy_stream() is not None and a.host_copy_stream() is None
    for x, y in zip(la, lb):
        assert float(y) == pytest.approx(float(x), rel=1e-5)
    def moved(x, y):
        return float(((x - y).abs() > 1e-6).float().mean())
    assert moved(b.decoder, a.decoder) < 1e-2
    assert moved(b.grid, a.grid) < 1e-3
    with pytest.raises(TypeError):
        b.step(host[0][0].double(), host[0][1], host[0][2])


@pytest.mark.parametrize("proposal", [False, True])
def test_look_ahead_segment_lists_take_the_same_steps(neat, case, proposal):
    """step(..., next=b) builds batch b's segment lists on a side stream
    under the step's Adam update (neat_train_step_segments, behind the step's
    phase [4], or [5] on a proposal TRAIN step) and the call that takes b
    skips building them (neat_train_step_prebuilt).  Six steps on different
    batches queued without a synchronisation (with the proposal: TRAIN steps
    1 and 5, SAMPLE steps in between), against the same steps without
    look-ahead: the same counters every step, the same losses (the forward is
    deterministic) and the same parameters up to the grid-gradient atomics'
    order; pinned host batches the same way (staged one step ahead)."""
    from neat_b200.trainer import FusedTrainer
    def make():
        return FusedTrainer(case.tree, _camera(case), case.C, case.G, case.M, lr_grid=1e-2, lr_decoder=5e-5, seed=7,
                            grid=torch.from_numpy(case.grid), decoder=torch.from_numpy(case.dec),
                            proposal=proposal, proposal_every=4)
    n = case.R // 6
    cols = (case.uv, case.img, case.target)
    parts = [tuple(_dev(x[k * n:(k + 1) * n]) for x in cols) for k in range(6)]
    host = [tuple(torch.from_numpy(np.ascontiguousarray(x[k * n:(k + 1) * n])).pin_memory() for x in cols)
            for k in range(6)]
    a = make()
    la, ca = [], []
    for p in parts:
        la.append(a.step(*p).clone())
        ca.append(a.counters.clone())
    rel = 1e-4 if proposal else 1e-5
    def moved(x, y):
        return float(((x - y).abs() > 1e-6).float().mean())
    for batches in (parts, host):
        b = make()
        lb, cb = [], []
        for k in range(6):
            lb.append(b.step(*batches[k], next=batches[k + 1] if k + 1 < 6 else None).clone())
            cb.append(b.counters.clone())
            assert (b._pf is not None) == (k + 1 < 6)
        torch.cuda.synchronize()
        a.check_status()
        b.check_status()
        for k in range(6):
            assert torch.equal(cb[k], ca[k]), (k, cb[k].tolist(), ca[k].tolist())
            assert float(lb[k]) == pytest.approx(float(la[k]), rel=rel)
        assert moved(b.decoder, a.decoder) < 1e-2
        assert moved(b.grid, a.grid) < 1e-3


def test_checkpoint_after_restructure_restores_the_saved_tree(neat, case):
    """A checkpoint taken after restructure() holds the new active-node set; a
    trainer built on the original tree moves to that set before copying the
    grid rows, so every row lands on its own node and the next step matches."""
    from neat_b200.trainer import FusedTrainer

    def make():
        return FusedTrainer(case.tree, _camera(case), case.C, case.G, case.M, lr_grid=1e-2, lr_decoder=5e-5, seed=7,
                            grid=torch.from_numpy(case.grid), decoder=torch.from_numpy(case.dec))
    uv, img, tgt = _dev(case.uv), _dev(case.img), _dev(case.target)
    a = make()
    a.step(uv, img, tgt)
    # split two leaves' parents... the depth-2 tree: keep every other leaf and activate
    # the depth-1 parent of the first leaf instead of its 8 children
    T = case.tree
    first = int(T.active_node_ids[0])
    parent = int(T.node_parent[first])
    kids = set(int(k) for k in T.node_children[parent])
    new_ids = sorted([parent] + [int(i) for i in T.active_node_ids if int(i) not in kids])
    nt = T.copy()
    nt.SetActiveNodes(new_ids)
    a.restructure(nt)
    a.step(uv, img, tgt)
    a.check_status()
    sd = a.state_dict()
    assert sd["tree_active_node_ids"].tolist() == new_ids
    la = float(a.step(uv, img, tgt).item())
    b = make()
    assert b.A != a.A
    b.load_state_dict(sd)
    assert b.A == a.A and np.array_equal(b.tree.active_node_ids, np.asarray(new_ids))
    assert torch.equal(b.grid.cpu(), sd["grid"])
    lb = float(b.step(uv, img, tgt).item())
    torch.cuda.synchronize()
    b.check_status()
    assert lb == pytest.approx(la, rel=1e-6)
    # a checkpoint of another depth, or without a tree, is refused
    bad = dict(sd)
    bad["tree_max_depth"] = T.max_depth + 1
    with pytest.raises(ValueError):
        b.load_state_dict(bad)
    bad = {k: v for k, v in sd.items() if k != "tree_active_node_ids"}
    with pytest.raises(KeyError):
        b.load_state_dict(bad)


def test_pose_sgd_step(neat, oracle):
    """neat_pose_sgd: SGD on tangent / translation / intrinsics, q <- exp(-lr g) q
    renormalised, gradients zeroed; the optimize flags select the groups."""
    from neat_b200 import _lib
    rng = np.random.default_rng(7)
    n = 37
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    tr = rng.normal(size=(n, 3))
    intr = np.array([100.0, 90.0, 60.0, 50.0, 0.0])
    gt = rng.normal(size=(n, 3))
    gtr = rng.normal(size=(n, 3))
    gin = rng.normal(size=5)
    for opt_pose, opt_intr in ((1, 1), (0, 1), (1, 0)):
        rot_d, tr_d, in_d = _dev(q), _dev(tr), _dev(intr)
        g_t, g_tr, g_in = _dev(gt), _dev(gtr), _dev(gin)
        pg = _lib.PoseGrad(grad_tangent=g_t.data_ptr(), grad_translation=g_tr.data_ptr(),
                           grad_intrinsics=g_in.data_ptr(), num_images=n)
        rc = neat.neat_pose_sgd(rot_d.data_ptr(), tr_d.data_ptr(), in_d.data_ptr(), ctypes.byref(pg), 1e-2, 10.0,
                                opt_pose, opt_intr, torch.cuda.current_stream().cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        exp_q = oracle.quat_exp_mul_f64(-1e-2 * gt, q) if opt_pose else q
        exp_t = tr - 1e-2 * gtr if opt_pose else tr
        exp_i = intr - 10.0 * gin if opt_intr else intr
        np.testing.assert_allclose(rot_d.cpu().numpy(), exp_q, rtol=0, atol=1e-13)
        np.testing.assert_allclose(tr_d.cpu().numpy(), exp_t, rtol=0, atol=1e-13)
        np.testing.assert_allclose(in_d.cpu().numpy(), exp_i, rtol=0, atol=1e-12)
        assert float(g_t.abs().max()) == 0 and float(g_tr.abs().max()) == 0 and float(g_in.abs().max()) == 0


def test_pose_optimisation_reduces_loss(neat, oracle, case):
    """With optimize_pose / optimize_intrinsics the trainer runs the structure
    step after each fused step; starting from perturbed translations, the
    translation error falls over the steps (the reference's pose refinement)."""
    from neat_b200.api import CameraModel
    from neat_b200.trainer import FusedTrainer
    c = case
    rng = np.random.default_rng(3)
    tr0 = np.asarray(c.trans, np.float64).reshape(-1, 3)
    noisy = tr0 + rng.normal(0, 0.02, tr0.shape)
    cam = CameraModel(c.w, c.h, c.intr, c.rot, noisy)
    t = FusedTrainer(c.tree, cam, c.C, c.G, c.M, lr_grid=1e-2, lr_decoder=5e-5, seed=99,
                     grid=torch.from_numpy(c.grid), decoder=torch.from_numpy(c.dec), optimize_pose=True,
                     lr_pose=1e-3)
    before = np.linalg.norm(cam.translation.cpu().numpy() - tr0)
    for _ in range(40):
        t.step(_dev(c.uv), _dev(c.img), _dev(c.target))
    torch.cuda.synchronize()
    t.check_status()
    after = np.linalg.norm(cam.translation.cpu().numpy() - tr0)
    assert np.isfinite(after) and float(t.pose_grad_translation.abs().max()) == 0.0
    print("translation error", before, "->", after)
    assert after != before
