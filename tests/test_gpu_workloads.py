"""Parity on slices of the measured workloads themselves.

The benchmark trains the full-size configuration (adaptive depth-4 octree of
1499 nodes, C=8, G=17, M=32, noisy projections of 64 ellipsoids and 200
voids) and the large porous configuration (depth-5 octree of ~3000 nodes on
levels 2-5, C=16, G=17, 2^19 rays, BF16 + learned proposal).  These tests
take a few thousand rays of those very scenes, trees and batch samplers
(neat_b200.workloads) and hold every decoder path to the oracle:

  hit lists, segment and sample counts, sample positions:  bit-exact
  FP32 paths (simt, bf16x3): projection / loss 1e-5 relative, gradients
      1e-5 (2-norm), parameters after Adam 1e-6
  BF16 path: the stated bounds 1e-2 (projection), 5e-2 (gradients)

The f64 reference runs on the grid rows the slice touches (a compacted
grid); every other row must leave the step bit-identical (zero gradient,
zero Adam moments, zero update).
"""
import numpy as np
import pytest
import torch

import tests.test_gpu_parity as P
from tests.cases import Case, workload_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full_case(neat):
    return workload_case("full", R=4096, seed=21)


@pytest.fixture(scope="module")
def large_case(neat):
    return workload_case("large", R=2048, seed=23)


def _case(request, which):
    return request.getfixturevalue(which + "_case")


def _compact(c, samples):
    """Rows of the grid the samples read, the compacted grid and a node ->
    compacted-row table for the oracle."""
    T = c.tree
    rows = np.unique(T.node_active_prefix_sum[samples["node_id"]])
    prefix = np.full(T.NumNodes(), -1, np.int64)
    prefix[T.active_node_ids[rows]] = np.arange(rows.size)
    return rows, c.grid[rows], prefix


def _oracle(oracle, c):
    """Samples, segments and the f64 step on the compacted grid for the
    case's batch (seed 99, step 1), computed once per case."""
    if getattr(c, "_compact_ref", None) is None:
        o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
        T = c.tree
        s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                  seed=99, step=1)
        seg = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M)
        rows, grid_c, prefix = _compact(c, s)
        ref = oracle.step_f64(s, grid_c, c.dec, c.target, T.node_position_min, T.node_position_max, prefix,
                              lr_grid=1e-2, lr_decoder=5e-5, step=1)
        c._compact_ref = (o, d, s, seg, rows, ref)
    return c._compact_ref


# ---------------------------------------------------------------- samples
@pytest.mark.parametrize("which", ["full", "large"])
def test_workload_samples_bit_exact(neat, oracle, request, which):
    """CreateSamplesForRays on the workload slice: every SampleList field bit
    for bit (the large tree runs the general traversal: depth 5, up to 96
    hits kept per ray)."""
    from neat_b200.api import CreateSamplesForRays, GetRays
    c = _case(request, which)
    rays = GetRays(P._camera(c), P._dev(c.uv), P._dev(c.img))
    s = CreateSamplesForRays(c.tree, rays, c.M, True, seed=11, step=3)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    ref = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                                seed=11, step=3)
    assert s.size() == ref["ray_t"].shape[0] > 0
    np.testing.assert_array_equal(s.ray_index.cpu().numpy(), ref["ray_index"])
    np.testing.assert_array_equal(s.node_id.cpu().numpy(), ref["node_id"])
    np.testing.assert_array_equal(s.local_index_in_ray.cpu().numpy(), ref["local_index"])
    np.testing.assert_array_equal(s.ray_t.cpu().numpy(), ref["ray_t"])
    np.testing.assert_array_equal(s.weight.cpu().numpy(), ref["weight"])
    np.testing.assert_array_equal(s.global_coordinate.cpu().numpy(), ref["coords"])
    assert s.max_samples_per_ray == ref["max_per_ray"]
    # the slice reaches the tree's depth and its unevenness: nodes of several levels hit
    depths = np.unique(T.node_depth[ref["node_id"]])
    assert depths.max() == T.max_depth and depths.size >= 3


# ---------------------------------------------------------------- fused step
STEP_CASES = [("full", p, r, False) for p in ("simt", "bf16x3", "bf16") for r in (0, -1) if not (p == "simt" and r)] \
    + [("large", p, r, False) for p in ("bf16x3", "bf16") for r in (0, -1)] + [("large", "bf16", 0, True)]


@pytest.mark.parametrize("which,path,records,grid_bf16", STEP_CASES)
def test_workload_fused_step(neat, oracle, request, which, path, records, grid_bf16):
    """One fused step on the workload slice against the f64 oracle: counts
    bit-exact, projection, loss, grid and decoder gradients and the Adam
    update within the path's bounds; records = -1 makes the backward
    recompute placement and gather instead of reading the forward's records;
    grid_bf16 gathers from the BF16 grid copy the large configuration trains
    with."""
    c = _case(request, which)
    _, tol_p, tol_g, tol_w = P.PATHS[path]
    tr = P._trainer(c, path, record_samples_per_ray=records, grid_bf16=grid_bf16)
    pred = torch.zeros(c.R, device="cuda")
    loss = tr.step(P._dev(c.uv), P._dev(c.img), P._dev(c.target), prediction=pred)
    torch.cuda.synchronize()
    tr.check_status()
    _, _, s, seg, rows, ref = _oracle(oracle, c)
    cnt = tr.counters.cpu().numpy()
    assert cnt[0] == seg["n"].shape[0] and cnt[1] == s["ray_t"].shape[0] and cnt[2] == seg["ray_nseg"].max()
    rows_t = torch.from_numpy(rows).cuda()
    g_all = tr.grad_reference_layout(tr.grid_m)
    g_used = g_all.index_select(0, rows_t).cpu().numpy().astype(np.float64) / 0.1  # m = (1 - b1) g
    p_all = tr.grid_reference_layout()
    p_used = p_all.index_select(0, rows_t).cpu().numpy()
    untouched = torch.ones(c.A, dtype=torch.bool, device="cuda")
    untouched[rows_t] = False
    assert float(g_all[untouched].abs().max()) == 0.0
    assert torch.equal(p_all[untouched].cpu(), torch.from_numpy(c.grid)[untouched.cpu()])
    err = dict(pred=P._rel2(pred.cpu().numpy(), ref["pred"]),
               loss=abs(float(loss.item()) - ref["loss"]) / ref["loss"],
               dec=P._rel2(tr.decoder_grad.cpu().numpy(), ref["grad_dec"]), grid=P._rel2(g_used, ref["grad_grid"]),
               pgrid=P._rel2(p_used, ref["grid"]), pdec=P._rel2(tr.decoder.cpu().numpy(), ref["dec"]))
    print(which, path, records, grid_bf16, f"{cnt[1]} samples, {rows.size} of {c.A} rows",
          {k: f"{v:.2e}" for k, v in err.items()})
    assert err["pred"] < tol_p and err["loss"] <= tol_p
    assert err["dec"] < tol_g and err["grid"] < tol_g
    assert err["pgrid"] < tol_w and err["pdec"] < tol_w


@pytest.mark.parametrize("which", ["full", "large"])
@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
@pytest.mark.parametrize("counts", [False, True])
def test_workload_proposal_sampling(neat, oracle, request, which, path, counts):
    """The learned proposal at the measured 12-sample budget on the workload
    slice: sample count bit-exact and projection within the path's bound of
    the f64 oracle that places the same samples from the same parameters.
    With counts, the count head sets each segment's count (count_eps 0.2,
    count_min 2); a segment within 1e-4 of a rounding boundary may round either
    way in f32, and its ray is set aside."""
    c = _case(request, which)
    eps, nmin = (0.2, 2) if counts else (0.0, 2)
    tr = P._prop_trainer(c, path, proposal_budget=12, proposal_count_eps=eps, proposal_count_min=nmin)
    params = P._random_proposal(tr)
    pred = tr.project(P._dev(c.uv), P._dev(c.img), use_proposal=True)
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    segs = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 12)
    f = oracle.proposal_features(o, d, segs, T.node_position_min, T.node_position_max,
                                 tr.prop_node_desc.cpu().numpy(), T.node_active_prefix_sum)
    Pt = torch.from_numpy(params)
    p = oracle.proposal_probs_f64(torch, Pt, f, tr.prop_struct.mix).numpy()
    cdf = np.cumsum(p, 1)
    cdf[:, -1] = 1.0
    n, x = oracle.proposal_counts(oracle.proposal_head_f64(torch, Pt, f).numpy(), segs["n"], eps, nmin)
    amb = (np.abs(x - np.round(x)) < 1e-4) & (x > nmin) & (x < segs["n"])
    s = oracle.proposal_samples(o, d, dict(segs, n=n), cdf, False, n_key=segs["n"])
    rows, grid_c, prefix = _compact(c, s)
    ref = oracle.image_f64(s, torch.from_numpy(grid_c.astype(np.float64)), torch.from_numpy(c.dec.astype(np.float64)),
                           T.node_position_min, T.node_position_max, prefix, c.R).numpy()
    keep = np.ones(c.R, bool)
    keep[segs["ray"][amb]] = False
    total = int(tr.counters[1].item())
    assert abs(total - s["weight"].shape[0]) <= int(amb.sum())
    if counts:
        assert total < 0.9 * int(segs["n"].sum())
    else:
        assert total == s["weight"].shape[0]
    err = P._rel2(pred.cpu().numpy()[keep], ref[keep])
    print(which, path, "counts" if counts else "", "12-sample proposal projection rel err", err, total, "samples of",
          int(segs["n"].sum()), "at the budget; ambiguous segments", int(amb.sum()))
    assert err < P.PATHS[path][1]


@pytest.mark.parametrize("path", ["bf16x3", "bf16"])
def test_large_workload_dda_hits_equal_the_octree_walk(neat, large_case, path):
    """At depth 5 the step finds each ray's hits by a DDA over the finest cells
    (the trainer's default); with the cell map off it walks the octree level by
    level.  On the large workload slice both give the same counters
    (segments, samples, largest hit count) and the same projection up to the
    rounding of a segment's two tile partials (the order of segments inside a
    node bucket comes from atomics, so where a tile boundary cuts a segment
    varies from call to call), with jitter (the step) and without (project)."""
    c = large_case
    a = P._trainer(c, path)
    b = P._trainer(c, path, cell_map=False)
    assert a.desc.cell_node and not b.desc.cell_node
    uv, img, tgt = P._dev(c.uv), P._dev(c.img), P._dev(c.target)
    out = []
    for tr in (a, b):
        pred = torch.zeros(c.R, device="cuda")
        loss = tr.step(uv, img, tgt, prediction=pred)
        proj = tr.project(uv, img)
        torch.cuda.synchronize()
        tr.check_status()
        out.append((tr.counters.cpu().numpy().copy(), float(loss.item()), pred.cpu().numpy(), proj.cpu().numpy()))
    print(path, "DDA", out[0][0][:3], "walk", out[1][0][:3])
    np.testing.assert_array_equal(out[0][0][:3], out[1][0][:3])
    assert abs(out[0][1] - out[1][1]) <= 1e-6 * abs(out[1][1])
    tol = 3e-7 if path == "bf16x3" else 1e-3
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=tol, atol=0)
    np.testing.assert_allclose(out[0][3], out[1][3], rtol=tol, atol=0)


# ---------------------------------------------------------------- gradient check
@pytest.mark.parametrize("path,bar", [("bf16x3", 1e-4), ("bf16", 5e-2)])
def test_large_workload_finite_differences(neat, oracle, large_case, path, bar):
    """The large configuration's gradient check: the fused step's analytic
    gradients on 1000 random parameters of its model (C = 16, G = 17, depth-5
    octree) -- 900 grid entries the slice touches and 100 decoder weights --
    against central differences (eps 1e-4) of the f64 loss on the same samples
    (256 rays of the workload).  Bars: 1e-4 on the FP32-accurate path, 5e-2 on
    the BF16 path the configuration trains with."""
    full = large_case
    c = Case()
    c.__dict__.update({k: v for k, v in full.__dict__.items() if not k.startswith("_")})
    c.R = 256
    c.uv, c.img, c.target = full.uv[:256], full.img[:256], full.target[:256]
    tr = P._trainer(c, path)
    tr.step(P._dev(c.uv), P._dev(c.img), P._dev(c.target))
    torch.cuda.synchronize()
    tr.check_status()
    T = c.tree
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True,
                              seed=99, step=1)
    rows, grid_c, prefix = _compact(c, s)
    g_grid = tr.grad_reference_layout(tr.grid_m).index_select(0, torch.from_numpy(rows).cuda()).cpu().numpy()
    g_grid = g_grid.astype(np.float64) / 0.1  # m = (1 - b1) g
    g_dec = tr.decoder_grad.cpu().numpy().astype(np.float64)

    # f64 loss with per-row caching: a grid entry moves only the samples of its row
    tg = torch.from_numpy(c.target.astype(np.float64))
    nmin = torch.from_numpy(T.node_position_min).double()[torch.from_numpy(s["node_id"])]
    nmax = torch.from_numpy(T.node_position_max).double()[torch.from_numpy(s["node_id"])]
    local = (torch.from_numpy(s["coords"]).double() - nmin) / (nmax - nmin) * 2 - 1
    row_of = torch.from_numpy(prefix[s["node_id"]])
    w = torch.from_numpy(s["weight"]).double()
    ray = torch.from_numpy(s["ray_index"])
    G64 = torch.from_numpy(grid_c.astype(np.float64))
    D64 = torch.from_numpy(c.dec.astype(np.float64))

    def dens(grid, dec, sel=None):
        if sel is None:
            f = oracle._trilinear_f64(torch, grid, row_of, local)
        else:
            f = oracle._trilinear_f64(torch, grid, row_of[sel], local[sel])
        return oracle.decoder_f64(torch, f, dec, c.C, 2.0)

    base_val = dens(G64, D64) * w
    base_pred = torch.zeros(c.R, dtype=torch.float64).index_add(0, ray, base_val)

    def loss_full(dec):
        pred = torch.zeros(c.R, dtype=torch.float64).index_add(0, ray, dens(G64, dec) * w)
        return float(((pred - tg) ** 2).mean())

    by_row = {}

    def loss_row(r):
        sel = by_row.setdefault(r, torch.nonzero(row_of == r)[:, 0])
        pred = base_pred.index_add(0, ray[sel], dens(G64, D64, sel) * w[sel] - base_val[sel])
        return float(((pred - tg) ** 2).mean())

    rng = np.random.default_rng(12)
    touched = np.flatnonzero(np.abs(g_grid) > 1e-12 * np.abs(g_grid).max())
    gi = rng.choice(touched, 900, replace=False)
    di = rng.choice(D64.numel(), 100, replace=False)
    eps = 1e-4
    fd, an = [], []
    per_row = grid_c[0].size
    for k in gi:
        r = int(k // per_row)
        flat = G64.view(-1)
        v = float(flat[k])
        flat[k] = v + eps
        lp = loss_row(r)
        flat[k] = v - eps
        lm = loss_row(r)
        flat[k] = v
        fd.append((lp - lm) / (2 * eps))
        an.append(g_grid.flat[k])
    for k in di:
        v = float(D64[k])
        D64[k] = v + eps
        lp = loss_full(D64)
        D64[k] = v - eps
        lm = loss_full(D64)
        D64[k] = v
        fd.append((lp - lm) / (2 * eps))
        an.append(g_dec[k])
    err = P._rel2(np.array(an), np.array(fd))
    print(path, f"finite differences vs analytic, 1000 params of the large model ({s['ray_t'].shape[0]} samples):",
          err)
    assert err < bar


# ---------------------------------------------------------------- hit limit
def test_more_than_256_hits_on_one_ray_is_flagged(neat, oracle):
    """A depth-7 octree whose active nodes lie along one diagonal ray: with
    256 of them the ray's SampleList matches the oracle bit for bit; with 257
    the sampler raises NEAT_ERR_TOO_MANY_HITS (the reference's kernel keeps 256
    intersections in shared memory and writes past them,
    src/structure/HyperTree.cu:220,281) and the oracle refuses the ray too."""
    from neat_b200 import _lib
    from neat_b200.api import CreateSamplesForRays, RayList
    from neat_b200.tree import HyperTreeBase
    T = HyperTreeBase(3, 7)
    o = np.array([[-1.5, -1.4989, -1.4977]], np.float32)
    d = np.array([[1.0, 1.0, 1.0]], np.float64)
    d = (d / np.linalg.norm(d)).astype(np.float32)
    lvl = np.nonzero(T.node_depth == 7)[0]
    hit, t0, t1 = oracle.intersect_boxes(T.node_position_min[lvl], T.node_position_max[lvl],
                                         np.repeat(o, lvl.size, 0), np.repeat(d, lvl.size, 0))
    keep = hit & ((t1 - t0).astype(np.float64) >= 1e-5)
    ids, tmin = lvl[keep], t0[keep]
    order = np.lexsort((ids, tmin))
    assert ids.size > 300  # a generic diagonal crosses ~3 * 128 cells
    for n, ok in ((256, True), (257, False)):
        T.SetActiveNodes(np.sort(ids[order[:n]]))
        rays = RayList(P._dev(o), P._dev(d))
        if ok:
            s = CreateSamplesForRays(T, rays, 4, False)
            ref = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 4, False)
            np.testing.assert_array_equal(s.node_id.cpu().numpy(), ref["node_id"])
            np.testing.assert_array_equal(s.ray_t.cpu().numpy(), ref["ray_t"])
            assert np.unique(s.node_id.cpu().numpy()).size == 256
        else:
            with pytest.raises(_lib.NeatError) as e:
                CreateSamplesForRays(T, rays, 4, False)
            assert e.value.status & _lib.NEAT_ERR_TOO_MANY_HITS
            with pytest.raises(RuntimeError):
                oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, 4, False)
