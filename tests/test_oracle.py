"""Pins of the CPU oracle (no GPU): known-answer tests and independent
restatements.  The reference ships no tests or golden vectors; the pins are
(a) the equivalence the reference documents between IndirectGridSample3D and
grid_sample(border, align_corners) (src/modules/IndirectGridSample3D.cu:30-40),
(b) published Philox4x32-10 known answers, (c) hand-derived slab-test and
sampling cases, (d) committed golden fixtures (tests/golden)."""
import math
import os

import numpy as np
import pytest
import torch

from tests.cases import cfg1_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# --------------------------------------------------------------------------
# Philox (Random123 kat_vectors, philox4x32_10)
# --------------------------------------------------------------------------
@pytest.mark.parametrize("seed,ctr,expect", [
    (0, (0, 0, 0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    (0xffffffffffffffff, (0xffffffff,) * 4, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    (0x299f31d0a4093822, (0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(oracle, seed, ctr, expect):
    assert tuple(int(v) for v in oracle.philox(seed, *ctr)) == expect


def test_uniform_range(oracle):
    u = np.array([oracle.uniform(3, i, 7, 1, 0x4a495454) for i in range(2000)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.03


# --------------------------------------------------------------------------
# IndirectGridSample3D
# --------------------------------------------------------------------------
def _grid_sample_ref(grid, idx, uv):
    g = torch.from_numpy(grid)[torch.from_numpy(idx)]
    p = torch.from_numpy(uv)[:, None, None, None, :]
    return torch.nn.functional.grid_sample(g, p, mode="bilinear", padding_mode="border", align_corners=True)


def test_igs_forward_equals_grid_sample(oracle):
    rng = np.random.default_rng(0)
    grid = rng.uniform(-1, 1, (6, 4, 11, 9, 7)).astype(np.float32)
    S = 3000
    idx = rng.integers(0, 6, S)
    uv = rng.uniform(-1, 1, (S, 3)).astype(np.float32)
    uv[:10] = np.array([[-1, -1, -1], [1, 1, 1], [1, -1, 1], [-1, 1, -1], [0, 0, 0], [1, 0, -1], [-1, 0, 1],
                        [0.5, -0.5, 1], [1, 1, -1], [-1, -1, 1]], np.float32)
    out = oracle.igs_forward(grid, idx, uv)
    ref = _grid_sample_ref(grid, idx, uv)[:, :, 0, 0, 0].numpy()
    np.testing.assert_allclose(out, ref, rtol=0, atol=4e-7)


def test_igs_backward_equals_grid_sample_autograd(oracle):
    rng = np.random.default_rng(1)
    grid = rng.uniform(-1, 1, (3, 2, 5, 6, 7)).astype(np.float32)
    S = 400
    idx = rng.integers(0, 3, S)
    uv = rng.uniform(-0.999, 0.999, (S, 3)).astype(np.float32)
    go = rng.normal(size=(S, 2)).astype(np.float32)
    gg, gu = oracle.igs_backward(grid, idx, uv, go)
    g = torch.from_numpy(grid).double().requires_grad_(True)
    p = torch.from_numpy(uv).double().requires_grad_(True)
    out = torch.nn.functional.grid_sample(g[torch.from_numpy(idx)], p[:, None, None, None, :], mode="bilinear",
                                          padding_mode="border", align_corners=True)[:, :, 0, 0, 0]
    (out * torch.from_numpy(go).double()).sum().backward()
    np.testing.assert_allclose(gg, g.grad.numpy(), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(gu, p.grad.numpy(), rtol=1e-4, atol=1e-5)


def test_igs_out_of_range_is_index_clamped(oracle):
    """Weights come from unclamped corners, indices are clamped (the
    reference's border-by-clamp): at uv = 1.5 on a 3-wide axis the x corners
    are 3 and 4, both clamped to 2, weights (-0.5, 1.5) sum to 1 -> value of
    the border cell."""
    grid = np.arange(27, dtype=np.float32).reshape(1, 1, 3, 3, 3)
    out = oracle.igs_forward(grid, np.array([0]), np.array([[1.5, -1, -1]], np.float32))
    assert out[0, 0] == pytest.approx(2.0)


# --------------------------------------------------------------------------
# IntersectBoxRayPrecise known answers
# --------------------------------------------------------------------------
UNIT = (np.array([-1, -1, -1], np.float32), np.array([1, 1, 1], np.float32))


def test_slab_axis_ray(oracle):
    hit, t0, t1 = oracle.intersect_box(*UNIT, [-3, 0.25, 0.5], [1, 0, 0])
    assert hit and t0 == 2.0 and t1 == 4.0


def test_slab_parallel_outside_and_on_max_face(oracle):
    assert not oracle.intersect_box(*UNIT, [-3, 1.5, 0], [1, 0, 0])[0]
    # o == max on a parallel axis is outside (o >= max)
    assert not oracle.intersect_box(*UNIT, [-3, 1.0, 0], [1, 0, 0])[0]
    # o == min on a parallel axis is inside
    assert oracle.intersect_box(*UNIT, [-3, -1.0, 0], [1, 0, 0])[0]


def test_slab_behind_origin_and_inside(oracle):
    assert not oracle.intersect_box(*UNIT, [3, 0, 0], [1, 0, 0])[0]
    hit, t0, t1 = oracle.intersect_box(*UNIT, [0, 0, 0], [1, 0, 0])
    assert hit and t0 == -1.0 and t1 == 1.0


def test_slab_corner_graze(oracle):
    d = np.array([1, 1, 0], np.float32) / np.float32(math.sqrt(2))
    hit, t0, t1 = oracle.intersect_box(np.array([0, 0, 0], np.float32), np.array([1, 1, 1], np.float32),
                                       [-1, 0, 0.5], d)
    # passes exactly through the edge x=0, y=1: tmin == tmax
    assert hit and t0 == t1


def test_sample_count_rule(oracle):
    """n = iCeil(((tmax - tmin) / diag) * M) and the 1e-5 skip
    (src/structure/HyperTree.cu:274-291)."""
    pmin = np.array([[0, 0, 0]], np.float32)
    pmax = np.array([[0.5, 0.5, 0.5]], np.float32)
    diag = np.float32(math.sqrt(0.75))
    o = np.array([[-1, 0.25, 0.25]], np.float32)
    d = np.array([[1, 0, 0]], np.float32)
    s = oracle.create_samples(o, d, np.array([0]), pmin, pmax, 16, False)
    n = len(s["ray_t"])
    assert n == math.ceil(float(np.float32(np.float32(0.5) / diag) * np.float32(16)))
    # a 5e-6 sliver is skipped
    o2 = np.array([[-1, 0.25, 0.4999975]], np.float32)
    d2 = np.array([[0, 0, 1]], np.float32)
    s2 = oracle.create_samples(np.array([[0.25, 0.25, -1]], np.float32), d2, np.array([0]),
                               np.array([[0, 0, 0]], np.float32), np.array([[0.5, 0.5, 0.000005]], np.float32), 16,
                               False)
    assert len(s2["ray_t"]) == 0


# --------------------------------------------------------------------------
# Octree / rays / samples
# --------------------------------------------------------------------------
def test_tree_numbering(oracle):
    t = oracle.tree_build(1)
    assert t["min"].shape == (9, 3)
    for i in range(8):
        bits = [(i >> k) & 1 for k in range(3)]
        np.testing.assert_array_equal(t["min"][1 + i], [0.0 if b else -1.0 for b in bits])
        np.testing.assert_array_equal(t["max"][1 + i], [1.0 if b else 0.0 for b in bits])
        assert t["parent"][1 + i] == 0 and t["children"][0, i] == 1 + i
    t4 = oracle.tree_build(4)
    assert t4["min"].shape[0] == 1 + 8 + 64 + 512 + 4096
    assert (t4["depth"] == 4).sum() == 4096


def test_center_ray_passes_origin(oracle):
    c = cfg1_case(R=4)
    w = h = 129
    from neat_b200 import scene as SC
    intr, rot, trans = SC.cone_beam_geometry(8, w, h)
    uv = np.array([[0.5, 0.5]] * 8, np.float32)
    o, d = oracle.make_rays(uv, np.arange(8), w, h, intr, rot, trans)
    for k in range(8):
        # closest approach of the central ray to the volume centre
        oo, dd = o[k].astype(np.float64), d[k].astype(np.float64)
        closest = oo - np.dot(oo, dd) * dd
        assert np.linalg.norm(closest) < 1e-6
        assert abs(np.linalg.norm(oo) - 3.0) < 1e-6


def test_samples_canonical_and_weights(oracle):
    c = cfg1_case(R=512, oracle=oracle)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True, seed=3)
    seg = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M)
    assert s["ray_t"].shape[0] == seg["n"].sum()
    # per ray: ray-major, local index contiguous, t increasing across segments
    ri = s["ray_index"]
    assert np.all(np.diff(ri) >= 0)
    for r in np.unique(ri)[:64]:
        m = ri == r
        np.testing.assert_array_equal(s["local_index"][m], np.arange(m.sum()))
        assert np.all(np.diff(s["ray_t"][m]) >= -1e-6)
    # weights of a segment sum to its length
    off = 0
    for k in range(min(len(seg["n"]), 500)):
        n = seg["n"][k]
        wsum = s["weight"][off:off + n].astype(np.float64).sum()
        assert abs(wsum - (seg["tmax"][k] - seg["tmin"][k])) < 1e-5
        off += n
    # jitter a=0.5 gives midpoints
    s0 = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, False)
    seg_t0 = seg["tmin"][0]
    step = np.float32(np.float32(seg["tmax"][0] - seg["tmin"][0]) / np.float32(seg["n"][0]))
    assert s0["ray_t"][0] == np.float32(np.float32(seg_t0 * np.float32(0.5)) +
                                        np.float32(np.float32(seg_t0 + step) * np.float32(0.5)))


def test_projector_matches_numeric_integral(oracle):
    from neat_b200 import scene as SC
    objs = SC.ellipsoid_phantom(4, 3, seed=5)
    objs[-1, 0:3] = objs[0, 0:3]  # put a void inside an ellipsoid
    rng = np.random.default_rng(2)
    for _ in range(5):
        o = np.array([0.1, -3.0, 0.05]) + rng.uniform(-0.2, 0.2, 3)
        d = np.array([0.0, 1.0, 0.0]) + rng.uniform(-0.1, 0.1, 3)
        d /= np.linalg.norm(d)
        t = np.linspace(1.0, 5.0, 40001)
        dens = oracle.phantom_density(objs, o[None, :] + t[:, None] * d[None, :])
        num = np.trapezoid(dens, t)
        ana = oracle.phantom_line(objs, o, d)
        assert abs(num - ana) < 2e-3 * max(1.0, ana)


def test_porous_projector_matches_numeric_integral(oracle):
    """Cylinder (additive) holding override spheres of their own density: the
    analytic chord sums against the trapezoid rule over the point density,
    for rays across the axis, along it (A = 0 in the radial quadratic) and in
    a plane of constant z (no slab crossing)."""
    from neat_b200 import scene as SC
    objs = SC.porous_phantom(60, seed=4, radius=(0.05, 0.12), cylinder_radius=0.6, cylinder_half_height=0.5)
    assert objs[0, 16] == 2 and np.all(objs[1:, 16] == 1) and np.all(objs[1:, 15] >= 0.2)
    # no two spheres overlap, each lies inside the cylinder
    c, r = objs[1:, 0:3], objs[1:, 3]
    dist = np.linalg.norm(c[:, None] - c[None], axis=2) + np.eye(len(r)) * 10
    assert np.all(dist >= r[:, None] + r[None, :])
    assert np.all(np.hypot(c[:, 0], c[:, 1]) + r <= 0.6) and np.all(np.abs(c[:, 2]) + r <= 0.5)
    rng = np.random.default_rng(8)
    rays = []
    for _ in range(6):
        o = np.array([0.0, -3.0, 0.0]) + rng.uniform(-0.3, 0.3, 3)
        d = np.array([0.0, 1.0, 0.0]) + rng.uniform(-0.15, 0.15, 3)
        rays.append((o, d / np.linalg.norm(d)))
    rays.append((np.array([0.1, 0.2, -3.0]), np.array([0.0, 0.0, 1.0])))   # along the axis
    rays.append((np.array([0.05, -3.0, 0.3]), np.array([0.0, 1.0, 0.0])))  # constant z inside the slab
    rays.append((np.array([0.05, -3.0, 0.7]), np.array([0.0, 1.0, 0.0])))  # constant z above it
    for o, d in rays:
        t = np.linspace(1.0, 5.0, 200001)
        dens = oracle.phantom_density(objs, o[None, :] + t[:, None] * d[None, :])
        num = np.trapezoid(dens, t)
        ana = oracle.phantom_line(objs, o, d)
        assert abs(num - ana) < 2e-4 * max(1.0, ana), (o, d, num, ana)
    # density: inside a sphere its own, elsewhere in the cylinder 0.3, outside 0
    grid = rng.uniform(-0.5, 0.5, (2000, 3))
    free = grid[np.all(np.linalg.norm(grid[:, None] - c[None], axis=2) > r[None, :], axis=1)
                & (np.hypot(grid[:, 0], grid[:, 1]) < 0.6)][0]
    rho = oracle.phantom_density(objs, np.stack([objs[1, 0:3], free, [0.9, 0.0, 0.0]]))
    assert rho[0] == objs[1, 15] and rho[1] == 0.3 and rho[2] == 0.0


def test_step_f64_gradient_matches_finite_differences(oracle):
    c = cfg1_case(R=64, oracle=oracle, n_angles=4, w=32, h=32)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True, seed=1)
    base = oracle.step_f64(s, c.grid, c.dec, c.target, T.node_position_min, T.node_position_max,
                           T.node_active_prefix_sum)
    rng = np.random.default_rng(0)
    flat_idx = np.nonzero(np.abs(base["grad_grid"].reshape(-1)) > 1e-6)[0]
    for i in rng.choice(flat_idx, 5, replace=False):
        for arr, gname in ((c.grid, "grad_grid"),):
            e = 1e-6
            gp = arr.astype(np.float64).copy().reshape(-1)
            gm = gp.copy()
            gp[i] += e
            gm[i] -= e
            lp = oracle.step_f64(s, gp.reshape(arr.shape), c.dec, c.target, T.node_position_min, T.node_position_max,
                                 T.node_active_prefix_sum)["loss"]
            lm = oracle.step_f64(s, gm.reshape(arr.shape), c.dec, c.target, T.node_position_min, T.node_position_max,
                                 T.node_active_prefix_sum)["loss"]
            fd = (lp - lm) / (2 * e)
            assert abs(fd - base[gname].reshape(-1)[i]) < 1e-6 * max(1.0, abs(fd)) + 1e-9


def test_igs_golden_from_reference_cpu(oracle):
    """IGS forward/backward against the reference's own CPU implementation
    (IndirectGridSample3D.cu:27-429, compiled from its source by oracle/Makefile
    `ref`; fixture made by tests/golden/make_golden.py)."""
    z = np.load(os.path.join(GOLDEN, "igs_reference_cpu.npz"))
    out = oracle.igs_forward(z["grid"], z["index"], z["uv"])
    np.testing.assert_array_equal(out, z["out"])  # same fma order: bit-exact
    gg, gu = oracle.igs_backward(z["grid"], z["index"], z["uv"], z["grad_out"])
    np.testing.assert_array_equal(gu, z["grad_uv"])
    # grad_grid sums the same terms; the reference build contracts += w*go
    np.testing.assert_allclose(gg, z["grad_grid"], rtol=0, atol=1e-6)


def test_slab_golden_from_reference(oracle):
    """IntersectBoxRayPrecise of the oracle against the reference's own
    (src/structure/HyperTree.h:41-83): identical hit decisions and float
    tmin/tmax on 12000 aimed, axis-parallel and inside-the-box pairs."""
    z = np.load(os.path.join(GOLDEN, "slab_reference.npz"))
    t = oracle.tree_build(int(z["depth"]))
    hit, t0, t1 = oracle.intersect_boxes(t["min"][z["node"]], t["max"][z["node"]], z["origin"], z["direction"])
    np.testing.assert_array_equal(hit, z["hit"].astype(bool))
    np.testing.assert_array_equal(t0[hit], z["tmin"][hit])
    np.testing.assert_array_equal(t1[hit], z["tmax"][hit])


REF_SO = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libneat_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built (make -C oracle ref)")
def test_oracle_matches_reference_cpu_live(oracle):
    """Fresh random inputs through the reference's CPU IGS and the oracle."""
    import ctypes
    lib = ctypes.CDLL(REF_SO)
    P, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
    lib.ref_igs_forward.argtypes = [P, L, I, I, I, I, P, P, L, P]
    rng = np.random.default_rng(77)
    for (N, C, G) in ((3, 4, 11), (2, 8, 17), (4, 16, 5)):
        grid = rng.uniform(-1, 1, (N, C, G, G, G)).astype(np.float32)
        S = 2000
        idx = rng.integers(0, N, S).astype(np.int64)
        uv = rng.uniform(-1, 1, (S, 3)).astype(np.float32)
        out = np.zeros((S, C), np.float32)
        lib.ref_igs_forward(grid.ctypes.data_as(P), N, C, G, G, G, idx.ctypes.data_as(P), uv.ctypes.data_as(P), S,
                            out.ctypes.data_as(P))
        np.testing.assert_array_equal(oracle.igs_forward(grid, idx, uv), out)


def test_volume_descent_face_ties(oracle):
    """ActiveNodeIdForGlobalPosition semantics: closed boxes, first child in
    order 0..7 wins a shared face, an inactive leaf gives -1."""
    from neat_b200.tree import HyperTreeBase
    t = HyperTreeBase(3, 2)
    t.SetActiveNodes([2] + list(range(9, 17)))  # root child 1 active; child 0 refined; others inactive leaves' parents
    p = np.array([[0.0, -0.5, -0.5],    # face x = 0 between child 0 (refined) and child 1 -> child 0's leaf
                  [0.5, -0.5, -0.5],    # inside child 1 (active)
                  [-0.5, 0.5, -0.5],    # child 2: inactive with no active child -> its leaf 25.. inactive -> -1
                  [-1.0, -1.0, -1.0]],  # corner: child 0 -> leaf 9
                 np.float32)
    n = oracle.active_node_for_positions(p, t.node_active, t.node_position_min, t.node_position_max, 2)
    assert n[1] == 2 and n[2] == -1 and n[3] == 9
    assert 9 <= n[0] <= 16 and (t.node_position_max[n[0]][0] == 0.0)
    pos = oracle.volume_positions(3, 2, 2)
    np.testing.assert_array_equal(pos[:4], np.array([[-1, -1, -1], [0, -1, -1], [1, -1, -1], [-1, 1, -1]], np.float32))


def test_proposal_inverse_cdf(oracle):
    """Inverse of the piecewise-linear proposal CDF: uniform bins give the
    identity, a bin holding 40% of the mass is sampled 40% of the time."""
    u = np.linspace(0, 0.999, 50)
    uni = np.tile(np.arange(1, 9) / 8.0, (50, 1))
    np.testing.assert_allclose(oracle.proposal_inverse(uni, u), u, atol=1e-12)
    c = np.tile(np.array([0.05, 0.1, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0]), (3, 1))
    s = oracle.proposal_inverse(c, np.array([0.1, 0.3, 0.5 - 1e-12]))
    np.testing.assert_allclose(s, [2 / 8, 2.5 / 8, 3 / 8], atol=1e-9)


def test_proposal_gradient_matches_finite_differences(oracle):
    """The f64 cross-entropy gradient of the proposal (the oracle the GPU
    training kernel is checked against) matches central differences."""
    import torch
    rng = np.random.default_rng(4)
    P = rng.normal(0, 0.3, oracle.PROP_TOTAL)
    f = rng.uniform(-1, 1, (40, 16)).astype(np.float32)
    f[:, 13:] = 0
    hist = rng.uniform(0, 1, (40, 8)) * (rng.uniform(0, 1, (40, 1)) > 0.2)
    a = rng.uniform(0, 0.3, 40) * (rng.uniform(0, 1, 40) > 0.2)
    a[3] = -1.0  # a segment without a count target
    loss, g, lh = oracle.proposal_grad_f64(P, f, hist, 0.1, a)
    trunk = rng.choice(oracle.PROP_TRUNK, 20, replace=False)
    head = oracle.PROP_TRUNK + rng.choice(oracle.PROP_TOTAL - oracle.PROP_TRUNK, 10, replace=False)
    for k in np.concatenate([trunk, head]):
        e = np.zeros_like(P)
        e[k] = 1e-6
        lp, _, hp = oracle.proposal_grad_f64(P + e, f, hist, 0.1, a)
        lm, _, hm = oracle.proposal_grad_f64(P - e, f, hist, 0.1, a)
        fd = (lp - lm) / 2e-6 if k < oracle.PROP_TRUNK else (hp - hm) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(g[k])


def test_proposal_counts_rule(oracle):
    """The count head's rule: n_ref where eps <= 0; else
    min(n_ref, max(min(nmin, n_ref), ceil(exp(v) / eps)))."""
    v = np.log(np.array([0.05, 0.25, 0.31, 10.0, 1e-9, 0.2]))
    n_ref = np.array([12, 12, 12, 12, 12, 1])
    n, x = oracle.proposal_counts(v, n_ref, 0.1, 2)
    np.testing.assert_array_equal(n, [2, 3, 4, 12, 2, 1])
    np.testing.assert_allclose(x[:3], [0.5, 2.5, 3.1])
    n0, _ = oracle.proposal_counts(v, n_ref, 0.0, 2)
    np.testing.assert_array_equal(n0, n_ref)


def test_pose_gradients_match_finite_differences(oracle):
    """The f64 pose / intrinsics gradient chain (the oracle of the GPU pose
    gradients) matches central differences of its own loss: rotation tangent,
    translation and intrinsics, with the samples (t, node, weight) held fixed as
    in the reference's autograd and the trilinear cells from the f64 positions.
    Steps are small enough (1e-7, 1e-6 pixels) that no sample changes cell."""
    c = cfg1_case(R=64, oracle=oracle, n_angles=4, w=32, h=32)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    T = c.tree
    s = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, True, seed=1)
    args = (s, c.uv, c.img, c.w, c.h)
    tail = (c.grid, c.dec, c.target, T.node_position_min, T.node_position_max, T.node_active_prefix_sum)
    g = oracle.pose_grads_f64(*args, c.intr, c.rot, c.trans, *tail, cells_from_coords=False)

    def loss(intr=c.intr, trans=c.trans, tangent=None):
        return float(oracle.pose_loss_f64(*args, intr, c.rot, trans, *tail, tangent=tangent,
                                          cells_from_coords=False)[0].detach())

    n_img = np.asarray(c.rot).reshape(-1, 4).shape[0]
    e = 1e-7
    for i in np.unique(c.img)[:3]:
        for k in range(3):
            tp = np.zeros((n_img, 3))
            tp[i, k] = e
            fd = (loss(tangent=tp) - loss(tangent=-tp)) / (2 * e)
            assert abs(fd - g["tangent"][i, k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
            trp = np.asarray(c.trans, np.float64).reshape(-1, 3).copy()
            trm = trp.copy()
            trp[i, k] += e
            trm[i, k] -= e
            fd = (loss(trans=trp) - loss(trans=trm)) / (2 * e)
            assert abs(fd - g["translation"][i, k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    for k in range(4):
        ip = np.asarray(c.intr, np.float64).reshape(-1).copy()
        im = ip.copy()
        ip[k] += 1e-6
        im[k] -= 1e-6
        fd = (loss(intr=ip) - loss(intr=im)) / 2e-6
        assert abs(fd - g["intrinsics"][k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    assert g["intrinsics"][4] == 0.0  # the skew does not enter Unproject


def test_quat_exp_mul_is_the_rotation_update(oracle):
    """quat_exp_mul_f64: exp of a rotation vector (axis * angle) times q, as a
    rotation matrix product (Rodrigues)."""
    rng = np.random.default_rng(2)
    q = rng.normal(size=(6, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w = rng.normal(size=(6, 3)) * 0.3
    w[0] = 0.0
    w[1] = 1e-12

    def mat(qq):
        x, y, z, s = qq
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - s * z), 2 * (x * z + s * y)],
                         [2 * (x * y + s * z), 1 - 2 * (x * x + z * z), 2 * (y * z - s * x)],
                         [2 * (x * z - s * y), 2 * (y * z + s * x), 1 - 2 * (x * x + y * y)]])

    out = oracle.quat_exp_mul_f64(w, q)
    for i in range(6):
        th = np.linalg.norm(w[i])
        K = np.array([[0, -w[i, 2], w[i, 1]], [w[i, 2], 0, -w[i, 0]], [-w[i, 1], w[i, 0], 0]])
        a = np.sin(th) / th if th > 0 else 1.0
        b = (1 - np.cos(th)) / th ** 2 if th > 1e-6 else 0.5
        np.testing.assert_allclose(mat(out[i]), (np.eye(3) + a * K + b * K @ K) @ mat(q[i]), rtol=0, atol=1e-12)
