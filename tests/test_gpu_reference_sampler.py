"""The ray sampler against the reference's own kernel.

ComputeRaySamples (src/structure/HyperTree.cu:206-391), compiled unmodified
for sm_100a with nvcc's defaults by `make -C oracle ref-sampler`
(oracle/_ref/libneat_ref_sampler.so, test infrastructure), is run on the same
rays and octree as this library's CreateSamplesForRays and the oracle's C
restatement; positions are recomputed from ray_t as the reference's
CreateSamplesForRays does with torch (HyperTree.cu:426-432).

The reference writes a ray's intersections in the order of a shared-memory
atomic (HyperTree.cu:281), so its SampleList is compared in canonical order:
per ray by (ray_t, node_id), local_index_in_ray renumbered by that order.  The
evaluation setting (a = 0.5, no jitter) makes the lists deterministic; the
jittered offsets come from torch::rand_like there and from Philox here.

Bar: bit-exact for the sample count, the largest count of one ray, and every
sample's ray, node, t, weight and position.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from tests.cases import cfg1_case, workload_case

pytestmark = pytest.mark.gpu

REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "libneat_ref_sampler.so")


@pytest.fixture(scope="module")
def ref_sampler(neat):
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libneat_ref_sampler.so is not built (make -C oracle ref-sampler)")
    lib = ctypes.CDLL(REF_SO)
    P, L, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    lib.ref_compute_ray_samples.argtypes = [P, P, L, P, L, P, P, L, P, I, L, P, P, P, P, P, P, P]
    lib.ref_compute_ray_samples.restype = I
    return lib


def _canonical(ray, t, node, w, coords):
    order = np.lexsort((node, t, ray))
    ray, t, node, w, coords = ray[order], t[order], node[order], w[order], coords[order]
    first = np.r_[0, np.flatnonzero(np.diff(ray)) + 1]
    local = np.arange(ray.size) - np.repeat(first, np.diff(np.r_[first, ray.size]))
    return dict(ray_index=ray, ray_t=t, node_id=node, weight=w, coords=coords, local_index=local)


def _reference(lib, oracle, c, o, d, M):
    """The reference kernel's SampleList, canonical order.  Its writes to the
    outputs and to its 256-entry shared hit arrays are unchecked, so: every
    ray must have at most 256 hits (checked with the oracle first, whose slab
    decisions are the same float operations), and the capacity is an upper
    bound that needs no agreement on the counts -- per ray at most
    min(A, 256) hits of at most M + 1 samples each (a segment is no longer
    than its box's diagonal, up to rounding)."""
    T = c.tree
    seg = oracle.ray_segments(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, M)
    assert seg["ray_nseg"].max() <= 256
    cap = o.shape[0] * min(T.NumActiveNodes(), 256) * (M + 1) + 1
    dev = torch.device("cuda")
    nmin, nmax = torch.from_numpy(T.node_position_min).to(dev), torch.from_numpy(T.node_position_max).to(dev)
    act = torch.from_numpy(T.active_node_ids).to(dev)
    od, dd = torch.from_numpy(np.ascontiguousarray(o)).to(dev), torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    R = od.shape[0]
    out = dict(coords=torch.empty((cap, 3), device=dev), weight=torch.empty(cap, device=dev),
               ray_t=torch.empty(cap, device=dev), ray_index=torch.empty(cap, dtype=torch.int64, device=dev),
               local_index=torch.empty(cap, dtype=torch.int64, device=dev),
               node_id=torch.empty(cap, dtype=torch.int64, device=dev))
    cnt = torch.zeros(2, dtype=torch.int32, device=dev)
    rc = lib.ref_compute_ray_samples(nmin.data_ptr(), nmax.data_ptr(), T.NumNodes(), act.data_ptr(), act.numel(),
                                     od.data_ptr(), dd.data_ptr(), R, None, M, cap, out["coords"].data_ptr(),
                                     out["weight"].data_ptr(), out["ray_t"].data_ptr(), out["ray_index"].data_ptr(),
                                     out["local_index"].data_ptr(), out["node_id"].data_ptr(), cnt.data_ptr())
    torch.cuda.synchronize()
    assert rc == 0
    S, mx = int(cnt[0]), int(cnt[1])
    assert S < cap
    ray = out["ray_index"][:S]
    t = out["ray_t"][:S]
    # CreateSamplesForRays recomputes the positions with torch (HyperTree.cu:426-432)
    pos = torch.index_select(od, 0, ray) + torch.index_select(dd, 0, ray) * t.unsqueeze(1)
    res = _canonical(ray.cpu().numpy(), t.cpu().numpy(), out["node_id"][:S].cpu().numpy(),
                     out["weight"][:S].cpu().numpy(), pos.cpu().numpy())
    res["max_per_ray"] = mx
    return res


def _compare(got, ref, what):
    for k in ("ray_index", "node_id", "local_index", "ray_t", "weight", "coords"):
        a, b = np.asarray(got[k]), np.asarray(ref[k])
        assert a.shape == b.shape, (what, k, a.shape, b.shape)
        bad = int(np.count_nonzero(a != b))
        assert bad == 0, f"{what}: {k} differs from the reference kernel in {bad} of {a.size} entries"


@pytest.mark.parametrize("which", ["cfg1", "adaptive", "full"])
def test_sampler_matches_the_reference_kernel(neat, oracle, ref_sampler, which):
    from neat_b200.api import CameraModel, CreateSamplesForRays, GetRays
    if which == "cfg1":
        c = cfg1_case(R=4096, oracle=oracle)
    elif which == "adaptive":
        c = cfg1_case(R=2048, seed=3, depth=4, G=9, M=16, oracle=oracle, adaptive=400)
    else:
        c = workload_case("full", R=2048, seed=41)
    o, d = oracle.make_rays(c.uv, c.img, c.w, c.h, c.intr, c.rot, c.trans)
    ref = _reference(ref_sampler, oracle, c, o, d, c.M)
    T = c.tree
    orc = oracle.create_samples(o, d, T.active_node_ids, T.node_position_min, T.node_position_max, c.M, False)
    assert orc["ray_t"].shape[0] == ref["ray_t"].shape[0] and orc["max_per_ray"] == ref["max_per_ray"]
    _compare(_canonical(orc["ray_index"], orc["ray_t"], orc["node_id"], orc["weight"], orc["coords"]), ref, "oracle")
    cam = CameraModel(c.w, c.h, c.intr, c.rot, c.trans)
    s = CreateSamplesForRays(T, GetRays(cam, torch.from_numpy(c.uv).cuda(), torch.from_numpy(c.img).cuda()), c.M,
                             False)
    assert s.max_samples_per_ray == ref["max_per_ray"]
    mine = dict(ray_index=s.ray_index.cpu().numpy(), node_id=s.node_id.cpu().numpy(),
                local_index=s.local_index_in_ray.cpu().numpy(), ray_t=s.ray_t.cpu().numpy(),
                weight=s.weight.cpu().numpy(), coords=s.global_coordinate.cpu().numpy())
    _compare(mine, ref, "CUDA sampler")  # already canonical: (tmin, node) segments, samples by j
    print(which, ref["ray_t"].shape[0], "samples bit-identical to the reference kernel")
