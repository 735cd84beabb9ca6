"""Generate the golden fixtures from the reference's own CPU code.

Needs oracle/_ref/libneat_ref.so, built in the container that holds the
reference checkout (`make -C oracle ref`: it compiles the unmodified text of
IndirectGridSample3DForwardCPU/BackwardCPU, src/modules/IndirectGridSample3D.cu:19-429,
and IntersectBoxRayPrecise, src/structure/HyperTree.h:41-83).  Writes:

  igs_reference_cpu.npz   seeded grid / index / uv / grad_out and the reference
                          CPU forward output, grad_grid and grad_uv
  slab_reference.npz      ray-box pairs (node boxes of a depth-4 octree, rays of
                          the cone-beam camera aimed at the boxes, plus
                          axis-parallel, face-grazing and inside-the-box cases)
                          and the reference's (hit, tmin, tmax)

Run: python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

P, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int


def _ptr(a):
    return a.ctypes.data_as(P)


def load_ref():
    path = os.path.join(ROOT, "oracle", "_ref", "libneat_ref.so")
    lib = ctypes.CDLL(path)
    lib.ref_igs_forward.argtypes = [P, L, I, I, I, I, P, P, L, P]
    lib.ref_igs_backward.argtypes = [P, L, I, I, I, I, P, P, L, P, P, P]
    lib.ref_intersect_box.argtypes = [P] * 6
    lib.ref_intersect_box.restype = I
    return lib


def igs_fixture(lib):
    rng = np.random.default_rng(20221)
    N, C, Z, Y, X = 5, 4, 9, 7, 11
    grid = rng.uniform(-1, 1, (N, C, Z, Y, X)).astype(np.float32)
    S = 3000
    index = rng.integers(0, N, S).astype(np.int64)
    uv = rng.uniform(-1.05, 1.05, (S, 3)).astype(np.float32)
    uv[:12] = [[-1, -1, -1], [1, 1, 1], [1, -1, 1], [-1, 1, -1], [0, 0, 0], [1, 0, -1], [-1, 0, 1],
               [0.5, -0.5, 1], [1, 1, -1], [-1, -1, 1], [1.05, 0, 0], [0, -1.05, 0.5]]
    grad_out = rng.normal(size=(S, C)).astype(np.float32)
    out = np.zeros((S, C), np.float32)
    lib.ref_igs_forward(_ptr(grid), N, C, Z, Y, X, _ptr(index), _ptr(uv), S, _ptr(out))
    gg = np.zeros_like(grid)
    gu = np.zeros_like(uv)
    lib.ref_igs_backward(_ptr(grid), N, C, Z, Y, X, _ptr(index), _ptr(uv), S, _ptr(grad_out), _ptr(gg), _ptr(gu))
    return dict(grid=grid, index=index, uv=uv, grad_out=grad_out, out=out, grad_grid=gg, grad_uv=gu)


def slab_fixture(lib):
    from neat_b200 import scene as SC
    from oracle import oracle as O
    rng = np.random.default_rng(20222)
    t = O.tree_build(4)
    pmin, pmax = t["min"], t["max"]
    n_nodes = pmin.shape[0]
    intr, rot, trans = SC.cone_beam_geometry(16, 64, 64)
    boxes, origins, dirs = [], [], []
    for k in range(12000):
        nid = int(rng.integers(0, n_nodes))
        img = int(rng.integers(0, 16))
        o = trans[img].astype(np.float32)
        target = (pmin[nid] + (pmax[nid] - pmin[nid]) * rng.uniform(-0.2, 1.2, 3)).astype(np.float64)
        d = target - o
        kind = k % 6
        if kind == 4:  # axis-parallel rays, some exactly on a face plane
            o = pmin[nid].astype(np.float64) + (pmax[nid] - pmin[nid]) * rng.choice([0.0, 0.5, 1.0], 3)
            ax = int(rng.integers(0, 3))
            o[ax] -= 2.0
            d = np.zeros(3)
            d[ax] = 1.0
            o = o.astype(np.float32)
        elif kind == 5:  # origin inside the box
            o = (pmin[nid] + (pmax[nid] - pmin[nid]) * rng.uniform(0.1, 0.9, 3)).astype(np.float32)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        boxes.append(nid)
        origins.append(o)
        dirs.append(d)
    boxes = np.array(boxes, np.int64)
    origins = np.array(origins, np.float32)
    dirs = np.array(dirs, np.float32)
    hit = np.zeros(len(boxes), np.int32)
    tmin = np.zeros(len(boxes), np.float32)
    tmax = np.zeros(len(boxes), np.float32)
    for i in range(len(boxes)):
        a0 = np.ascontiguousarray(pmin[boxes[i]])
        a1 = np.ascontiguousarray(pmax[boxes[i]])
        o = np.ascontiguousarray(origins[i])
        d = np.ascontiguousarray(dirs[i])
        t0 = np.zeros(1, np.float32)
        t1 = np.zeros(1, np.float32)
        hit[i] = lib.ref_intersect_box(_ptr(a0), _ptr(a1), _ptr(o), _ptr(d), _ptr(t0), _ptr(t1))
        tmin[i], tmax[i] = t0[0], t1[0]
    return dict(node=boxes, origin=origins, direction=dirs, hit=hit, tmin=tmin, tmax=tmax, depth=np.int64(4))


if __name__ == "__main__":
    lib = load_ref()
    igs = igs_fixture(lib)
    np.savez_compressed(os.path.join(HERE, "igs_reference_cpu.npz"), **igs)
    slab = slab_fixture(lib)
    np.savez_compressed(os.path.join(HERE, "slab_reference.npz"), **slab)
    print("igs samples", igs["index"].shape[0], "slab pairs", slab["node"].shape[0], "hits", int(slab["hit"].sum()))
