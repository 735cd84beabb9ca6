"""Oracle for the NeAT forward-projection training step -- TEST INFRASTRUCTURE.

Two layers:
* ctypes wrappers of oracle/libneat_oracle.so (the C restatement in
  neat_oracle.c: tree tables, rays, slab test, CreateSamplesForRays, IGS,
  synthetic projector), built by oracle/Makefile;
* step_f64: a float64 CPU restatement (torch f64 autograd) of
  ComputeImage -> MSE -> backward -> Adam on the oracle's SampleList:
    local coords       src/structure/HyperTree.cu:177-192
    IGS (trilinear)    src/modules/IndirectGridSample3D.cu:27-191
    FCBlock + softplus src/geometry/ImplicitNet.h:18-73, src/geometry/geometry.cpp:102-163
    integral           src/geometry/geometry.cpp:393-424 (index_add_)
    loss               samples/reconstruct.cpp:378-386 (mean of squares)
    Adam               src/geometry/geometry.h:66-88 (torch::optim::Adam)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.  The product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libneat_oracle.so")

_f = ctypes.c_float
_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_long
_p = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32

_SIGS = {
    "oracle_philox": (None, [_u64, _u32, _u32, _u32, _u32, _p]),
    "oracle_uniform": (_f, [_u64, _u32, _u32, _u32, _u32]),
    "oracle_tree_num_nodes": (_i, [_i]),
    "oracle_tree_build": (None, [_i, _p, _p, _p, _p, _p]),
    "oracle_make_rays": (None, [_i, _p, _p, _i, _i, _p, _p, _p, _p, _p]),
    "oracle_intersect_box": (_i, [_p, _p, _p, _p, _p, _p]),
    "oracle_intersect_boxes": (None, [_l, _p, _p, _p, _p, _p, _p, _p]),
    "oracle_node_diag": (_f, [_p, _p]),
    "oracle_create_samples": (_l, [_i, _p, _p, _i, _p, _p, _p, _i, _i, _u64, _u32, _l, _p, _p, _p, _p, _p, _p, _p,
                                   _p]),
    "oracle_ray_segments": (_l, [_i, _p, _p, _i, _p, _p, _p, _i, _l, _p, _p, _p, _p, _p, _p, _p]),
    "oracle_local_samples": (None, [_l, _p, _p, _p, _p, _p]),
    "oracle_igs_forward": (None, [_p, _l, _i, _i, _i, _i, _p, _p, _l, _p]),
    "oracle_igs_backward": (None, [_p, _l, _i, _i, _i, _i, _p, _p, _l, _p, _p, _p]),
    "oracle_phantom_line": (_d, [_p, _i, _p, _p]),
    "oracle_phantom_density": (_d, [_p, _i, _p]),
    "oracle_project": (None, [_p, _i, _i, _i, _i, _p, _p, _p, _p]),
    "oracle_project_pixels": (None, [_p, _i, _l, _p, _p, _p, _p, _p, _p, _p]),
    "oracle_phantom_density_batch": (None, [_p, _i, _l, _p, _p]),
}

_lib = None


def build():
    """Builds the oracle library and, where the reference checkout the
    Makefile's REF names is present, oracle/_ref (the reference's own CPU
    IGS; its GPU IGS kernels for sm_100a, timed by bench.py's comparison leg;
    its GPU ray sampler for sm_100a, which the tests compare against).
    Without that checkout the prebuilt oracle/_ref, if any, is kept."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if subprocess.run(["make", "-s", "-C", HERE, "-q", "ref-available"], capture_output=True).returncode == 0:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "ref-cuda"], check=True)
        subprocess.run(["make", "-s", "-C", HERE, "ref-sampler"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        for k, (r, a) in _SIGS.items():
            fn = getattr(L, k)
            fn.restype = r
            fn.argtypes = a
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# --------------------------------------------------------------------------
# wrappers
# --------------------------------------------------------------------------
def uniform(seed, c0, c1, c2, c3):
    return lib().oracle_uniform(seed, c0, c1, c2, c3)


def philox(seed, c0, c1, c2, c3):
    out = np.zeros(4, np.uint32)
    lib().oracle_philox(seed, c0, c1, c2, c3, _ptr(out))
    return out


def tree_build(max_depth):
    N = lib().oracle_tree_num_nodes(max_depth)
    pmin = np.zeros((N, 3), np.float32)
    pmax = np.zeros((N, 3), np.float32)
    depth = np.zeros(N, np.int32)
    parent = np.zeros(N, np.int32)
    children = np.zeros((N, 8), np.int32)
    lib().oracle_tree_build(max_depth, _ptr(pmin), _ptr(pmax), _ptr(depth), _ptr(parent), _ptr(children))
    return dict(min=pmin, max=pmax, depth=depth, parent=parent, children=children)


def make_rays(uv, image_id, w, h, intr, rot, trans):
    uv = _c(uv, np.float32)
    image_id = _c(image_id, np.int32)
    R = uv.shape[0]
    o = np.zeros((R, 3), np.float32)
    d = np.zeros((R, 3), np.float32)
    lib().oracle_make_rays(R, _ptr(uv), _ptr(image_id), w, h, _ptr(_c(intr, np.float64)), _ptr(_c(rot, np.float64)),
                           _ptr(_c(trans, np.float64)), _ptr(o), _ptr(d))
    return o, d


def intersect_box(pmin, pmax, o, d):
    pmin, pmax, o, d = (_c(x, np.float32) for x in (pmin, pmax, o, d))
    t0 = np.zeros(1, np.float32)
    t1 = np.zeros(1, np.float32)
    hit = lib().oracle_intersect_box(_ptr(pmin), _ptr(pmax), _ptr(o), _ptr(d), _ptr(t0), _ptr(t1))
    return bool(hit), float(t0[0]), float(t1[0])


def intersect_boxes(pmin, pmax, o, d):
    """Vectorised slab test over pairs: arrays [n,3] -> (hit, tmin, tmax)."""
    pmin, pmax, o, d = (_c(x, np.float32) for x in (pmin, pmax, o, d))
    n = pmin.shape[0]
    hit = np.zeros(n, np.int32)
    t0 = np.zeros(n, np.float32)
    t1 = np.zeros(n, np.float32)
    lib().oracle_intersect_boxes(n, _ptr(pmin), _ptr(pmax), _ptr(o), _ptr(d), _ptr(hit), _ptr(t0), _ptr(t1))
    return hit.astype(bool), t0, t1


def create_samples(o, d, active_ids, pmin, pmax, M, jitter, seed=0, step=1, cap=None):
    """Canonical SampleList of the rays; the arrays are sized to the exact
    sample count (a first call reports it when the estimate is short)."""
    o, d = _c(o, np.float32), _c(d, np.float32)
    act = _c(active_ids, np.int64)
    pmin, pmax = _c(pmin, np.float32), _c(pmax, np.float32)
    R = o.shape[0]
    cap = max(16, int(R * M * 4) if cap is None else int(cap))
    while True:
        out = dict(coords=np.empty((cap, 3), np.float32), ray_t=np.empty(cap, np.float32),
                   weight=np.empty(cap, np.float32), ray_index=np.empty(cap, np.int64),
                   local_index=np.empty(cap, np.int64), node_id=np.empty(cap, np.int64))
        mx = np.zeros(1, np.int32)
        need = np.zeros(1, np.int64)
        S = lib().oracle_create_samples(R, _ptr(o), _ptr(d), act.shape[0], _ptr(act), _ptr(pmin), _ptr(pmax), M,
                                        int(jitter), seed, step, cap, _ptr(out["coords"]), _ptr(out["ray_t"]),
                                        _ptr(out["weight"]), _ptr(out["ray_index"]), _ptr(out["local_index"]),
                                        _ptr(out["node_id"]), _ptr(mx), _ptr(need))
        if S == -1 and need[0] > cap:
            cap = int(need[0])
            continue
        if S < 0:
            raise RuntimeError(f"oracle_create_samples failed ({S})")
        res = {k: v[:S] for k, v in out.items()}
        res["max_per_ray"] = int(mx[0])
        return res


def ray_segments(o, d, active_ids, pmin, pmax, M, cap=None):
    o, d = _c(o, np.float32), _c(d, np.float32)
    act = _c(active_ids, np.int64)
    pmin, pmax = _c(pmin, np.float32), _c(pmax, np.float32)
    R = o.shape[0]
    cap = cap or R * 256
    seg = {k: np.zeros(cap, t) for k, t in (("ray", np.int32), ("node", np.int32), ("local", np.int32),
                                            ("tmin", np.float32), ("tmax", np.float32), ("n", np.int32))}
    nseg = np.zeros(R, np.int32)
    ns = lib().oracle_ray_segments(R, _ptr(o), _ptr(d), act.shape[0], _ptr(act), _ptr(pmin), _ptr(pmax), M, cap,
                                   _ptr(seg["ray"]), _ptr(seg["node"]), _ptr(seg["local"]), _ptr(seg["tmin"]),
                                   _ptr(seg["tmax"]), _ptr(seg["n"]), _ptr(nseg))
    if ns < 0:
        raise RuntimeError(f"oracle_ray_segments failed ({ns})")
    res = {k: v[:ns].copy() for k, v in seg.items()}
    res["ray_nseg"] = nseg
    return res


def local_samples(g, node_id, pmin, pmax):
    g = _c(g, np.float32)
    nid = _c(node_id, np.int64)
    out = np.zeros_like(g)
    lib().oracle_local_samples(g.shape[0], _ptr(g), _ptr(nid), _ptr(_c(pmin, np.float32)), _ptr(_c(pmax, np.float32)),
                               _ptr(out))
    return out


def igs_forward(grid, index, uv):
    grid = _c(grid, np.float32)
    N, C, Z, Y, X = grid.shape
    index = _c(index, np.int64)
    uv = _c(uv, np.float32)
    out = np.zeros((index.shape[0], C), np.float32)
    lib().oracle_igs_forward(_ptr(grid), N, C, Z, Y, X, _ptr(index), _ptr(uv), index.shape[0], _ptr(out))
    return out


def igs_backward(grid, index, uv, grad_out):
    grid = _c(grid, np.float32)
    N, C, Z, Y, X = grid.shape
    index = _c(index, np.int64)
    uv = _c(uv, np.float32)
    go = _c(grad_out, np.float32)
    gg = np.zeros_like(grid)
    gu = np.zeros_like(uv)
    lib().oracle_igs_backward(_ptr(grid), N, C, Z, Y, X, _ptr(index), _ptr(uv), index.shape[0], _ptr(go), _ptr(gg),
                              _ptr(gu))
    return gg, gu


def project(objects, n_img, w, h, intr, rot, trans):
    obj = _c(objects, np.float64)
    out = np.zeros((n_img, h, w), np.float32)
    lib().oracle_project(_ptr(obj), obj.shape[0], n_img, w, h, _ptr(_c(intr, np.float64)), _ptr(_c(rot, np.float64)),
                         _ptr(_c(trans, np.float64)), _ptr(out))
    return out


def phantom_line(objects, o, d):
    obj = _c(objects, np.float64)
    return lib().oracle_phantom_line(_ptr(obj), obj.shape[0], _ptr(_c(o, np.float64)), _ptr(_c(d, np.float64)))


def phantom_density(objects, points):
    obj = _c(objects, np.float64)
    pts = _c(points, np.float64).reshape(-1, 3)
    out = np.zeros(pts.shape[0], np.float64)
    lib().oracle_phantom_density_batch(_ptr(obj), obj.shape[0], pts.shape[0], _ptr(pts), _ptr(out))
    return out


def project_pixels(objects, img, px, py, intr, rot, trans):
    obj = _c(objects, np.float64)
    img, px, py = _c(img, np.int32), _c(px, np.int32), _c(py, np.int32)
    out = np.zeros(img.shape[0], np.float32)
    lib().oracle_project_pixels(_ptr(obj), obj.shape[0], img.shape[0], _ptr(img), _ptr(px), _ptr(py),
                                _ptr(_c(intr, np.float64)), _ptr(_c(rot, np.float64)), _ptr(_c(trans, np.float64)),
                                _ptr(out))
    return out


# --------------------------------------------------------------------------
# float64 step
# --------------------------------------------------------------------------
def _trilinear_f64(torch, grid, row, uvw):
    """IGS in f64 with autograd: grid [N,C,G,G,G] (z,y,x), uvw [S,3] (x,y,z)."""
    N, C, Z, Y, X = grid.shape
    dims = torch.tensor([X - 1, Y - 1, Z - 1], dtype=torch.float64)
    p = (uvw + 1) / 2 * dims
    p0 = torch.floor(p)
    f = p - p0
    i0 = p0.long()
    out = 0
    for q in range(8):
        bx, by, bz = q & 1, (q >> 1) & 1, (q >> 2) & 1
        wx = f[:, 0] if bx else 1 - f[:, 0]
        wy = f[:, 1] if by else 1 - f[:, 1]
        wz = f[:, 2] if bz else 1 - f[:, 2]
        ix = (i0[:, 0] + bx).clamp(0, X - 1)
        iy = (i0[:, 1] + by).clamp(0, Y - 1)
        iz = (i0[:, 2] + bz).clamp(0, Z - 1)
        v = grid[row, :, iz, iy, ix]  # [S, C]
        out = out + v * (wx * wy * wz)[:, None]
    return out


def decoder_f64(torch, x, dec, C, beta):
    H = 64
    W1, b1, W2, b2, W3, b3 = torch.split(dec, [H * C, H, H * H, H, H, 1])
    h1 = torch.nn.functional.silu(x @ W1.reshape(H, C).T + b1)
    h2 = torch.nn.functional.silu(h1 @ W2.reshape(H, H).T + b2)
    y = h2 @ W3.reshape(1, H).T + b3
    return torch.nn.functional.softplus(y, beta=beta, threshold=20.0)[:, 0]


def image_f64(samples, grid, dec, node_min, node_max, prefix, R, beta=2.0):
    """Forward projection in f64 (with autograd graph); returns pred [R]."""
    import torch
    g = torch.from_numpy(samples["coords"]).double()
    nid = torch.from_numpy(samples["node_id"])
    mn = torch.from_numpy(node_min).double()[nid]
    mx = torch.from_numpy(node_max).double()[nid]
    local = (g - mn) / (mx - mn) * 2 - 1
    row = torch.from_numpy(prefix[samples["node_id"]])
    C = grid.shape[1]
    feat = _trilinear_f64(torch, grid, row, local)
    dens = decoder_f64(torch, feat, dec, C, beta)
    val = dens * torch.from_numpy(samples["weight"]).double()
    pred = torch.zeros(R, dtype=torch.float64).index_add(0, torch.from_numpy(samples["ray_index"]), val)
    return pred


def volume_positions(nx, ny, nz):
    """VolumeSamples (src/structure/HyperTree.cu:546-580, swap_xy = false):
    voxel v = x + nx (y + ny z) at p_d = (c_d / (n_d - 1)) * 2 - 1, each op
    rounded to float32.  Returns [V, 3] f32."""
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1).astype(np.float32)
    n1 = np.array([nx - 1, ny - 1, nz - 1], np.float32)
    return (c / n1) * np.float32(2) - np.float32(1)


def active_node_for_positions(p, node_active, node_min, node_max, max_depth):
    """ActiveNodeIdForGlobalPosition (src/structure/HyperTree.cu:598-637) for
    every row of p: descend from the root into the first child (order 0..7)
    whose closed box holds the point until an active node; -1 when a leaf is
    inactive or no child holds the point."""
    first_leaf = sum(8 ** d for d in range(max_depth))
    V = p.shape[0]
    cur = np.zeros(V, np.int64)
    res = np.full(V, -2, np.int64)  # -2: still descending
    for _ in range(max_depth + 1):
        live = res == -2
        act = live & (node_active[cur] > 0)
        res[act] = cur[act]
        live &= ~act
        leaf = live & (cur >= first_leaf)
        res[leaf] = -1
        live &= ~leaf
        nxt = np.full(V, -1, np.int64)
        for cid in range(8):
            c = 8 * cur + 1 + cid
            c = np.where(live, c, 0)
            inside = np.all((node_min[c] <= p) & (node_max[c] >= p), axis=1)
            take = live & (nxt < 0) & inside
            nxt[take] = c[take]
        none = live & (nxt < 0)
        res[none] = -1
        cur = np.where(live & (nxt >= 0), nxt, cur)
    res[res == -2] = -1
    return res


def volume_f64(nx, ny, nz, grid, dec, node_active, node_min, node_max, prefix, max_depth, beta=2.0):
    """UniformSampledVolume (src/geometry/geometry.cpp:166-248) in f64: density
    of every voxel in its active node, 0 outside.  Returns (vol [V], node [V],
    valid [V])."""
    import torch
    p = volume_positions(nx, ny, nz)
    node = active_node_for_positions(p, node_active, node_min, node_max, max_depth)
    valid = node >= 0
    vol = np.zeros(p.shape[0], np.float64)
    if valid.any():
        nid = node[valid]
        g = torch.from_numpy(p[valid]).double()
        mn = torch.from_numpy(node_min[nid]).double()
        mx = torch.from_numpy(node_max[nid]).double()
        local = (g - mn) / (mx - mn) * 2 - 1
        row = torch.from_numpy(prefix[nid])
        grid_t = torch.as_tensor(np.asarray(grid, np.float64))
        dec_t = torch.as_tensor(np.asarray(dec, np.float64))
        feat = _trilinear_f64(torch, grid_t, row, local)
        vol[valid] = decoder_f64(torch, feat, dec_t, grid_t.shape[1], beta).numpy()
    return vol, np.where(valid, node, 0), valid.astype(np.float32)


def adam_f64(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    bc1 = 1 - b1 ** step
    bc2 = 1 - b2 ** step
    p = p - (lr / bc1) * m / (np.sqrt(v) / np.sqrt(bc2) + eps)
    return p, m, v


def step_f64(samples, grid_ref, dec, target, node_min, node_max, prefix, beta=2.0, lr_grid=1e-2, lr_decoder=5e-5,
             step=1, state=None):
    """One training step in f64.  grid_ref [A,C,G,G,G], dec packed.  Returns
    dict(loss, pred, grad_grid, grad_dec, grid, dec, state)."""
    import torch
    R = target.shape[0]
    grid = torch.from_numpy(np.asarray(grid_ref, np.float64)).requires_grad_(True)
    d = torch.from_numpy(np.asarray(dec, np.float64)).requires_grad_(True)
    pred = image_f64(samples, grid, d, node_min, node_max, prefix, R, beta)
    loss = ((pred - torch.from_numpy(np.asarray(target, np.float64))) ** 2).mean()
    loss.backward()
    gg = grid.grad.numpy()
    gd = d.grad.numpy()
    if state is None:
        state = dict(gm=np.zeros_like(gg), gv=np.zeros_like(gg), dm=np.zeros_like(gd), dv=np.zeros_like(gd))
    new_grid, gm, gv = adam_f64(grid.detach().numpy(), gg, state["gm"], state["gv"], lr_grid, step)
    new_dec, dm, dv = adam_f64(d.detach().numpy(), gd, state["dm"], state["dv"], lr_decoder, step)
    return dict(loss=float(loss.detach()), pred=pred.detach().numpy(), grad_grid=gg, grad_dec=gd, grid=new_grid, dec=new_dec,
                state=dict(gm=gm, gv=gv, dm=dm, dv=dv))


# --------------------------------------------------------------------------
# camera pose and intrinsics gradients (f64 autograd)
# --------------------------------------------------------------------------
def _quat_rotate_t(torch, q, v):
    """v rotated by unit quaternions q = (x, y, z, w): v + w t + u x t, t = 2 u x v."""
    u, w = q[:, :3], q[:, 3:4]
    t = 2 * torch.cross(u, v, dim=1)
    return v + w * t + torch.cross(u, t, dim=1)


def pose_loss_f64(samples, uv, image_id, w, h, intr, rot, trans, grid, dec, target, node_min, node_max, prefix,
                  beta=2.0, tangent=None, cells_from_coords=True):
    """The step's loss in f64 as a function of the camera parameters, the
    reference's autograd chain (SceneBase::GetRays, src/data/SceneBase.cpp:171-193;
    Unproject, src/modules/CameraPose.cu:262-274; RotatePoint, CameraPose.cu:37-127
    with the rotation on a left tangent; positions o + d t with t constant,
    src/structure/HyperTree.cu:426-432; local coordinates, IGS, decoder,
    index_add, MSE).  Returns (loss, tangent, translation, intrinsics), the last
    three leaf tensors with gradients.  cells_from_coords: the trilinear cells
    from the sampler's f32 coordinates (the f64 positions carry only the
    gradient), else from the f64 positions themselves.  tangent [N,3] (default
    0): applied as exp(w) to first order, exact for the gradient at 0."""
    import torch
    R = target.shape[0]
    rot64 = torch.from_numpy(np.asarray(rot, np.float64).reshape(-1, 4))
    n_img = rot64.shape[0]
    tg = np.zeros((n_img, 3)) if tangent is None else np.asarray(tangent, np.float64)
    tangent = torch.from_numpy(tg.copy()).requires_grad_(True)
    tr = torch.from_numpy(np.asarray(trans, np.float64).reshape(-1, 3).copy()).requires_grad_(True)
    k = torch.from_numpy(np.asarray(intr, np.float64).reshape(-1)[:5].copy()).requires_grad_(True)
    uvf = np.asarray(uv, np.float32)
    px = torch.from_numpy((uvf[:, 0] * np.float32(w - 1)).astype(np.float64))
    py = torch.from_numpy((uvf[:, 1] * np.float32(h - 1)).astype(np.float64))
    img = torch.from_numpy(np.asarray(image_id, np.int64))
    x = (px - k[2]) / k[0]
    y = (py - k[3]) / k[1]
    u = torch.stack([x, y, torch.ones_like(x)], 1)
    n = u / u.norm(dim=1, keepdim=True)
    Rn = _quat_rotate_t(torch, rot64[img], n)
    d = Rn + torch.cross(tangent[img], Rn, dim=1)
    o = tr[img]
    ray = torch.from_numpy(samples["ray_index"])
    t = torch.from_numpy(samples["ray_t"].astype(np.float64))
    pg = o[ray] + d[ray] * t[:, None]
    p = torch.from_numpy(samples["coords"].astype(np.float64)) + (pg - pg.detach()) if cells_from_coords else pg
    nid = torch.from_numpy(samples["node_id"])
    mn = torch.from_numpy(node_min).double()[nid]
    mx = torch.from_numpy(node_max).double()[nid]
    local = (p - mn) / (mx - mn) * 2 - 1
    row = torch.from_numpy(prefix[samples["node_id"]])
    g = torch.from_numpy(np.asarray(grid, np.float64))
    feat = _trilinear_f64(torch, g, row, local)
    dens = decoder_f64(torch, feat, torch.from_numpy(np.asarray(dec, np.float64)), g.shape[1], beta)
    val = dens * torch.from_numpy(samples["weight"]).double()
    pred = torch.zeros(R, dtype=torch.float64).index_add(0, ray, val)
    loss = ((pred - torch.from_numpy(np.asarray(target, np.float64))) ** 2).mean()
    return loss, tangent, tr, k


def pose_grads_f64(samples, uv, image_id, w, h, intr, rot, trans, grid, dec, target, node_min, node_max, prefix,
                   beta=2.0, cells_from_coords=True):
    """d loss / d(rotation tangent [N,3] at 0, translation [N,3], intrinsics [5])
    in f64 (pose_loss_f64's chain)."""
    loss, tangent, tr, k = pose_loss_f64(samples, uv, image_id, w, h, intr, rot, trans, grid, dec, target, node_min,
                                         node_max, prefix, beta, cells_from_coords=cells_from_coords)
    loss.backward()
    return dict(loss=float(loss.detach()), tangent=tangent.grad.numpy(), translation=tr.grad.numpy(),
                intrinsics=k.grad.numpy())


def quat_exp_mul_f64(tangent, q):
    """exp(tangent) * q for rotation vectors [N,3] and unit quaternions [N,4]
    (x, y, z, w), renormalised: the rotation update of the structure step."""
    tangent = np.asarray(tangent, np.float64)
    q = np.asarray(q, np.float64)
    th = np.linalg.norm(tangent, axis=1)
    small = th < 1e-10
    ths = np.where(small, 1.0, th)
    im = np.where(small, 0.5 - th ** 2 / 48, np.sin(0.5 * th) / ths)
    re = np.where(small, 1 - th ** 2 / 8, np.cos(0.5 * th))
    a = np.concatenate([im[:, None] * tangent, re[:, None]], 1)
    ax, ay, az, aw = a.T
    bx, by, bz, bw = q.T
    out = np.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                    aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], 1)
    return out / np.linalg.norm(out, axis=1, keepdims=True)


# --------------------------------------------------------------------------
# learned sample proposal (restatement of neat_b200/csrc/neat_proposal.cuh)
# --------------------------------------------------------------------------
PROP_IN, PROP_H, PROP_B = 16, 32, 8
PROP_TRUNK = PROP_H * PROP_IN + PROP_H + PROP_H * PROP_H + PROP_H + PROP_B * PROP_H + PROP_B
PROP_TOTAL = PROP_TRUNK + PROP_H + PROP_IN + 1  # then the count head Wv [32] | Uv [16] | bv
JITTER_STREAM = 0x4a495454


def node_descriptors_f64(grid, dec, beta=2.0):
    """Per active node: the decoded density on the 4^3 lattice at local
    coordinates (i + 0.5) / 2 - 1 -> [centroid (3), spread, log(mean + 1e-3),
    log((peak + 1e-3) / (mean + 1e-3))], f64.  grid [A, C, G, G, G]."""
    import torch
    g = torch.as_tensor(np.asarray(grid, np.float64))
    A = g.shape[0]
    l = np.arange(4) * 0.5 - 0.75
    z, y, x = np.meshgrid(l, l, l, indexing="ij")
    pts = np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1)  # thread t: x = t & 3, y = (t >> 2) & 3, z = t >> 4
    uvw = torch.from_numpy(np.tile(pts, (A, 1)))
    row = torch.from_numpy(np.repeat(np.arange(A), 64))
    rho = decoder_f64(torch, _trilinear_f64(torch, g, row, uvw), torch.as_tensor(np.asarray(dec, np.float64)),
                      g.shape[1], beta).numpy().reshape(A, 64)
    S = rho.sum(1)
    mean = S / 64
    c = np.where(S[:, None] > 1e-12, (rho @ pts) / np.where(S > 1e-12, S, 1.0)[:, None], 0.0)
    r2 = (rho * (pts ** 2).sum(1)).sum(1)
    spread = np.where(S > 1e-12, np.sqrt(np.maximum(r2 / np.where(S > 1e-12, S, 1.0) - (c ** 2).sum(1), 0.0)), 0.968246)
    return np.stack([c[:, 0], c[:, 1], c[:, 2], spread, np.log(mean + 1e-3),
                     np.log((rho.max(1) + 1e-3) / (mean + 1e-3))], 1)


def proposal_features(o, d, segs, pmin, pmax, node_desc, prefix):
    """[Nseg, 16] f32: the node's descriptor, entry and exit points in
    node-local coordinates (every op in f32 as the device computes them),
    chord length over the node edge, three zeros."""
    r, nd = segs["ray"], segs["node"]
    mn, mx = pmin[nd].astype(np.float32), pmax[nd].astype(np.float32)
    oo, dd = o[r].astype(np.float32), d[r].astype(np.float32)
    t0, t1 = segs["tmin"].astype(np.float32)[:, None], segs["tmax"].astype(np.float32)[:, None]
    size = mx - mn
    loc = lambda g: ((g - mn) / size) * np.float32(2) - np.float32(1)
    f = np.zeros((r.shape[0], PROP_IN), np.float32)
    f[:, 0:6] = np.asarray(node_desc, np.float32)[prefix[nd]]
    f[:, 6:9] = loc(oo + dd * t0)
    f[:, 9:12] = loc(oo + dd * t1)
    f[:, 12] = (t1[:, 0] - t0[:, 0]) / size[:, 0]
    e = f[:, 9:12] - f[:, 6:9]
    cv = f[:, 0:3] - f[:, 6:9]
    L2 = (e * e).sum(1) + np.float32(1e-12)
    us = (cv * e).sum(1) / L2
    p2 = np.maximum((cv * cv).sum(1) - us * us * L2, 0)
    f[:, 13] = np.clip(us, -0.5, 1.5)
    f[:, 14] = np.sqrt(p2) / (f[:, 3] + np.float32(0.05))
    return f


def _proposal_trunk_f64(torch, params, f):
    H, I, B = PROP_H, PROP_IN, PROP_B
    W1, b1, W2, b2, W3, b3, Wv, Uv, bv = torch.split(params, [H * I, H, H * H, H, B * H, B, H, I, 1])
    x = torch.as_tensor(f, dtype=torch.float64)
    h1 = torch.nn.functional.silu(x @ W1.reshape(H, I).T + b1)
    h2 = torch.nn.functional.silu(h1 @ W2.reshape(H, H).T + b2)
    return x, h2, (W3, b3, Wv, Uv, bv)


def proposal_probs_f64(torch, params, f, mix):
    """Mixed bin probabilities p = (1 - mix) softmax(MLP(f)) + mix / 8, f64."""
    _, h2, (W3, b3, _, _, _) = _proposal_trunk_f64(torch, params, f)
    z = h2 @ W3.reshape(PROP_B, PROP_H).T + b3
    return (1 - mix) * torch.softmax(z, 1) + mix / PROP_B


def proposal_head_f64(torch, params, f, detach_trunk=False):
    """The count head v = bv + Wv . h2 + Uv . f (neat_proposal.cuh: PropOff::VW),
    a prediction of log(a + 1e-4), f64; detach_trunk: no gradient into h2."""
    x, h2, (_, _, Wv, Uv, bv) = _proposal_trunk_f64(torch, params, f)
    if detach_trunk:
        h2 = h2.detach()
    return h2 @ Wv + x @ Uv + bv


def proposal_counts(v, n_ref, eps, nmin):
    """Samples a segment gets from the count head (neat_proposal.cuh:
    proposal_count): min(n_ref, max(min(nmin, n_ref), ceil(exp(v) / eps))),
    n_ref where eps <= 0; also the unrounded exp(v) / eps (for callers that
    set aside counts within rounding of an integer)."""
    n_ref = np.asarray(n_ref, np.int64)
    if eps <= 0:
        return n_ref.copy(), np.full(n_ref.shape, np.inf)
    x = np.minimum(np.exp(np.asarray(v, np.float64)) / eps, n_ref)
    n = np.maximum(np.ceil(x).astype(np.int64), np.minimum(nmin, n_ref))
    return np.minimum(n, n_ref), x


def proposal_inverse(c, u):
    """Position in [0,1] of CDF value u under the piecewise-linear CDF with bin
    ends c[:, 0..7] (c[:, 7] = 1), row-wise."""
    b = (u[:, None] >= c[:, :PROP_B - 1]).sum(1)
    lo = np.where(b > 0, np.take_along_axis(c, np.maximum(b - 1, 0)[:, None], 1)[:, 0], 0.0)
    hi = np.take_along_axis(c, b[:, None], 1)[:, 0]
    w = hi - lo
    fr = np.where(w > 0, (u - lo) / np.where(w > 0, w, 1.0), 0.5)
    return (b + np.clip(fr, 0.0, 1.0)) / PROP_B


def sample_offsets(segs, jitter, seed, step, n_key=None):
    """Per sample of the segments (segment-major, j inside): segment index, j,
    stratified offset a (Philox jitter stream or 0.5) and u = (j + a) / n in f32.
    The jitter is keyed on the index in the ray of the segment's first sample
    under the counts n_key (default: the segments' own counts; the count head's
    counts keep the keys of the reference's counts)."""
    n = segs["n"].astype(np.int64)
    sid = np.repeat(np.arange(n.shape[0]), n)
    start = np.concatenate([[0], np.cumsum(n)[:-1]])
    j = np.arange(sid.shape[0]) - start[sid]
    # index in the ray of each segment's first sample (segments are ray-major)
    nk = n if n_key is None else np.asarray(n_key, np.int64)
    kstart = np.concatenate([[0], np.cumsum(nk)[:-1]])
    first = np.concatenate([[0], np.cumsum(segs["ray_nseg"].astype(np.int64))[:-1]])
    base = kstart - kstart[first[segs["ray"]]]
    if jitter:
        a = np.array([uniform(seed, int(segs["ray"][s]), int(base[s] + jj), step, JITTER_STREAM)
                      for s, jj in zip(sid, j)], np.float32)
    else:
        a = np.full(sid.shape[0], 0.5, np.float32)
    u = (j.astype(np.float32) + a) / n[sid].astype(np.float32)
    return sid, j, a, u.astype(np.float32)


def proposal_samples(o, d, segs, cdf, jitter, seed=0, step=1, n_key=None):
    """Samples placed by the proposal CDF (one row of bin ends per segment):
    t = tmin + (tmax - tmin) F^-1((j + a) / n), midpoint-rule weights on the
    placed positions, f64.  Returns a SampleList-like dict for image_f64."""
    sid, j, a, u = sample_offsets(segs, jitter, seed, step, n_key)
    t0 = segs["tmin"].astype(np.float64)[sid]
    t1 = segs["tmax"].astype(np.float64)[sid]
    n = segs["n"][sid]
    t = t0 + (t1 - t0) * proposal_inverse(np.asarray(cdf, np.float64)[sid], u.astype(np.float64))
    tp = np.concatenate([[0.0], t[:-1]])
    tn = np.concatenate([t[1:], [0.0]])
    lo = np.where(j == 0, t0, (tp + t) * 0.5)
    hi = np.where(j == n - 1, t1, (tn + t) * 0.5)
    r = segs["ray"][sid]
    coords = o[r].astype(np.float64) + d[r].astype(np.float64) * t[:, None]
    return dict(coords=coords, weight=hi - lo, ray_index=r.astype(np.int64), node_id=segs["node"][sid].astype(np.int64))


def proposal_targets(o, d, segs, M, grid, dec, node_min, node_max, prefix, jitter, seed, step, beta=2.0):
    """Uniformly sampled contributions density * weight of every sample (f64),
    binned into eighths of its segment by u = (j + a) / n: [Nseg, 8]."""
    import torch
    s = create_samples(o, d, np.nonzero(prefix >= 0)[0], node_min, node_max, M, jitter, seed, step)
    sid, j, a, u = sample_offsets(segs, jitter, seed, step)
    assert sid.shape[0] == s["ray_t"].shape[0]
    g = torch.from_numpy(s["coords"]).double()
    nid = torch.from_numpy(s["node_id"])
    mn = torch.from_numpy(node_min).double()[nid]
    mx = torch.from_numpy(node_max).double()[nid]
    local = (g - mn) / (mx - mn) * 2 - 1
    row = torch.from_numpy(prefix[s["node_id"]])
    grid_t = torch.as_tensor(np.asarray(grid, np.float64))
    feat = _trilinear_f64(torch, grid_t, row, local)
    dens = decoder_f64(torch, feat, torch.as_tensor(np.asarray(dec, np.float64)), grid_t.shape[1], beta).numpy()
    c = dens * s["weight"].astype(np.float64)
    b = np.minimum(7, (u * np.float32(8)).astype(np.int64))
    hist = np.zeros((segs["n"].shape[0], PROP_B))
    np.add.at(hist, (sid, b), c)
    return hist


def proposal_count_targets(o, d, segs, M, grid, dec, node_min, node_max, prefix, jitter, seed, step, beta=2.0):
    """The count head's target argument per segment of a uniformly sampled
    step (neat_proposal.cu: k_seg_variation): a = (tmax - tmin) times the total
    variation sum_j |rho_j - rho_j-1| of its samples' densities, f64."""
    import torch
    s = create_samples(o, d, np.nonzero(prefix >= 0)[0], node_min, node_max, M, jitter, seed, step)
    sid, j, _, _ = sample_offsets(segs, jitter, seed, step)
    assert sid.shape[0] == s["ray_t"].shape[0]
    g = torch.from_numpy(s["coords"]).double()
    nid = torch.from_numpy(s["node_id"])
    mn = torch.from_numpy(node_min).double()[nid]
    mx = torch.from_numpy(node_max).double()[nid]
    row = torch.from_numpy(prefix[s["node_id"]])
    grid_t = torch.as_tensor(np.asarray(grid, np.float64))
    feat = _trilinear_f64(torch, grid_t, row, (g - mn) / (mx - mn) * 2 - 1)
    dens = decoder_f64(torch, feat, torch.as_tensor(np.asarray(dec, np.float64)), grid_t.shape[1], beta).numpy()
    step_tv = np.where(j > 0, np.abs(dens - np.concatenate([[0.0], dens[:-1]])), 0.0)
    tv = np.zeros(segs["n"].shape[0])
    np.add.at(tv, sid, step_tv)
    return (segs["tmax"].astype(np.float64) - segs["tmin"].astype(np.float64)) * tv


def proposal_variation_targets(hist):
    """Binned masses m [Nseg, 8] -> (targets v / sum v with v_b = |m_b - m_b-1|
    + |m_b+1 - m_b|, total variation sum_b |m_b - m_b-1| as the segment's weight)."""
    dm = np.abs(np.diff(hist, axis=1))
    v = np.zeros_like(hist)
    v[:, 1:] += dm
    v[:, :-1] += dm
    tv = dm.sum(1)
    return v / np.where(tv > 0, 2 * tv, 1.0)[:, None], tv


def proposal_grad_f64(params, f, hist, mix, a=None):
    """Cross-entropy between the variation targets of the binned masses and the
    proposal, averaged over the segments weighted by their total variation,
    and its gradient w.r.t. the trunk and placement head (f64).  With the
    count targets a (proposal_count_targets; < 0: no target), also the count
    head's loss mean((v - log(a + 1e-4))^2) / 2 over the segments and its
    gradient w.r.t. the count head (the trunk held fixed): (ce, gradient,
    head loss or None)."""
    import torch
    qv, tv = proposal_variation_targets(hist)
    use = tv > 1e-20
    q = torch.from_numpy(qv[use])
    m = torch.from_numpy(tv[use])
    P = torch.tensor(np.asarray(params, np.float64), requires_grad=True)
    p = proposal_probs_f64(torch, P, f[use], mix)
    loss = (-(q * torch.log(p)).sum(1) * m).sum() / m.sum()
    loss.backward()
    grad = P.grad.numpy().copy()
    grad[PROP_TRUNK:] = 0.0
    if a is None:
        return float(loss.detach()), grad, None
    a = np.asarray(a, np.float64)
    ok = a >= 0
    P2 = torch.tensor(np.asarray(params, np.float64), requires_grad=True)
    v = proposal_head_f64(torch, P2, f[ok], detach_trunk=True)
    y = torch.from_numpy(np.log(a[ok] + 1e-4))
    lh = 0.5 * ((v - y) ** 2).mean()
    lh.backward()
    grad[PROP_TRUNK:] = P2.grad.numpy()[PROP_TRUNK:]
    return float(loss.detach()), grad, float(lh.detach())


# --------------------------------------------------------------------------
# volume regularisers (src/geometry/geometry_ex_ex.h:18-58, geometry_ex_ex.cpp:86-156)
# --------------------------------------------------------------------------
def tv_f64(grid, w):
    """TVLoss without weights: w * C * sum over the 3 grid axes of
    mean_node mean_{c,cells} |difference|, and its gradient (f64)."""
    import torch
    g = torch.tensor(np.asarray(grid, np.float64), requires_grad=True)
    C = g.shape[1]
    loss = 0
    for d in (2, 3, 4):
        n = g.shape[d]
        diff = (g.narrow(d, 0, n - 1) - g.narrow(d, 1, n - 1)).abs().mean((1, 2, 3, 4))
        loss = loss + diff.mean()
    loss = loss * C * w
    loss.backward()
    return float(loss.detach()), g.grad.numpy()


def edge_pairs(tree_min, tree_max, node_active, active_ids, max_depth, G, eps):
    """NodeNeighborSamples: (node, face, point index, other node, point) of
    every pair, in (node, face, point) order; every op in f32."""
    per = 6 * G * G
    A = active_ids.shape[0]
    a = np.repeat(np.arange(A), per)
    f = np.tile(np.repeat(np.arange(6), G * G), A)
    k = np.tile(np.arange(G * G), 6 * A)
    node = active_ids[a]
    side, front = f // 2, f % 2
    sa, sb = (side + 1) % 3, (side + 2) % 3
    loc = np.zeros((a.shape[0], 3), np.float32)
    idx = np.arange(a.shape[0])
    loc[idx, side] = front.astype(np.float32)
    loc[idx, sa] = (k % G).astype(np.float32) / np.float32(G - 1)
    loc[idx, sb] = (k // G).astype(np.float32) / np.float32(G - 1)
    mn, mx = tree_min[node].astype(np.float32), tree_max[node].astype(np.float32)
    p = loc * (mx - mn) + mn
    q = p.copy()
    q[idx, side] = q[idx, side] + np.where(front == 1, np.float32(eps), np.float32(-eps))
    other = active_node_for_positions(q, node_active, tree_min, tree_max, max_depth)
    keep = (other != -1) & (other != node)
    return a[keep], f[keep], k[keep], node[keep], other[keep], p[keep]


def edge_f64(grid, tree_min, tree_max, node_active, active_ids, prefix, max_depth, eps, w, seed, step):
    """Edge loss and its gradient (f64): pairs of NodeNeighborSamples, error
    mean_c |f_node - f_other| * r, loss = w * C * mean over pairs."""
    import torch
    G = grid.shape[2]
    a, f, k, node, other, p = edge_pairs(tree_min, tree_max, node_active, active_ids, max_depth, G, eps)
    g = torch.tensor(np.asarray(grid, np.float64), requires_grad=True)
    C = g.shape[1]
    pt = torch.from_numpy(p.astype(np.float64))

    def feat(nd):
        mn = torch.from_numpy(tree_min[nd].astype(np.float64))
        mx = torch.from_numpy(tree_max[nd].astype(np.float64))
        return _trilinear_f64(torch, g, torch.from_numpy(prefix[nd]), (pt - mn) / (mx - mn) * 2 - 1)

    r = torch.tensor([uniform(seed, int(ai), int(fi * G * G + ki), step, 0x45444745) for ai, fi, ki in zip(a, f, k)],
                     dtype=torch.float64)
    err = (feat(node) - feat(other)).abs().mean(1) * r
    loss = err.mean() * w * C
    loss.backward()
    return float(loss.detach()), g.grad.numpy(), a.shape[0]


# --------------------------------------------------------------------------
# structure updates (samples/reconstruct.cpp:254-319, geometry_ex_ex.cpp:182-209)
# --------------------------------------------------------------------------
def node_lattice(node_min, node_max, nodes, G):
    """UniformGlobalSamples: [len(nodes), G^3, 3] f32, cells x fastest."""
    z, y, x = np.meshgrid(np.arange(G), np.arange(G), np.arange(G), indexing="ij")
    r = np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1).astype(np.float32)
    l = r / np.float32(G - 1)
    mn = node_min[nodes].astype(np.float32)[:, None, :]
    mx = node_max[nodes].astype(np.float32)[:, None, :]
    return l[None] * (mx - mn) + mn


def point_in_any_image(p, intr, rot, trans, w, h):
    """PointInAnyImage (src/data/SceneBase.cu:13-45), f64, per row of p."""
    fx, fy, cx, cy = intr.reshape(-1)[:4]
    p = np.asarray(p, np.float64)
    out = np.zeros(p.shape[0], bool)
    for q, t in zip(rot, trans):
        u, qw = -np.asarray(q[:3]), q[3]
        v = p - t
        tt = 2 * np.cross(u, v)
        c = v + qw * tt + np.cross(u, tt)
        px = np.round(fx * c[:, 0] / c[:, 2] + cx)
        py = np.round(fy * c[:, 1] / c[:, 2] + cy)
        out |= (px >= 0) & (px < w) & (py >= 0) & (py < h)
    return out


def node_max_density_f64(grid, dec, node_min, node_max, active_ids, G, beta=2.0, cam=None):
    """ComputeMaxDensity: per active node the max f64 density over its lattice
    (times the PointInAnyImage mask when cam = (intr, rot, trans, w, h))."""
    import torch
    A = active_ids.shape[0]
    P = node_lattice(node_min, node_max, active_ids, G).reshape(-1, 3)
    node = np.repeat(active_ids, G ** 3)
    mn = torch.from_numpy(node_min[node].astype(np.float64))
    mx = torch.from_numpy(node_max[node].astype(np.float64))
    local = (torch.from_numpy(P.astype(np.float64)) - mn) / (mx - mn) * 2 - 1
    row = torch.from_numpy(np.repeat(np.arange(A), G ** 3))
    g = torch.as_tensor(np.asarray(grid, np.float64))
    rho = decoder_f64(torch, _trilinear_f64(torch, g, row, local), torch.as_tensor(np.asarray(dec, np.float64)),
                      g.shape[1], beta).numpy()
    if cam is not None:
        rho = rho * point_in_any_image(P, *cam)
    return rho.reshape(A, -1).max(1)


def interpolate_grid_f64(old_grid, node_min, node_max, old_active, old_ids, old_prefix, max_depth, new_ids, G):
    """InterpolateInactiveNodes: the new rows [len(new_ids), C, G, G, G] from the
    old grid at the new nodes' lattice points, f64."""
    import torch
    P = node_lattice(node_min, node_max, new_ids, G).reshape(-1, 3)
    on = active_node_for_positions(P, old_active, node_min, node_max, max_depth)
    on = np.where(on >= 0, on, old_ids[0])
    mn = torch.from_numpy(node_min[on].astype(np.float64))
    mx = torch.from_numpy(node_max[on].astype(np.float64))
    local = (torch.from_numpy(P.astype(np.float64)) - mn) / (mx - mn) * 2 - 1
    g = torch.as_tensor(np.asarray(old_grid, np.float64))
    f = _trilinear_f64(torch, g, torch.from_numpy(old_prefix[on]), local).numpy()
    C = g.shape[1]
    return f.reshape(len(new_ids), G, G, G, C).transpose(0, 4, 1, 2, 3)


# --------------------------------------------------------------------------
# photometric calibration (src/modules/ToneMapper.cpp:14-223), with torch's own
# grid_sample as the reference calls it
# --------------------------------------------------------------------------
def tonemap_f64(torch, x, uv, img, ef, eb, sb, resp, rng, exposure=True, mult=False, sensor=True, response=True,
                training=True):
    """PhotometricCalibration::forward on ray integrals x [R] (f64 autograd)."""
    F = torch.nn.functional
    y = x
    if exposure:
        if mult:
            y = y * ef[img]
        y = y + eb[img]
    if sensor:
        g = (uv * 2 - 1).unsqueeze(0).unsqueeze(0)
        s = F.grid_sample(sb.reshape(1, 1, *sb.shape), g, mode="bilinear", padding_mode="border", align_corners=False)
        y = y + s.reshape(-1)
    if response:
        leak = (y - rng) * (y > rng) if training else 0
        xi = (y * (1.0 / rng)) * 2 - 1
        grid = torch.stack([xi, torch.zeros_like(xi)], 1).reshape(1, 1, -1, 2)
        r = F.grid_sample(resp.reshape(1, 1, 1, -1), grid, mode="bilinear", padding_mode="border", align_corners=True)
        y = r.reshape(-1) + leak
    return y


def response_param_loss_f64(torch, resp):
    """CameraResponseNet::ParamLoss (src/modules/ToneMapper.cpp:100-119)."""
    P = resp.shape[0]
    target = resp.clone()
    target = torch.cat([torch.zeros(1, dtype=resp.dtype), (resp[2:] + resp[:-2]) * 0.5, resp[-1:]])
    f = P * np.sqrt(1e-5)
    return ((resp * f - target * f) ** 2).sum()
