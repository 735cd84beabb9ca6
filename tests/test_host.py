"""Host-side tests (no GPU): the C ABI library loads and exports every entry
point include/neat_b200.h declares; host octree bookkeeping equals the
oracle's; synthetic geometry conventions; the multi-rank timing helpers of
bench.py over gloo."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    src = open(os.path.join(ROOT, "include", "neat_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(neat_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from neat_b200.csrc import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = _header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from neat_b200 import _lib
    assert sorted(_lib.exported_symbols()) == names


def test_torch_shim_loads_and_registers_its_operators():
    """libneat_torch.so (the reference's libtorch module API in C++) is built
    against the installed torch, links libneat_b200.so and registers one torch
    operator per entry of neat_torch.h; a call with CPU tensors is refused."""
    import torch
    from neat_b200 import _lib
    from neat_b200.csrc import build
    build.build()
    ops = _lib.load_torch_ops()
    for name in _lib.TORCH_OPS:
        assert hasattr(ops, name), name
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        ops.IndirectGridSample3D(torch.zeros(1, 1, 2, 2, 2), torch.zeros(1, dtype=torch.long), torch.zeros(1, 3))


def test_library_host_calls_without_gpu():
    from neat_b200 import _lib
    lib = _lib.load()
    assert lib.neat_version() >= 1
    assert lib.neat_decoder_params(8) == 64 * 8 + 64 + 64 * 64 + 64 + 64 + 1
    assert lib.neat_tree_table_bytes(2) == 73 * 16 + 512  # entries + descendant marks
    assert lib.neat_tree_table_bytes(0) == 0
    assert b"capacity" in lib.neat_status_string(_lib.NEAT_ERR_CAPACITY)
    # argument validation happens on the host before any launch
    assert lib.neat_make_rays(None, None, None, -1, 16, 16, None, None, None, None, None, None) == \
        _lib.NEAT_ERR_BAD_INPUT
    assert lib.neat_tree_prepare(None, None, None, 4, 9, None, None, None) == _lib.NEAT_ERR_BAD_INPUT
    # the look-ahead entries refuse missing arguments the same way
    assert lib.neat_train_step_segments(None, None, None, None, None, None, 0, None) == _lib.NEAT_ERR_BAD_INPUT
    assert lib.neat_train_step_prebuilt(None, None, None, 0, 1, None, None, 0, None) == _lib.NEAT_ERR_BAD_INPUT


def test_proposal_count_arguments_checked_before_any_launch():
    """A SAMPLE-mode proposal with the count head on needs count_min >= 1 and a
    finite, non-negative count_eps: otherwise the call is refused on the host
    (bad input); valid ones get as far as the workspace size check (a zero-byte
    workspace: capacity), before any launch."""
    import ctypes
    import math
    from neat_b200 import _lib
    lib = _lib.load()
    d = _lib.StepDesc(tree_table=16, num_active=8, max_depth=2, node_min=16, node_max=16, w=64, h=64,
                      intrinsics=16, rotation=16, translation=16, C=8, G=9, softplus_beta=2.0,
                      max_samples_per_node=8, seg_capacity=4096, decoder_path=_lib.NEAT_DECODER_TC_BF16, proposal=1)
    b = _lib.StepBatch(uv=16, image_id=16, target=16, num_rays=512)
    cnt = (ctypes.c_int64 * 4)()
    status = ctypes.c_int(0)

    def call(eps, nmin):
        pr = _lib.Proposal(mode=_lib.NEAT_PROPOSAL_SAMPLE, params=16, node_desc=16, mix=0.25, count_eps=eps,
                           count_min=nmin)
        return lib.neat_train_step_segments(ctypes.byref(d), ctypes.byref(pr), ctypes.byref(b), ctypes.addressof(cnt),
                                            ctypes.addressof(status), 16, 0, None)

    assert call(0.05, 0) == _lib.NEAT_ERR_BAD_INPUT
    assert call(-0.1, 2) == _lib.NEAT_ERR_BAD_INPUT
    assert call(math.nan, 2) == _lib.NEAT_ERR_BAD_INPUT
    assert call(0.05, 2) == _lib.NEAT_ERR_CAPACITY
    assert call(0.0, 0) == _lib.NEAT_ERR_CAPACITY  # counts off: count_min unused


def test_no_cpu_fallback_when_library_missing(monkeypatch):
    from neat_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libneat_b200.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


@pytest.mark.parametrize("depth", [1, 2, 4])
def test_tree_tables_match_oracle(oracle, depth):
    from neat_b200.tree import HyperTreeBase
    T = HyperTreeBase(3, depth)
    t = oracle.tree_build(depth)
    np.testing.assert_array_equal(T.node_position_min, t["min"])
    np.testing.assert_array_equal(T.node_position_max, t["max"])
    np.testing.assert_array_equal(T.node_children, t["children"])
    np.testing.assert_array_equal(T.node_parent, t["parent"])
    T.SetActive(depth)
    assert T.NumActiveNodes() == 8 ** depth
    assert np.all(np.diff(T.active_node_ids) > 0)
    pre = T.node_active_prefix_sum
    assert np.all(pre[T.active_node_ids] == np.arange(8 ** depth))
    assert np.all(pre[T.node_depth != depth] == -1)


def test_cell_node_map(oracle):
    """The finest-cell map of the step's DDA hit search: every finest cell
    holds the active node whose box contains its centre (or -1); a tree with an
    active node inside another, or deeper than 5, has none."""
    from neat_b200 import scene as SC
    from neat_b200.tree import HyperTreeBase
    objs = SC.ellipsoid_phantom(8, 10, seed=3)
    T = HyperTreeBase(3, 4)
    T.RefineByVariance(lambda p: oracle.phantom_density(objs, p), 200, samples_per_axis=3)
    act = T.active_node_ids
    keep = act[np.random.default_rng(1).random(act.shape[0]) < 0.7]  # holes: cells of no active node
    T.SetActiveNodes(keep)
    cells = T.cell_node_map()
    N = 16
    c = (np.arange(N) + 0.5) / N * 2 - 1
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    p = np.stack([x, y, z], -1).reshape(-1, 3)
    mn, mx = T.node_position_min[keep], T.node_position_max[keep]
    inside = np.all((p[:, None] >= mn[None]) & (p[:, None] < mx[None]), axis=2)
    want = np.where(inside.any(1), keep[inside.argmax(1)], -1)
    np.testing.assert_array_equal(cells.reshape(-1), want)
    nested = np.concatenate([keep[:5], [int(T.node_parent[keep[0]])]])
    T.SetActiveNodes(np.unique(nested))
    assert T.cell_node_map() is None
    assert HyperTreeBase(3, 6).cell_node_map() is None


def test_refine_by_variance_partitions_the_cube(oracle):
    from neat_b200 import scene as SC
    from neat_b200.tree import HyperTreeBase
    objs = SC.ellipsoid_phantom(8, 10, seed=3)
    T = HyperTreeBase(3, 4)
    T.RefineByVariance(lambda p: oracle.phantom_density(objs, p), 300, samples_per_axis=3)
    A = T.NumActiveNodes()
    assert 290 <= A <= 300
    # active leaves tile [-1,1]^3 exactly: volumes sum to 8, no active ancestor of an active node
    vol = np.prod(T.node_position_max[T.active_node_ids] - T.node_position_min[T.active_node_ids], axis=1)
    assert abs(vol.sum() - 8.0) < 1e-9
    act = set(T.active_node_ids.tolist())
    for n in T.active_node_ids:
        p = T.node_parent[n]
        while p >= 0:
            assert p not in act
            p = T.node_parent[p]
    # refinement follows the density: finest nodes where the phantom varies
    assert T.node_depth[T.active_node_ids].max() == 4


def test_cone_beam_geometry():
    from neat_b200 import scene as SC
    intr, rot, trans = SC.cone_beam_geometry(8, 64, 48)
    assert intr.shape == (1, 5) and intr[0, 2] == 31.5 and intr[0, 3] == 23.5
    # the cube's bounding sphere (radius sqrt 3) spans the detector width
    assert abs(64 / intr[0, 0] / 2 - np.tan(np.arcsin(np.sqrt(3) / 3))) < 1e-12
    for q, t in zip(rot, trans):
        assert abs(np.linalg.norm(q) - 1) < 1e-12
        assert abs(np.linalg.norm(t) - 3) < 1e-12 and t[2] == 0


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    q.put((rank, float(t.item())))
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    """bench.py takes the max of the per-rank device times over ranks; the
    replicas-only multi-GPU path has no other collective."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, 11.0), (1, 11.0)]


def test_ctypes_structs_match_header(tmp_path):
    """Every ctypes mirror of a C-ABI struct has the header's size and field offsets
    (a probe compiled with gcc against include/neat_b200.h)."""
    import shutil
    import subprocess
    from neat_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    pairs = {"neat_step_desc": _lib.StepDesc, "neat_proposal": _lib.Proposal, "neat_tonemap": _lib.ToneMap,
             "neat_pose_grad": _lib.PoseGrad, "neat_step_state": _lib.StepState, "neat_step_batch": _lib.StepBatch,
             "neat_step_out": _lib.StepOut, "neat_project_out": _lib.ProjectOut}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "neat_b200.h"', "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0; }"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            parts = line.split()
            got[(parts[0], parts[1])] = int(parts[2])
    for cname, cls in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, *_ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_step_roofline_arithmetic():
    """The whole-step roofline bench.py reports: F = 6 (C H + H^2 + H) S flops,
    B = 16 R + 36 P bytes, T* = max of the flop and byte times."""
    import bench
    peaks = {"hbm_gbs": 1000.0, "bf16_tflops_sustained": 100.0}
    r = bench.step_roofline(S=1000, R=10, P=100, C=8, ms_step=1.0, peaks=peaks, simt_peak_tflops=10.0)
    F = 6.0 * (8 * 64 + 64 * 64 + 64) * 1000
    assert r["flops"] == F and r["bytes"] == 16 * 10 + 36 * 100
    assert r["t_star_ms_tensor"] == pytest.approx(1e3 * max(F / 100e12, 3760 / 1000e9))
    assert r["frac_fp32_simt"] == pytest.approx(1e3 * max(F / 10e12, 3760 / 1000e9) / 1.0)
    assert r["bound_tensor"] == "tensor" and r["bound_fp32_simt"] == "fp32"
    r = bench.step_roofline(S=1, R=10, P=10 ** 6, C=8, ms_step=1.0, peaks=peaks, simt_peak_tflops=10.0)
    assert r["bound_tensor"] == "hbm" and r["bound_fp32_simt"] == "hbm"


SETTINGS_TEXT = """
[TrainParams]
random_seed = 3746934646
batch_size = 16000
lr_exex_grid_adam = 0.0399999991
exex_op = adam
train_interval_jitter = true
loss_tv = 0.0000000000
loss_edge = 0.001
optimize_pose = true
optimize_intrinsics = false
lr_pose = 0.002
lr_intrinsics = 50.0

[PhotometricCalibrationParams]
response_enable = true
response_range = 2
exposure_enable = true
exposure_mult = false
sensor_bias_enable = false
sensor_bias_size_w = 32

[Netparams]
grid_size = 17
grid_features = 8
last_activation_function = softplus
softplus_beta = 2
decoder_skip = false
decoder_lr = 4.999999874e-05
decoder_activation = silu
decoder_hidden_layers = 1
decoder_hidden_features = 64

[OctreeParams]
start_layer = 2
tree_depth = 4
max_samples_per_node = 32
tree_optimizer_params.max_active_nodes = 512
"""


def test_settings_map_to_trainer_arguments():
    """The reference's INI section and key names map onto FusedTrainer arguments."""
    from neat_b200 import config
    st = config.load_settings(text=SETTINGS_TEXT)
    assert st["OctreeParams"]["tree_optimizer_params.max_active_nodes"] == "512"
    kw = config.trainer_kwargs(st)
    assert kw["num_features"] == 8 and kw["grid_size"] == 17 and kw["max_samples_per_node"] == 32
    assert kw["lr_grid"] == pytest.approx(0.04) and kw["lr_decoder"] == pytest.approx(5e-5)
    assert kw["softplus_beta"] == 2.0 and kw["seed"] == 3746934646
    assert kw["loss_edge"] == pytest.approx(0.001) and kw["loss_tv"] == 0.0
    assert kw["optimize_pose"] is True and kw["optimize_intrinsics"] is False and kw["lr_pose"] == 0.002
    # keys the section lists, the rest from PhotometricCalibrationParams' initialisers
    assert kw["tonemap"] == {"response_enable": True, "response_range": 2.0, "response_lr": 0.1,
                             "exposure_enable": True, "exposure_mult": False, "exposure_lr": 0.01,
                             "sensor_bias_enable": False, "sensor_bias_size_w": 32, "sensor_bias_lr": 0.05}
    run = config.run_settings(st)
    assert run == {"batch_size": 16000, "train_interval_jitter": True, "tree_depth": 4, "start_layer": 2}
    # the signature of FusedTrainer accepts every mapped argument
    import inspect
    from neat_b200.trainer import FusedTrainer
    params = inspect.signature(FusedTrainer.__init__).parameters
    assert all(k in params for k in kw)


def test_settings_defaults_follow_the_reference():
    """An INI without the keys gets the reference's struct initialisers
    (src/Settings.h: Netparams :46-57, OctreeParams :85-89, MyTrainParams
    :216-240; src/modules/ToneMapper.h:36-47): regularisers, pose and
    intrinsics refinement and the photometric calibration are on."""
    from neat_b200 import config
    for text in ("", "[TrainParams]\n[Netparams]\n[OctreeParams]\n"):
        st = config.load_settings(text=text)
        kw = config.trainer_kwargs(st)
        assert kw["num_features"] == 4 and kw["grid_size"] == 17 and kw["softplus_beta"] == 2.0
        assert kw["lr_decoder"] == pytest.approx(5e-5) and kw["lr_grid"] == pytest.approx(0.04)
        assert kw["max_samples_per_node"] == 32
        assert kw["loss_tv"] == pytest.approx(1e-4) and kw["loss_edge"] == pytest.approx(1e-3)
        assert kw["optimize_pose"] is True and kw["optimize_intrinsics"] is True
        assert kw["lr_pose"] == pytest.approx(1e-3) and kw["lr_intrinsics"] == 100.0
        assert kw["tonemap"] == config.TONEMAP_DEFAULTS
        assert kw["tonemap"]["response_enable"] and kw["tonemap"]["exposure_enable"]
        assert kw["tonemap"]["sensor_bias_enable"] and kw["tonemap"]["sensor_bias_size_w"] == 32
        run = config.run_settings(st)
        assert run["tree_depth"] == 4 and run["start_layer"] == 3
    # all three calibration parts disabled: no tone mapper
    st = config.load_settings(text="[PhotometricCalibrationParams]\nresponse_enable = false\n"
                                   "exposure_enable = false\nsensor_bias_enable = false\n")
    assert "tonemap" not in config.trainer_kwargs(st)


@pytest.mark.parametrize("section,key,value", [("Netparams", "decoder_hidden_layers", "2"),
                                               ("Netparams", "decoder_hidden_features", "128"),
                                               ("Netparams", "decoder_activation", "relu"),
                                               ("Netparams", "decoder_skip", "true"),
                                               ("TrainParams", "exex_op", "rms")])
def test_settings_the_step_does_not_implement_are_refused(section, key, value):
    from neat_b200 import config
    st = config.load_settings(text=SETTINGS_TEXT)
    st[section][key] = value
    with pytest.raises(ValueError):
        config.trainer_kwargs(st)
