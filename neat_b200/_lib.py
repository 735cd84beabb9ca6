"""ctypes bindings of libneat_b200.so (the C ABI declared in include/neat_b200.h).

The shared library is built in-tree by neat_b200/csrc/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libneat_b200.so")
TORCH_SHIM_PATH = os.path.join(_HERE, "libneat_torch.so")

NEAT_OK = 0
NEAT_ERR_BAD_INPUT = 1
NEAT_ERR_CAPACITY = 2
NEAT_ERR_TOO_MANY_HITS = 4
NEAT_ERR_NON_DYADIC = 8
NEAT_ERR_CUDA = 16
NEAT_ERR_UNSUPPORTED = 32
NEAT_ERR_TIMEOUT = 64
NEAT_DECODER_SIMT_FP32 = 0
NEAT_DECODER_TC_BF16X3 = 1
NEAT_DECODER_TC_BF16 = 2
NEAT_MAX_HITS_PER_RAY = 256
NEAT_HIDDEN = 64
NEAT_NOALLOC_MAX_RAYS = 1 << 18

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_int64 = ctypes.c_int64
c_uint64 = ctypes.c_uint64
c_uint32 = ctypes.c_uint32
c_float = ctypes.c_float
c_size_t = ctypes.c_size_t


class StepDesc(ctypes.Structure):
    _fields_ = [
        ("tree_table", c_void_p), ("num_active", c_int), ("max_depth", c_int),
        ("node_min", c_void_p), ("node_max", c_void_p),
        ("w", c_int), ("h", c_int),
        ("intrinsics", c_void_p), ("rotation", c_void_p), ("translation", c_void_p),
        ("C", c_int), ("G", c_int), ("softplus_beta", c_float), ("max_samples_per_node", c_int),
        ("lr_grid", c_float), ("lr_decoder", c_float), ("beta1", c_float), ("beta2", c_float), ("eps", c_float),
        ("seg_capacity", c_int64), ("decoder_path", c_int), ("proposal", c_int), ("pose_grad", c_int),
        ("record_samples_per_ray", c_int), ("cell_node", c_void_p),
    ]


NEAT_PROPOSAL_OFF, NEAT_PROPOSAL_SAMPLE, NEAT_PROPOSAL_TRAIN = 0, 1, 2
NEAT_PROPOSAL_IN, NEAT_PROPOSAL_HIDDEN, NEAT_PROPOSAL_BINS = 16, 32, 8


class Proposal(ctypes.Structure):
    _fields_ = [("mode", c_int), ("params", c_void_p), ("m", c_void_p), ("v", c_void_p), ("grad", c_void_p),
                ("step_counter", c_void_p), ("loss", c_void_p), ("lr", c_float), ("beta1", c_float),
                ("beta2", c_float), ("eps", c_float), ("mix", c_float), ("iters", c_int), ("node_desc", c_void_p),
                ("count_eps", c_float), ("count_min", c_int)]


NEAT_RESPONSE_PARAMS = 25


class ToneMap(ctypes.Structure):
    _fields_ = [("exposure", c_int), ("exposure_mult", c_int), ("sensor_bias", c_int), ("response", c_int),
                ("num_images", c_int), ("bias_w", c_int), ("bias_h", c_int), ("response_range", c_float),
                ("lr_exposure", c_float), ("lr_sensor_bias", c_float), ("lr_response", c_float),
                ("params", c_void_p), ("grad", c_void_p), ("param_loss", c_void_p)]


class PoseGrad(ctypes.Structure):
    _fields_ = [("grad_tangent", c_void_p), ("grad_translation", c_void_p), ("grad_intrinsics", c_void_p),
                ("num_images", c_int)]


class StepState(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("grid", "grid_m", "grid_v", "grid_grad",
                                        "decoder", "decoder_m", "decoder_v", "decoder_grad", "step_counter",
                                        "proposal", "grid_bf16", "tonemap", "pose")]


class StepBatch(ctypes.Structure):
    _fields_ = [("uv", c_void_p), ("image_id", c_void_p), ("target", c_void_p), ("num_rays", c_int64)]


class StepOut(ctypes.Structure):
    _fields_ = [("loss", c_void_p), ("counters", c_void_p), ("status", c_void_p), ("prediction", c_void_p),
                ("phase_events", c_void_p)]


NEAT_STEP_PHASES = 6


class ProjectOut(ctypes.Structure):
    _fields_ = [("prediction", c_void_p), ("error_sums", c_void_p), ("counters", c_void_p), ("status", c_void_p),
                ("tonemap", c_void_p)]


# name -> (restype, argtypes)
_SIGS = {
    "neat_status_string": (ctypes.c_char_p, [c_int]),
    "neat_version": (c_int, []),
    "neat_make_rays": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p]),
    "neat_tree_table_bytes": (c_size_t, [c_int]),
    "neat_tree_prepare": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "neat_samples_workspace_bytes": (c_size_t, [c_int64]),
    "neat_create_samples": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_int64, c_int, c_int, c_uint64,
                                    c_uint32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_create_samples_noalloc": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_int64, c_int, c_int,
                                            c_uint64, c_uint32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_local_samples": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_igs_forward": (c_int, [c_void_p, c_int64, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_int64,
                                 c_void_p, c_void_p]),
    "neat_igs_backward": (c_int, [c_void_p, c_int64, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_int64,
                                  c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_pose_sgd": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.POINTER(PoseGrad), ctypes.c_double,
                              ctypes.c_double, c_int, c_int, c_void_p]),
    "neat_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_float, c_float, c_float, c_float, c_int,
                          c_int, c_void_p]),
    "neat_decoder_params": (c_int64, [c_int]),
    "neat_compute_image_forward": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_float, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                                           c_void_p]),
    "neat_compute_image_backward": (c_int, [c_void_p, c_int64, c_int, c_int, c_void_p, c_float, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                                            c_void_p, c_void_p, c_void_p]),
    "neat_train_step_workspace_bytes": (c_size_t, [ctypes.POINTER(StepDesc), c_int64]),
    "neat_train_step": (c_int, [ctypes.POINTER(StepDesc), ctypes.POINTER(StepState), ctypes.POINTER(StepBatch),
                                c_uint64, c_int, ctypes.POINTER(StepOut), c_void_p, c_size_t, c_void_p]),
    "neat_train_step_prebuilt": (c_int, [ctypes.POINTER(StepDesc), ctypes.POINTER(StepState),
                                         ctypes.POINTER(StepBatch), c_uint64, c_int, ctypes.POINTER(StepOut), c_void_p,
                                         c_size_t, c_void_p]),
    "neat_train_step_segments": (c_int, [ctypes.POINTER(StepDesc), c_void_p, ctypes.POINTER(StepBatch), c_void_p,
                                         c_void_p, c_void_p, c_size_t, c_void_p]),
    "neat_project": (c_int, [ctypes.POINTER(StepDesc), c_void_p, c_void_p, c_void_p, ctypes.POINTER(StepBatch),
                             ctypes.POINTER(ProjectOut), c_void_p, c_size_t, c_void_p]),
    "neat_proposal_params": (c_int64, []),
    "neat_regularizer_workspace_bytes": (c_size_t, []),
    "neat_node_max_density": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p,
                                      c_float, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p]),
    "neat_interpolate_grid": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int64, c_void_p,
                                      c_int, c_int, c_void_p, c_void_p]),
    "neat_tv_loss": (c_int, [c_void_p, c_int64, c_int, c_int, c_float, c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_edge_loss": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int, c_int,
                               c_float, c_float, c_uint64, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_sample_volume": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p,
                                   c_float, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "neat_grid_to_channel_last": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p]),
    "neat_grid_from_channel_last": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p]),
    "neat_synth_project": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p]),
    "neat_synth_density": (c_int, [c_void_p, c_int, c_void_p, c_int64, c_void_p, c_void_p]),
}

_lib = None


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m neat_b200.csrc.build` (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


_torch_ops = None

# operators the libtorch shim registers (namespace "neat"); each runs the C++
# API of neat_b200/shim/neat_torch.h
TORCH_OPS = ("IndirectGridSample3D", "GetRays", "CreateSamplesForRays", "ComputeLocalSamples", "ComputeImage",
             "AdamSteps")


def load_torch_ops():
    """Load the libtorch shim (libneat_torch.so) into this process and return
    torch.ops.neat; raises if it was not built."""
    global _torch_ops
    if _torch_ops is not None:
        return _torch_ops
    import torch
    if not os.path.exists(TORCH_SHIM_PATH):
        raise RuntimeError(f"{TORCH_SHIM_PATH} is missing: build it with `python -m neat_b200.csrc.build`")
    load()
    torch.ops.load_library(TORCH_SHIM_PATH)
    _torch_ops = torch.ops.neat
    return _torch_ops


class NeatError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = load().neat_status_string(status).decode()
        super().__init__(f"{where}: neat status {status} ({msg})" if where else f"neat status {status} ({msg})")


def check(status, where=""):
    if status != NEAT_OK:
        raise NeatError(status, where)
