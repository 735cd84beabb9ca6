"""The reference's INI experiment settings for the fused training step.

NeAT reads its settings with saiga's ParamsBase from INI sections
[TrainParams], [Netparams], [OctreeParams] and [PhotometricCalibrationParams]
(src/Settings.h:26-284, src/modules/ToneMapper.h:13-48; sample file
configs/pepper.ini).  `load_settings` reads such a file with the same section
and key names, and `trainer_kwargs` maps the keys the training step uses to
`FusedTrainer` arguments:

    [Netparams]      grid_features -> num_features, grid_size, softplus_beta,
                     decoder_lr -> lr_decoder (geometry.cpp:90-97)
    [TrainParams]    lr_exex_grid_adam -> lr_grid (geometry_ex_ex.cpp:40-50),
                     random_seed -> seed, loss_tv, loss_edge, optimize_pose,
                     optimize_intrinsics, lr_pose, lr_intrinsics
    [OctreeParams]   max_samples_per_node
    [PhotometricCalibrationParams]  every key, as the tonemap dict

`run_settings` returns the rest of what a training loop needs (batch_size,
train_interval_jitter, tree_depth, start_layer).  Settings the fused step does
not implement raise ValueError rather than being silently ignored: a decoder
other than Linear(C,64)-SiLU-Linear(64,64)-SiLU-Linear(64,1)-softplus, a
grid optimizer other than Adam, or decoder skip connections.

A key that is absent takes the reference's default from its struct
initialisers: Netparams, OctreeParams and MyTrainParams in src/Settings.h
(e.g. loss_tv 1e-4, loss_edge 1e-3, optimize_pose and optimize_intrinsics on,
start_layer 3) and PhotometricCalibrationParams in src/modules/ToneMapper.h:36-47
(response, exposure and sensor bias all enabled, so an absent section still
calibrates).  batch_size and train_interval_jitter belong to saiga's
TrainParams base, whose source is not in the reference; their defaults here are
the values of configs/pepper.ini (16000, true).
"""
import configparser

SECTIONS = ("TrainParams", "Netparams", "OctreeParams", "PhotometricCalibrationParams")
TONEMAP_KEYS = ("response_enable", "response_range", "response_lr", "exposure_enable", "exposure_mult",
                "exposure_lr", "sensor_bias_enable", "sensor_bias_size_w", "sensor_bias_lr")
# PhotometricCalibrationParams initialisers (src/modules/ToneMapper.h:36-47)
TONEMAP_DEFAULTS = {"response_enable": True, "response_range": 2.0, "response_lr": 0.1, "exposure_enable": True,
                    "exposure_mult": False, "exposure_lr": 0.01, "sensor_bias_enable": True,
                    "sensor_bias_size_w": 32, "sensor_bias_lr": 0.05}


def load_settings(path=None, text=None):
    """Sections of an INI settings file (or text) as {section: {key: str}};
    keys keep their case and dotted names."""
    cp = configparser.ConfigParser(interpolation=None, strict=False)
    cp.optionxform = str
    if text is not None:
        cp.read_string(text)
    else:
        with open(path) as f:
            cp.read_file(f)
    return {s: dict(cp.items(s)) for s in cp.sections()}


def _bool(v):
    s = str(v).strip().lower()
    if s in ("1", "true", "yes", "on"):
        return True
    if s in ("0", "false", "no", "off", ""):
        return False
    raise ValueError(f"not a boolean: {v!r}")


def _get(settings, section, key, conv, default):
    v = settings.get(section, {}).get(key)
    return default if v is None or str(v).strip() == "" else conv(v)


def trainer_kwargs(settings):
    """FusedTrainer keyword arguments from the settings (the reference's
    defaults where a key is absent)."""
    net = settings.get("Netparams", {})
    if _get(settings, "Netparams", "decoder_hidden_layers", int, 1) != 1:
        raise ValueError("the fused step implements one hidden layer pair (decoder_hidden_layers = 1)")
    if _get(settings, "Netparams", "decoder_hidden_features", int, 64) != 64:
        raise ValueError("the fused step implements 64 hidden features")
    if str(net.get("decoder_activation", "silu")).strip().lower() != "silu":
        raise ValueError("the fused step implements decoder_activation = silu")
    if str(net.get("last_activation_function", "softplus")).strip().lower() != "softplus":
        raise ValueError("the fused step implements last_activation_function = softplus")
    if _get(settings, "Netparams", "decoder_skip", _bool, False):
        raise ValueError("the fused step has no decoder skip connections")
    opt = str(settings.get("TrainParams", {}).get("exex_op", "adam")).strip().lower()
    if opt != "adam":
        raise ValueError(f"the fused step optimizes the grid with Adam (exex_op = {opt!r})")
    kw = {
        "num_features": _get(settings, "Netparams", "grid_features", int, 4),
        "grid_size": _get(settings, "Netparams", "grid_size", int, 17),
        "softplus_beta": _get(settings, "Netparams", "softplus_beta", float, 2.0),
        "lr_decoder": _get(settings, "Netparams", "decoder_lr", float, 5e-5),
        "lr_grid": _get(settings, "TrainParams", "lr_exex_grid_adam", float, 0.04),
        "max_samples_per_node": _get(settings, "OctreeParams", "max_samples_per_node", int, 32),
        "seed": _get(settings, "TrainParams", "random_seed", int, 0) % (1 << 63),
        "loss_tv": _get(settings, "TrainParams", "loss_tv", float, 1e-4),
        "loss_edge": _get(settings, "TrainParams", "loss_edge", float, 1e-3),
        "optimize_pose": _get(settings, "TrainParams", "optimize_pose", _bool, True),
        "optimize_intrinsics": _get(settings, "TrainParams", "optimize_intrinsics", _bool, True),
        "lr_pose": _get(settings, "TrainParams", "lr_pose", float, 1e-3),
        "lr_intrinsics": _get(settings, "TrainParams", "lr_intrinsics", float, 100.0),
    }
    conv = {k: (_bool if k.endswith(("_enable", "_mult")) else (int if k == "sensor_bias_size_w" else float))
            for k in TONEMAP_KEYS}
    tm = {k: _get(settings, "PhotometricCalibrationParams", k, conv[k], TONEMAP_DEFAULTS[k]) for k in TONEMAP_KEYS}
    if any(tm[k] for k in ("response_enable", "exposure_enable", "sensor_bias_enable")):
        kw["tonemap"] = tm
    return kw


def run_settings(settings):
    """The settings of the training loop around the step."""
    return {
        "batch_size": _get(settings, "TrainParams", "batch_size", int, 16000),
        "train_interval_jitter": _get(settings, "TrainParams", "train_interval_jitter", _bool, True),
        "tree_depth": _get(settings, "OctreeParams", "tree_depth", int, 4),
        "start_layer": _get(settings, "OctreeParams", "start_layer", int, 3),
    }
