"""ctypes binding of ``libsplat_cuda.so`` (the C ABI in ``include/splat_cuda.h``).

The library is loaded from this package directory. If it is missing the
import fails loudly: there is no fallback renderer behind this module.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsplat_cuda.so")

SPLAT_OK = 0
SPLAT_ERR_INVALID_ARG = 1
SPLAT_ERR_OOM = 2
SPLAT_ERR_CAPACITY = 3
SPLAT_ERR_DEVICE = 4
SPLAT_ERR_TIMEOUT = 5
SPLAT_ERR_UNSUPPORTED = 6

SPLAT_PRECISION_FP32 = 0
SPLAT_PRECISION_FP16 = 1

SPLAT_OPT_EXACT_BLEND = 1
SPLAT_OPT_PAIR_CAPACITY = 2
SPLAT_OPT_STAGE_EVENTS = 3
SPLAT_OPT_DEBUG_CAPTURE = 4
SPLAT_OPT_FP64_CONICS = 5
SPLAT_OPT_KERNEL_LAUNCHES = 6
SPLAT_OPT_BLEND_CONFIG = 7
SPLAT_OPT_SCENE_SPLATS = 8
SPLAT_OPT_PAIR_LIMIT = 9
SPLAT_OPT_INJECT_FAULT = 10
SPLAT_FAULT_ALLOC = 1
SPLAT_FAULT_LOST_WAIT = 2
SPLAT_OPT_COUNT_EVALS = 11
SPLAT_OPT_BLEND_EVALS = 12
SPLAT_OPT_BBOX_PAIRS = 13

SPLAT_RECORD_BYTES = 48

SPLAT_CELLS_TRUECOLOR = 0
SPLAT_CELLS_ANSI256 = 1

_STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CAPACITY", 4: "DEVICE", 5: "TIMEOUT", 6: "UNSUPPORTED"}

# Every symbol include/splat_cuda.h declares.
EXPORTS = [
    "splat_cuda_abi_version", "splat_cuda_backend_name", "splat_cuda_create", "splat_cuda_create_error",
    "splat_cuda_render", "splat_cuda_render_rows", "splat_cuda_render_device", "splat_cuda_finish",
    "splat_cuda_shard_records", "splat_cuda_render_records",
    "splat_cuda_set_stream",
    "splat_cuda_get_stream", "splat_cuda_set_option", "splat_cuda_get_option", "splat_cuda_debug_dump",
    "splat_cuda_destroy", "splat_cuda_last_error", "splat_cuda_sort_tile_noalloc",
    "splat_cuda_batch_create", "splat_cuda_batch_create_error", "splat_cuda_batch_set_config",
    "splat_cuda_batch_get_config", "splat_cuda_batch_autotune", "splat_cuda_batch_run", "splat_cuda_batch_finish",
    "splat_cuda_batch_set_option", "splat_cuda_batch_get_option", "splat_cuda_batch_set_stream",
    "splat_cuda_batch_get_stream", "splat_cuda_batch_last_error", "splat_cuda_batch_destroy",
    "splat_cuda_create_learned", "splat_cuda_learner_create", "splat_cuda_learner_create_error",
    "splat_cuda_learner_train", "splat_cuda_learner_set_params", "splat_cuda_learner_params",
    "splat_cuda_learner_step_debug", "splat_cuda_learner_directions", "splat_cuda_learner_get_option",
    "splat_cuda_learner_set_option", "splat_cuda_learner_state_bytes", "splat_cuda_learner_save_state",
    "splat_cuda_learner_load_state",
    "splat_cuda_learner_last_error", "splat_cuda_learner_destroy", "splat_cuda_mlp_gradient",
    "splat_cuda_create_from_splat", "splat_cuda_create_from_ply", "splat_cuda_render_cells",
]

# Learned colour (include/splat_cuda.h).
MLP_LATENT = 16
MLP_W1, MLP_W2, MLP_B2, MLP_W3, MLP_B3, MLP_PARAMS = 0, 2048, 6144, 6208, 7232, 7248
LEARN_STEPS_PER_EPOCH = 100
LEARN_SHUFFLE_BITS = 101
LEARN_TRAIN_CTAS = 102


class SplatError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint64), ("sh_degree", ctypes.c_uint32), ("precision", ctypes.c_uint32),
        ("positions", ctypes.c_void_p), ("opacities", ctypes.c_void_p), ("colors", ctypes.c_void_p),
        ("cov3d", ctypes.c_void_p), ("sh_rest", ctypes.c_void_p), ("scales_f16", ctypes.c_void_p),
        ("rotations_f16", ctypes.c_void_p), ("opacities_f16", ctypes.c_void_p), ("sh_f16", ctypes.c_void_p),
    ]


class ViewDesc(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("right", ctypes.c_float * 3), ("down", ctypes.c_float * 3),
                ("forward", ctypes.c_float * 3), ("fov_y", ctypes.c_float), ("near_plane", ctypes.c_float)]


class BatchViewC(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("downsample", ctypes.c_uint32), ("view", ViewDesc), ("bg", ctypes.c_float * 3),
                ("reserved", ctypes.c_uint32), ("dev_out", ctypes.c_void_p)]


class BlendConfigC(ctypes.Structure):
    _fields_ = [("tile_w", ctypes.c_uint32), ("tile_h", ctypes.c_uint32), ("threads", ctypes.c_uint32)]


class TuneResultC(ctypes.Structure):
    _fields_ = [("config", BlendConfigC), ("reserved", ctypes.c_uint32), ("ms", ctypes.c_double)]


class LearnConfigC(ctypes.Structure):
    _fields_ = [("directions", ctypes.c_uint32), ("batch", ctypes.c_uint32), ("lr", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("seed", ctypes.c_uint64)]


class LearnStatsC(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("epochs", ctypes.c_double), ("mean_loss", ctypes.c_double),
                ("last_loss", ctypes.c_double), ("ms", ctypes.c_double), ("steps_per_epoch", ctypes.c_uint64),
                ("samples_per_epoch", ctypes.c_uint64)]


class RenderStatsC(ctypes.Structure):
    _fields_ = [("visible", ctypes.c_uint64), ("overlaps", ctypes.c_uint64), ("project_ms", ctypes.c_double),
                ("sort_ms", ctypes.c_double), ("raster_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m splat_b200.build` "
                              "(the CUDA backend has no fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, f32p = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)
        L.splat_cuda_abi_version.restype = ctypes.c_int
        L.splat_cuda_backend_name.restype = ctypes.c_char_p
        L.splat_cuda_create.argtypes = [ctypes.POINTER(SceneDesc), ctypes.c_int, ctypes.POINTER(vp)]
        L.splat_cuda_create_error.restype = ctypes.c_char_p
        L.splat_cuda_render.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, f32p, u32, vp, ctypes.c_size_t,
                                        ctypes.POINTER(RenderStatsC)]
        L.splat_cuda_render_rows.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, f32p, u32, u32, vp,
                                             ctypes.c_size_t, ctypes.POINTER(RenderStatsC)]
        L.splat_cuda_render_device.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, f32p, u32, vp,
                                               ctypes.c_size_t]
        L.splat_cuda_shard_records.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, u32, ctypes.POINTER(u32),
                                               vp, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.splat_cuda_render_records.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, f32p, vp, u64, u32, u32,
                                                vp, ctypes.c_size_t, ctypes.POINTER(RenderStatsC)]
        L.splat_cuda_finish.argtypes = [vp, ctypes.POINTER(RenderStatsC), ctypes.POINTER(ctypes.c_int)]
        L.splat_cuda_set_stream.argtypes = [vp, vp]
        L.splat_cuda_get_stream.argtypes = [vp]
        L.splat_cuda_get_stream.restype = vp
        L.splat_cuda_set_option.argtypes = [vp, u32, u64]
        L.splat_cuda_get_option.argtypes = [vp, u32, ctypes.POINTER(u64)]
        L.splat_cuda_debug_dump.argtypes = [vp, vp, vp, vp, vp, vp, u64, vp, u64, ctypes.POINTER(u64)]
        L.splat_cuda_destroy.argtypes = [vp]
        L.splat_cuda_sort_tile_noalloc.argtypes = [vp, u32, vp]
        L.splat_cuda_last_error.argtypes = [vp]
        L.splat_cuda_last_error.restype = ctypes.c_char_p
        L.splat_cuda_batch_create.argtypes = [ctypes.POINTER(vp), u32, ctypes.POINTER(BatchViewC), u32,
                                              ctypes.POINTER(vp)]
        L.splat_cuda_batch_create_error.restype = ctypes.c_char_p
        L.splat_cuda_batch_set_config.argtypes = [vp, ctypes.POINTER(BlendConfigC)]
        L.splat_cuda_batch_get_config.argtypes = [vp, ctypes.POINTER(BlendConfigC)]
        L.splat_cuda_batch_autotune.argtypes = [vp, u32, ctypes.POINTER(TuneResultC), u32, ctypes.POINTER(u32)]
        L.splat_cuda_batch_run.argtypes = [vp]
        L.splat_cuda_batch_finish.argtypes = [vp, ctypes.POINTER(RenderStatsC), ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_int)]
        L.splat_cuda_batch_set_option.argtypes = [vp, u32, u64]
        L.splat_cuda_batch_get_option.argtypes = [vp, u32, ctypes.POINTER(u64)]
        L.splat_cuda_batch_set_stream.argtypes = [vp, vp]
        L.splat_cuda_batch_get_stream.argtypes = [vp]
        L.splat_cuda_batch_get_stream.restype = vp
        L.splat_cuda_batch_last_error.argtypes = [vp]
        L.splat_cuda_batch_last_error.restype = ctypes.c_char_p
        L.splat_cuda_batch_destroy.argtypes = [vp]
        L.splat_cuda_render_cells.argtypes = [vp, ctypes.POINTER(ViewDesc), u32, u32, f32p, u32, u32, vp,
                                              ctypes.c_size_t, ctypes.POINTER(u32), ctypes.POINTER(u32),
                                              ctypes.POINTER(RenderStatsC)]
        L.splat_cuda_create_from_splat.argtypes = [vp, ctypes.c_size_t, u32, ctypes.c_int, ctypes.POINTER(vp)]
        L.splat_cuda_create_from_ply.argtypes = [vp, ctypes.c_size_t, u32, ctypes.c_int, ctypes.POINTER(vp)]
        L.splat_cuda_create_learned.argtypes = [ctypes.POINTER(SceneDesc), vp, vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.splat_cuda_learner_create.argtypes = [vp, ctypes.POINTER(LearnConfigC), ctypes.POINTER(vp)]
        L.splat_cuda_learner_create_error.restype = ctypes.c_char_p
        L.splat_cuda_learner_train.argtypes = [vp, u64, ctypes.POINTER(LearnStatsC)]
        L.splat_cuda_learner_set_params.argtypes = [vp, vp, vp]
        L.splat_cuda_learner_params.argtypes = [vp, vp, vp, vp, vp]
        L.splat_cuda_learner_step_debug.argtypes = [vp, vp, vp]
        L.splat_cuda_learner_directions.argtypes = [vp, vp]
        L.splat_cuda_learner_get_option.argtypes = [vp, u32, ctypes.POINTER(u64)]
        L.splat_cuda_learner_set_option.argtypes = [vp, u32, u64]
        L.splat_cuda_learner_state_bytes.argtypes = [vp]
        L.splat_cuda_learner_state_bytes.restype = ctypes.c_size_t
        L.splat_cuda_learner_save_state.argtypes = [vp, vp, ctypes.c_size_t]
        L.splat_cuda_learner_load_state.argtypes = [vp, vp, ctypes.c_size_t]
        L.splat_cuda_learner_last_error.argtypes = [vp]
        L.splat_cuda_learner_last_error.restype = ctypes.c_char_p
        L.splat_cuda_learner_destroy.argtypes = [vp]
        L.splat_cuda_mlp_gradient.argtypes = [ctypes.c_int, vp, vp, vp, vp, u32, vp, vp, vp,
                                              ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def check(rc: int, handle=None, what: str = "", batch=None):
    if rc != SPLAT_OK:
        if handle:
            msg = lib().splat_cuda_last_error(handle).decode()
        elif batch:
            msg = lib().splat_cuda_batch_last_error(batch).decode()
        else:
            msg = ""
        raise SplatError(rc, f"{what}: {msg}" if what else msg)


def pack_blend_config(tile_w: int, tile_h: int, threads: int) -> int:
    """SPLAT_OPT_BLEND_CONFIG value."""
    return int(tile_w) | (int(tile_h) << 8) | (int(threads) << 16)


BLEND_CONFIGS = [(16, 16, 256), (16, 16, 128), (16, 16, 512), (8, 8, 128), (8, 8, 256), (8, 8, 512),
                 (32, 16, 128), (32, 16, 256), (32, 16, 512)]
