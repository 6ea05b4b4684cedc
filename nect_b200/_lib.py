"""ctypes binding of libnectb.so (the C ABI declared in include/nectb.h).

The library is the only compute path: if it is missing or fails to load,
importing this module raises, and every op that needs it fails loudly.  There
is no CPU or PyTorch fallback.  ctypes releases the GIL for the duration of
each call; every call is stream-ordered on the stream passed in (torch's
current stream by default) and never synchronises the device.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NECTB_LIB", _PKG / "_lib" / "libnectb.so"))

c_int = ctypes.c_int32
c_i64 = ctypes.c_int64
c_f32 = ctypes.c_float
c_f64 = ctypes.c_double
c_ptr = ctypes.c_void_p
c_size = ctypes.c_size_t

# Geometry kinds (include/nectb.h)
CONE_VOXEL, CONE_CYLINDRICAL, PARALLEL_VOXEL, PARALLEL_CYLINDRICAL = 0, 1, 2, 3
F32, F16, BF16 = 0, 1, 2
ACT = {"none": 0, "relu": 1, "leakyrelu": 2, "softplus": 3, "sigmoid": 4}


class NectbGeometry(ctypes.Structure):
    _fields_ = [
        ("kind", c_int),
        ("nDetector", c_int * 2),
        ("dDetector", c_f32 * 2),
        ("offOrigin", c_f32 * 3),
        ("offDetector", c_f32 * 2),
        ("rotDetector", c_f32 * 3),
        ("COR", c_f32),
        ("distance_source_to_origin", c_f32),
        ("distance_origin_to_detector", c_f32),
        ("sVoxel", c_f32 * 3),
        ("dVoxel", c_f32 * 3),
        ("object_radius", c_f32),
        ("object_height", c_f32),
        ("remove_factor_top", c_f32),
        ("remove_factor_bottom", c_f32),
    ]


class NectbHashGrid(ctypes.Structure):
    _fields_ = [
        ("n_dims", c_int),
        ("n_levels", c_int),
        ("n_features", c_int),
        ("log2_hashmap_size", c_int),
        ("feature_dtype", c_int),
        ("base_resolution", ctypes.c_double),
        ("per_level_scale", ctypes.c_double),
        ("base_resolution_t", ctypes.c_double),
    ]


class NectbMLP(ctypes.Structure):
    _fields_ = [
        ("n_input", c_int),
        ("n_hidden_layers", c_int),
        ("width", c_int),
        ("activation", c_int),
        ("output_activation", c_int),
        ("compute_dtype", c_int),
    ]


class NectbTrainBatch(ctypes.Structure):
    _fields_ = [
        ("random_ray_index", c_ptr),
        ("random_ray_index_len", c_i64),
        ("starting_ray_index", c_i64),
        ("num_rays", c_int),
        ("num_points_per_ray", c_int),
        ("angle_rad", c_f32),
        ("t", c_f32),
        ("max_ray_distance_per_point", c_f32),
        ("uniform_ray_spacing", c_int),
        ("max_distance_traveled", c_f32),
        ("jitter", c_ptr),
        ("detector_offset", c_ptr),
        ("projection", c_ptr),
        ("loss_type", c_int),
        ("loss_scale", c_f32),
    ]


class NectbTuning(ctypes.Structure):
    _fields_ = [
        ("forward_blocks_per_sm", c_int),
        ("backward_blocks_per_sm", c_int),
        ("scatter_blocks_per_sm", c_int),
        ("staged_rounds", c_int),
        ("scatter_group_bytes", c_i64),
        ("run_threshold_3d", c_f32),
        ("run_threshold_4d", c_f32),
        ("time_slice", c_int),
        ("encoding_store", c_int),
    ]


# name -> (restype, argtypes)
_SIGNATURES = {
    "nectb_version": (ctypes.c_char_p, []),
    "nectb_last_error": (ctypes.c_char_p, []),
    "nectb_sample": (
        c_int,
        [ctypes.POINTER(NectbGeometry), c_ptr, c_i64, c_i64, c_int, c_int, c_f32, c_f32, c_int, c_ptr, c_ptr, c_ptr,
         c_ptr, c_ptr, c_ptr],
    ),
    "nectb_hashgrid_layout": (
        c_i64, [ctypes.POINTER(NectbHashGrid), c_ptr, c_ptr, c_ptr, c_ptr, c_ptr]),
    "nectb_mlp_param_count": (c_i64, [ctypes.POINTER(NectbMLP)]),
    "nectb_hashgrid_encode": (c_int, [ctypes.POINTER(NectbHashGrid), c_ptr, c_ptr, c_i64, c_ptr, c_ptr]),
    "nectb_hashgrid_encode_backward": (c_int, [ctypes.POINTER(NectbHashGrid), c_ptr, c_i64, c_ptr, c_ptr, c_ptr]),
    "nectb_hashgrid_corners": (c_int, [ctypes.POINTER(NectbHashGrid), c_ptr, c_i64, c_ptr, c_ptr, c_ptr]),
    "nectb_quadcubes_workspace_bytes": (c_size, [ctypes.POINTER(NectbHashGrid)]),
    "nectb_quadcubes_encode": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), c_ptr, c_ptr, c_i64, c_ptr, c_int, c_ptr, c_i64, c_int, c_ptr, c_size, c_ptr]),
    "nectb_quadcubes_encode_backward": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), c_ptr, c_i64, c_ptr, c_ptr, c_i64, c_int, c_ptr, c_ptr, c_size, c_ptr]),
    "nectb_model_forward": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_i64, c_f32, c_ptr, c_ptr],
    ),
    "nectb_model_forward_t": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_i64, c_ptr, c_ptr, c_ptr],
    ),
    "nectb_model_backward_t": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_i64, c_ptr, c_ptr, c_ptr,
         c_ptr, c_ptr],
    ),
    "nectb_model_backward": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_i64, c_f32, c_ptr, c_ptr,
         c_ptr, c_ptr],
    ),
    "nectb_train_workspace_bytes": (
        c_size, [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_int]),
    "nectb_train_step": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_forward": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_backward": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_ptr, c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_scan_workspace_bytes": (
        c_size, [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_int,
                 c_int]),
    "nectb_train_scan_staging_bytes": (
        c_size, [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_int, c_int,
                 c_int]),
    "nectb_train_scan_step": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_int, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_scan_forward": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_int, c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_scan_backward": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_int, c_ptr, c_ptr, c_ptr, c_ptr, c_size, c_ptr],
    ),
    "nectb_train_scan_error_word": (c_ptr, [ctypes.POINTER(NectbGeometry), c_int, c_int, c_ptr]),
    "nectb_train_step_static": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr,
         ctypes.POINTER(NectbTrainBatch), c_ptr, c_ptr, c_ptr, c_ptr, c_ptr],
    ),
    "nectb_train_static_scratch_bytes": (c_size, []),
    "nectb_query_points": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_int, c_i64, c_ptr, c_int,
         c_ptr],
    ),
    "nectb_time_slice_bytes": (c_size, [ctypes.POINTER(NectbHashGrid)]),
    "nectb_time_slice": (c_int, [ctypes.POINTER(NectbHashGrid), c_ptr, c_f32, c_ptr, c_size, c_ptr]),
    "nectb_query_points_slice": (
        c_int,
        [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_ptr, c_int, c_i64, c_ptr, c_int,
         c_ptr],
    ),
    "nectb_query_reproject": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_f32,
         c_f32, c_int, c_f32, c_f32, c_ptr, c_ptr, c_size, c_int, c_ptr],
    ),
    "nectb_query_reproject_range": (
        c_int,
        [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_ptr, c_ptr, c_f32,
         c_f32, c_int, c_f32, c_f32, c_ptr, c_int, c_int, c_ptr, c_size, c_int, c_int, c_ptr],
    ),
    "nectb_query_reproject_slice_bytes": (c_size, [ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_int]),
    "nectb_train_error_word": (c_ptr, [ctypes.POINTER(NectbGeometry), c_int, c_ptr]),
    "nectb_train_rays": (c_int, [ctypes.POINTER(NectbGeometry), c_int, c_int, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr]),
    "nectb_train_staging_bytes": (
        c_size, [ctypes.POINTER(NectbGeometry), ctypes.POINTER(NectbHashGrid), ctypes.POINTER(NectbMLP), c_int, c_int]),
    "nectb_selftest_bounded_wait": (c_int, [c_ptr, ctypes.c_uint32, c_ptr]),
    "nectb_get_tuning": (c_int, [ctypes.POINTER(NectbTuning)]),
    "nectb_set_tuning": (c_int, [ctypes.POINTER(NectbTuning)]),
    "nectb_profile_enable": (c_int, [c_int]),
    "nectb_profile_collect": (c_int, [c_ptr, c_ptr]),
    "nectb_probe_gather": (c_int, [c_ptr, c_i64, c_int, c_int, c_i64, c_ptr, c_ptr]),
    "nectb_probe_reduce": (c_int, [c_ptr, c_i64, c_int, c_int, c_i64, c_ptr]),
    "nectb_probe_ops": (c_i64, [c_i64]),
    "nectb_adam_step": (
        c_int,
        [c_ptr, c_ptr, c_ptr, c_ptr, c_i64, c_f64, c_f64, c_f64, c_f64, c_f64, c_int, c_ptr, c_int, c_ptr],
    ),
}


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"libnectb.so not found at {LIB_PATH}; build it with `python -m nect_b200.build` "
            "(there is no fallback implementation)"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def exported_symbols() -> list[str]:
    return [n for n in _SIGNATURES if hasattr(lib, n)]


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.nectb_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed (status {rc}): {msg}")


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the B200 path has no CPU implementation)")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
