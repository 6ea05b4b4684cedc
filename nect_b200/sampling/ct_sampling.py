"""Drop-in for the reference extension module ``nect.sampling.ct_sampling``.

Same four geometry classes (constructor keywords, defaults and read/write
attributes of the pybind11 bindings, nect/sampling/ct_sampling.cu:650-749) and
the same ``sample`` function (:756-807), backed by the sm_100a kernel behind
``nectb_sample`` in libnectb.so.

Differences a caller can observe are none in values: the two random draws
(``rand(R) - 0.5`` and ``(rand(R, 2) - 0.5) * random_detector_offset``, made on
the device's default generator in the reference's order, :619-622) are taken
here with torch and passed to the kernel, so a seeded call reproduces the
reference's jitter exactly.  The call is stream-ordered on torch's current
stream instead of synchronising the whole device (:640), and CUDA errors raise
RuntimeError like the reference (:641-644).
"""
from __future__ import annotations

import ctypes
import struct

import torch

from .. import _lib


def _f32(v) -> float:
    return struct.unpack("f", struct.pack("f", float(v)))[0]


def _required(**kw):
    missing = [k for k, v in kw.items() if v is None]
    if missing:
        raise TypeError(f"missing required argument(s): {', '.join(missing)}")


class _GeometryBase:
    _kind = -1
    _scalar = {
        "COR": "COR",
        "distance_source_to_origin": "distance_source_to_origin",
        "distance_origin_to_detector": "distance_origin_to_detector",
        "object_radius": "object_radius",
        "object_height": "object_height",
        "remove_factor_top": "remove_factor_top",
        "remove_factor_bottom": "remove_factor_bottom",
    }
    _tuples = {"nDetector": 2, "dDetector": 2, "offOrigin": 3, "offDetector": 2, "rotDetector": 3, "sVoxel": 3,
               "dVoxel": 3}
    _fields: tuple[str, ...] = ()

    def __init__(self, **kw):
        object.__setattr__(self, "_c", _lib.NectbGeometry())
        self._c.kind = self._kind
        for name in self._fields:
            setattr(self, name, kw[name])

    def __setattr__(self, name, value):
        if name in self._fields:
            if name in self._tuples:
                n = self._tuples[name]
                vals = tuple(value)
                if len(vals) != n:
                    raise TypeError(f"{name} expects a tuple of {n} values")
                arr = getattr(self._c, name)
                for i, v in enumerate(vals):
                    arr[i] = int(v) if name == "nDetector" else float(v)
            else:
                setattr(self._c, name, float(value))
            return
        object.__setattr__(self, name, value)

    def __getattr__(self, name):
        c = object.__getattribute__(self, "_c")
        if name in type(self)._fields:
            if name in type(self)._tuples:
                arr = getattr(c, name)
                return tuple(int(x) if name == "nDetector" else _f32(x) for x in arr)
            return _f32(getattr(c, name))
        raise AttributeError(name)

    @property
    def c_struct(self) -> _lib.NectbGeometry:
        return self._c

    def __repr__(self):
        body = ", ".join(f"{k}={getattr(self, k)!r}" for k in self._fields)
        return f"{type(self).__name__}({body})"


class ConeGeometryVoxel(_GeometryBase):
    _kind = _lib.CONE_VOXEL
    _fields = ("distance_source_to_origin", "distance_origin_to_detector", "nDetector", "dDetector", "offOrigin",
               "offDetector", "rotDetector", "COR", "sVoxel", "dVoxel")

    def __init__(self, distance_source_to_origin, distance_origin_to_detector, nDetector, dDetector,
                 offOrigin=(0.0, 0.0, 0.0), offDetector=(0.0, 0.0), rotDetector=(0.0, 0.0, 0.0), COR=0.0,
                 sVoxel=None, dVoxel=None):
        _required(sVoxel=sVoxel, dVoxel=dVoxel)
        super().__init__(**{k: v for k, v in locals().items() if k in self._fields})


class ParallelGeometryVoxel(_GeometryBase):
    _kind = _lib.PARALLEL_VOXEL
    _fields = ("nDetector", "dDetector", "offOrigin", "offDetector", "rotDetector", "COR", "sVoxel", "dVoxel")

    def __init__(self, nDetector, dDetector, offOrigin=(0.0, 0.0, 0.0), offDetector=(0.0, 0.0),
                 rotDetector=(0.0, 0.0, 0.0), COR=0.0, sVoxel=None, dVoxel=None):
        _required(sVoxel=sVoxel, dVoxel=dVoxel)
        super().__init__(**{k: v for k, v in locals().items() if k in self._fields})


class ConeGeometryCylindrical(_GeometryBase):
    _kind = _lib.CONE_CYLINDRICAL
    _fields = ("distance_source_to_origin", "distance_origin_to_detector", "nDetector", "dDetector", "offOrigin",
               "offDetector", "rotDetector", "COR", "object_radius", "object_height", "remove_factor_top",
               "remove_factor_bottom")

    def __init__(self, distance_source_to_origin, distance_origin_to_detector, nDetector, dDetector,
                 offOrigin=(0.0, 0.0, 0.0), offDetector=(0.0, 0.0), rotDetector=(0.0, 0.0, 0.0), COR=0.0,
                 object_radius=None, object_height=None, remove_factor_top=0.0, remove_factor_bottom=0.0):
        _required(object_radius=object_radius, object_height=object_height)
        super().__init__(**{k: v for k, v in locals().items() if k in self._fields})


class ParallelGeometryCylindrical(_GeometryBase):
    _kind = _lib.PARALLEL_CYLINDRICAL
    _fields = ("nDetector", "dDetector", "object_radius", "object_height", "offOrigin", "offDetector", "rotDetector",
               "COR", "remove_factor_top", "remove_factor_bottom")

    def __init__(self, nDetector, dDetector, object_radius, object_height, offOrigin=(0.0, 0.0, 0.0),
                 offDetector=(0.0, 0.0), rotDetector=(0.0, 0.0, 0.0), COR=0.0, remove_factor_top=0.0,
                 remove_factor_bottom=0.0):
        super().__init__(**{k: v for k, v in locals().items() if k in self._fields})


GeometryTypes = (ConeGeometryVoxel, ParallelGeometryVoxel, ConeGeometryCylindrical, ParallelGeometryCylindrical)


def draw_ray_randoms(num_rays: int, random_detector_offset: float, device: torch.device):
    """The reference's two per-call draws, in its order (ct_sampling.cu:619-622)."""
    jitter = torch.rand(num_rays, device=device, dtype=torch.float32) - 0.5
    det_off = (torch.rand(num_rays, 2, device=device, dtype=torch.float32) - 0.5) * random_detector_offset
    return jitter, det_off


def sample_with_draws(random_ray_index: torch.Tensor, geometry, angle_rad: float, num_points_per_ray: int,
                      num_rays: int, starting_ray_index: int, max_ray_distance_per_point: float,
                      uniform_ray_spacing: bool, jitter: torch.Tensor, detector_offset: torch.Tensor,
                      want_points: bool = True, want_counts: bool = False):
    """``sample`` with the random draws given; returns (points, distances[, counts])."""
    if not isinstance(geometry, GeometryTypes):
        raise TypeError(f"unsupported geometry type {type(geometry).__name__}")
    _lib.require_cuda(random_ray_index, "random_ray_index")
    if random_ray_index.dtype != torch.int64:
        raise TypeError("random_ray_index must be int64")
    dev = random_ray_index.device
    S, R = int(num_points_per_ray), int(num_rays)
    points = torch.empty((R, S, 3), device=dev, dtype=torch.float32) if want_points else None
    distances = torch.empty((R,), device=dev, dtype=torch.float32)
    counts = torch.empty((R,), device=dev, dtype=torch.int32) if want_counts else None
    jitter = jitter.contiguous()
    detector_offset = detector_offset.contiguous()
    rc = _lib.lib.nectb_sample(
        ctypes.byref(geometry.c_struct), random_ray_index.data_ptr(), random_ray_index.numel(),
        int(starting_ray_index), R, S, float(angle_rad), float(max_ray_distance_per_point),
        1 if uniform_ray_spacing else 0, jitter.data_ptr(), detector_offset.data_ptr(), _lib.ptr(points),
        distances.data_ptr(), _lib.ptr(counts), _lib.stream_ptr(dev))
    _lib.check(rc, "nectb_sample")
    if want_counts:
        return points, distances, counts
    return points, distances


def sample(random_ray_index: torch.Tensor, geometry, angle_rad: float, num_points_per_ray: int, num_rays: int,
           starting_ray_index: int, max_ray_distance_per_point: float, uniform_ray_spacing: bool,
           random_detector_offset: float, device: int):
    """Sample points along ``num_rays`` rays (reference ct_sampling.cu:606-648).

    Returns ``points`` fp32 [num_rays, num_points_per_ray, 3] in (z, y, x) order,
    normalised to the unit cube but not yet clamped (the Projector clamps), with
    samples beyond each ray's exit exactly 0, and ``distances`` fp32 [num_rays].
    """
    dev = torch.device("cuda", device)
    if random_ray_index.device != dev:
        raise ValueError(f"random_ray_index is on {random_ray_index.device}, expected {dev}")
    jitter, det_off = draw_ray_randoms(int(num_rays), float(random_detector_offset), dev)
    return sample_with_draws(random_ray_index, geometry, angle_rad, num_points_per_ray, num_rays,
                             starting_ray_index, max_ray_distance_per_point, uniform_ray_spacing, jitter, det_off)
