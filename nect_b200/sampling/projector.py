"""Ray batches of one projection, behind the reference's ``Projector`` interface.

The reference's projector (nect/sampling/projector.py:35-131) is the object
its trainer asks for "the points and measured values of batch k of the
current projection".  This module keeps that contract: the constructor
arguments, ``update``/``update_angle``/``set_geometry``/``to_dict``, the
attributes a trainer reads (``batch_size``, ``batch_per_epoch``,
``random_indexes``, ``distance_between_points``, ``distances``) and
``__call__(batch_num, proj) -> (points [R, S, 3] clamped to [0, 1],
proj[perm[batch]])``.

Inside, the pixel order is one device permutation per ``update``, the batch
windows come from ``batching`` (shared with the fused trainer's
``make_batch``), and the points come from the sm_100a sampler.  The fused
training path never materialises points; ``ray_batch`` hands it the same
batch as arguments.
"""
from __future__ import annotations

import torch

from . import batching, ct_sampling
from .geometry import Geometry


def resolve_cuda_device(device) -> torch.device:
    """The CUDA device named by an index, "cuda", "cuda:N" or a torch.device.

    Raises ValueError when CUDA is absent, the name is not a CUDA device, or
    the index is not one of the visible devices."""
    if not torch.cuda.is_available():
        raise ValueError("no CUDA device is visible: the projector samples on the GPU")
    try:
        dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    except (RuntimeError, TypeError) as e:
        raise ValueError(f"cannot read {device!r} as a device: {e}") from None
    if dev.type != "cuda":
        raise ValueError(f"{device!r} is a {dev.type} device; the projector needs a CUDA device")
    index = 0 if dev.index is None else dev.index
    visible = torch.cuda.device_count()
    if not 0 <= index < visible:
        raise ValueError(f"{device!r} asks for CUDA device {index}, but only devices 0..{visible - 1} are visible")
    return torch.device("cuda", index)


class Projector:
    """Batches of sampled rays over one projection at a time."""

    def __init__(self, geometry: Geometry, points_per_batch: int, points_per_ray: int, device,
                 random_offset_detector: float = 0.0, uniform_ray_spacing: bool = True):
        if points_per_ray < 1:
            raise ValueError(f"points_per_ray must be at least 1, got {points_per_ray}")
        if points_per_batch < points_per_ray:
            raise ValueError(f"a batch of {points_per_batch} points cannot hold one ray of {points_per_ray} points")
        self.device = resolve_cuda_device(device)
        self.points_per_batch = points_per_batch
        self.points_per_ray = points_per_ray
        self.random_offset_detector = random_offset_detector
        self.uniform_ray_spacing = uniform_ray_spacing
        self.set_geometry(geometry)

    def set_geometry(self, geometry: Geometry) -> None:
        self.geometry = geometry
        self.c_geometry = geometry.get_c_geometry()

    def to_dict(self) -> dict:
        return dict(geometry=self.geometry.to_dict(), points_per_batch=self.points_per_batch,
                    reconstruction_mode=self.geometry.reconstruction_mode, points_per_ray=self.points_per_ray,
                    uniform_ray_spacing=self.uniform_ray_spacing)

    def update(self, angle: float, detector_binning: int | None = None, points_per_ray: int | None = None,
               random_offset_detector: float | None = None, uniform_ray_spacing: bool | None = None) -> None:
        """Start a new projection: optional setting changes, then a fresh
        pixel permutation at this angle."""
        if detector_binning is not None:
            self.geometry.set_detector_binning(detector_binning)
            self.set_geometry(self.geometry)
        for name, value in (("points_per_ray", points_per_ray), ("random_offset_detector", random_offset_detector),
                            ("uniform_ray_spacing", uniform_ray_spacing)):
            if value is not None:
                setattr(self, name, value)
        rows, cols = (n // self.geometry.detector_binning for n in self.geometry.nDetector)
        self.total_detector_pixels = rows * cols
        self.batch_size = batching.rays_per_batch(self.points_per_batch, self.points_per_ray)
        self.batch_per_epoch = batching.batches_per_projection(self.total_detector_pixels, self.batch_size)
        self.distance_between_points = self.geometry.max_distance_traveled / self.points_per_ray
        self.random_indexes = torch.randperm(self.total_detector_pixels, dtype=torch.int64, device=self.device)
        self.angle = angle

    def update_angle(self, angle: float) -> None:
        """Same pixels, another angle (the continuous-scan sub-angles)."""
        self.angle = angle

    def batch_range(self, batch_num: int) -> tuple[int, int] | None:
        """(starting_ray_index, rays) of batch ``batch_num``; None past the end."""
        return batching.batch_window(self.random_indexes.numel(), self.batch_size, batch_num)

    def __call__(self, batch_num: int, proj: torch.Tensor):
        window = self.batch_range(batch_num)
        if window is None:
            return None, None
        start, rays = window
        points, self.distances = ct_sampling.sample(
            random_ray_index=self.random_indexes, geometry=self.c_geometry, angle_rad=self.angle,
            num_points_per_ray=self.points_per_ray, num_rays=rays, starting_ray_index=start,
            max_ray_distance_per_point=self.distance_between_points, uniform_ray_spacing=self.uniform_ray_spacing,
            random_detector_offset=self.random_offset_detector, device=self.device.index)
        points.clamp_(0.0, 1.0)
        return points, proj[self.random_indexes[start:start + rays]]
