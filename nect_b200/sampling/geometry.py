"""Acquisition geometry with the reference's constructor, attributes and rules.

Mirrors ``nect.sampling.geometry.Geometry`` (nect/sampling/geometry.py:26-407):
the same arguments and validation errors, the derived ``sVoxel``,
``max_distance_traveled`` (:156-174) and ``sDetector``, YAML/config loaders and
``get_c_geometry`` (:322-407), which here returns the geometry objects of
``nect_b200.sampling.ct_sampling`` so the B200 sampler receives it.
"""
from __future__ import annotations

from pathlib import Path
from warnings import warn

import numpy as np
import torch
import yaml

from . import ct_sampling


def _as_tuple(t, length: int, var_name: str, mode: str):
    if t is None:
        if var_name in "Detector":
            raise ValueError(f"{var_name} is required")
        raise ValueError(f"{var_name} is required for {mode} reconstruction")
    if isinstance(t, (list, tuple)):
        if len(t) != length:
            raise ValueError(f"{var_name} should have {length} elements")
    elif isinstance(t, (np.ndarray, torch.Tensor)):
        if tuple(t.shape) != (length,):
            raise ValueError(f"{var_name} should have {length} elements")
    return tuple(t[i] for i in range(length))


def _as_floats(t, length, var_name, mode):
    t = _as_tuple(t, length, var_name, mode)
    out = []
    for i in range(length):
        v = t[i]
        if isinstance(v, (np.generic, torch.Tensor)):
            v = v.item()
        if not isinstance(v, (float, int)):
            raise ValueError(f"{var_name}[{i}] should be a float")
        out.append(float(v))
    return tuple(out)


def _as_ints(t, length, var_name, mode):
    t = _as_tuple(t, length, var_name, mode)
    vals = [v.item() if isinstance(v, (np.generic, torch.Tensor)) else v for v in t]
    # The reference validates the first element only (geometry.py:416-425).
    v0 = vals[0]
    if not isinstance(v0, int):
        if not (isinstance(v0, float) and v0.is_integer()):
            raise ValueError(f"{var_name}[0] should be an integer")
    return tuple(int(v) for v in vals)


class Geometry:
    """CT acquisition geometry (see the reference docstring, geometry.py:48-90)."""

    def __init__(self, nDetector, dDetector, mode: str, DSD: float | None = None, DSO: float | None = None,
                 nVoxel=None, dVoxel=None, radius: float | None = None, height: float | None = None,
                 offOrigin=(0.0, 0.0, 0.0), COR: float = 0.0, offDetector=(0.0, 0.0), rotDetector=(0.0, 0.0, 0.0),
                 reconstruction_mode: str = "voxel", detector_binning: int = 1, angles=None, radians: bool = True,
                 timesteps=None):
        if mode not in ("cone", "parallel"):
            raise ValueError(f"Unsupported mode '{mode}'")
        if mode == "cone":
            if DSD is None:
                raise ValueError("DSD is required for cone geometry")
            if DSO is None:
                raise ValueError("DSO is required for cone geometry")
            self.DSD, self.DSO = float(DSD), float(DSO)
        else:
            if DSD is not None:
                warn("DSD is not required for parallel geometry. Ignoring the value of DSD")
            if DSO is not None:
                warn("DSO is not required for parallel geometry. Ignoring the value of DSO")
            self.DSD = self.DSO = None
        if reconstruction_mode not in ("voxel", "cylindrical"):
            raise ValueError(f"Unsupported reconstruction mode '{reconstruction_mode}'")
        self.mode = mode
        self.reconstruction_mode = reconstruction_mode
        self.detector_binning = detector_binning
        rm = reconstruction_mode
        self.dDetector = _as_floats(dDetector, 2, "dDetector", rm)
        self.nDetector = _as_ints(nDetector, 2, "nDetector", rm)
        self.offDetector = _as_floats(offDetector, 2, "offDetector", rm)
        self.rotDetector = _as_floats(rotDetector, 3, "rotDetector", rm)
        self.COR = COR
        self.set_angles(angles, radians)
        self.set_timesteps(timesteps)
        if radius is None or height is None:
            self.nVoxel = _as_ints(nVoxel, 3, "nVoxel", rm)
            self.dVoxel = _as_floats(dVoxel, 3, "dVoxel", rm)
            self.sVoxel = tuple(self.nVoxel[i] * self.dVoxel[i] for i in range(3))
            self.offOrigin = _as_floats(offOrigin, 3, "offOrigin", rm)
            if rm == "cylindrical":
                # the reference only fills the values that were not given (geometry.py:128-132)
                self.radius = max(self.sVoxel[1], self.sVoxel[2]) / 2 if radius is None else radius
                self.height = self.sVoxel[0] if height is None else height
            else:
                self.radius = None
                self.height = None
        else:
            self.radius = radius
            self.height = height
            self.nVoxel = (_as_ints(nVoxel, 3, "nVoxel", rm) if nVoxel is not None
                           else (self.nDetector[0], self.nDetector[1], self.nDetector[1]))
            self.dVoxel = (_as_floats(dVoxel, 3, "dVoxel", rm) if dVoxel is not None
                           else (self.nDetector[0] / height, self.nDetector[1] / (2 * radius),
                                 self.nDetector[1] / (2 * radius)))
            self.sVoxel = tuple(self.nVoxel[i] * self.dVoxel[i] for i in range(3))
        self.max_distance_traveled = self._max_distance(nVoxel, dVoxel)
        self.sDetector = (self.nDetector[0] * self.dDetector[0], self.nDetector[1] * self.dDetector[1])

    def _max_distance(self, nVoxel, dVoxel) -> float:
        """Longest chord a ray can travel through the object (geometry.py:156-174)."""
        sv, dv = self.sVoxel, self.dVoxel
        if self.mode == "cone":
            if (nVoxel is None or dVoxel is None) and self.reconstruction_mode == "cylindrical":
                length = self.radius * 2
                theta = np.arctan((self.height / 2) / (self.DSO + length / 2))
            else:
                length = ((sv[1] - dv[1]) ** 2 + (sv[2] - dv[2]) ** 2) ** 0.5
                theta = np.arctan(((sv[0] - dv[0]) / 2) / (self.DSO + length / 2))
            return float(length / np.cos(theta))
        if self.reconstruction_mode == "voxel":
            return float(((sv[1] - dv[1]) ** 2 + (sv[2] - dv[2]) ** 2) ** 0.5)
        if nVoxel is None or dVoxel is None:
            return float(self.radius * 2)
        return float(max(sv[1], sv[2]))

    @classmethod
    def from_yaml(cls, path: str | Path, reconstruction_mode: str | None = None) -> "Geometry":
        with open(path, "r") as f:
            cfg = yaml.safe_load(f)
        if reconstruction_mode is None:
            reconstruction_mode = cfg.get("reconstruction_mode", "voxel")
        elif reconstruction_mode not in ("voxel", "cylindrical"):
            raise NotImplementedError(
                f"Only reconstruction mode 'voxel' and 'cylindrical' is implemented, got '{reconstruction_mode}'")
        return cls(nDetector=cfg["nDetector"], dDetector=cfg["dDetector"], mode=cfg["mode"], DSD=cfg.get("DSD"),
                   DSO=cfg.get("DSO"), nVoxel=cfg.get("nVoxel"), dVoxel=cfg.get("dVoxel"), radius=cfg.get("radius"),
                   height=cfg.get("height"), offOrigin=cfg.get("offOrigin", (0.0, 0.0, 0.0)),
                   COR=cfg.get("COR", 0.0), offDetector=cfg.get("offDetector", (0.0, 0.0)),
                   rotDetector=cfg.get("rotDetector", (0.0, 0.0, 0.0)), reconstruction_mode=reconstruction_mode,
                   detector_binning=1, angles=cfg.get("angles"), timesteps=cfg.get("timesteps"),
                   radians=cfg.get("radians", True))

    @classmethod
    def from_cfg(cls, cfg, reconstruction_mode: str = "voxel", sample_outside: int = 0) -> "Geometry":
        nVoxel = cfg.nVoxel
        if sample_outside > 0:
            nVoxel = [s + 2 * sample_outside for s in nVoxel]
        return cls(nDetector=cfg.nDetector, dDetector=cfg.dDetector, mode=cfg.mode,
                   DSD=getattr(cfg, "DSD", None), DSO=getattr(cfg, "DSO", None), nVoxel=nVoxel, dVoxel=cfg.dVoxel,
                   radius=cfg.radius, height=cfg.height, offOrigin=cfg.offOrigin, COR=cfg.COR,
                   offDetector=cfg.offDetector,
                   rotDetector=cfg.rotDetector if cfg.rotDetector is not None else (0.0, 0.0, 0.0),
                   reconstruction_mode=reconstruction_mode, detector_binning=1, angles=cfg.angles,
                   timesteps=cfg.timesteps)

    def set_angles(self, angles, radians: bool):
        self.angles = angles
        if self.angles is not None:
            if isinstance(self.angles, list):
                self.angles = np.array(self.angles)
            elif isinstance(self.angles, torch.Tensor):
                self.angles = self.angles.cpu().numpy()
            if radians is False:
                self.angles = np.radians(self.angles)

    def set_detector_binning(self, detector_binning: int):
        self.detector_binning = detector_binning

    def set_timesteps(self, timesteps):
        self.timesteps = timesteps

    def to_dict(self):
        return {
            "nDetector": self.nDetector, "dDetector": self.dDetector, "sDetector": self.sDetector,
            "mode": self.mode, "DSD": self.DSD, "DSO": self.DSO, "nVoxel": self.nVoxel, "dVoxel": self.dVoxel,
            "sVoxel": self.sVoxel, "radius": self.radius, "height": self.height, "angles": self.angles,
            "radians": True, "offOrigin": self.offOrigin, "COR": self.COR, "offDetector": self.offDetector,
            "rotDetector": self.rotDetector, "timesteps": self.timesteps,
        }

    def get_c_geometry(self):
        """The sampler geometry object for the current binning (geometry.py:322-407)."""
        b = self.detector_binning
        nDet = (self.nDetector[0] // b, self.nDetector[1] // b)
        dDet = (self.dDetector[0] * b, self.dDetector[1] * b)
        common = dict(nDetector=nDet, dDetector=dDet, offOrigin=self.offOrigin, offDetector=self.offDetector,
                      rotDetector=self.rotDetector, COR=self.COR)
        if self.mode == "cone":
            if self.DSD <= self.DSO:
                raise ValueError("DSD should be greater than DSO")
            if self.DSO <= 0:
                raise ValueError("DSO should be greater than 0")
            if self.DSD <= 0:
                raise ValueError("DSD should be greater than 0")
            cone = dict(distance_source_to_origin=self.DSO, distance_origin_to_detector=self.DSD - self.DSO)
            if self.reconstruction_mode == "cylindrical":
                return ct_sampling.ConeGeometryCylindrical(**cone, **common, object_radius=self.radius,
                                                           object_height=self.height, remove_factor_top=0,
                                                           remove_factor_bottom=0)
            return ct_sampling.ConeGeometryVoxel(**cone, **common, sVoxel=self.sVoxel, dVoxel=self.dVoxel)
        if self.reconstruction_mode == "cylindrical":
            return ct_sampling.ParallelGeometryCylindrical(**common, object_radius=self.radius,
                                                           object_height=self.height, remove_factor_top=0,
                                                           remove_factor_bottom=0)
        return ct_sampling.ParallelGeometryVoxel(**common, sVoxel=self.sVoxel, dVoxel=self.dVoxel)
