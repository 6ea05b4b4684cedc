"""Sampling cases shared by the golden-fixture generator and the parity tests.

Each case names one of the reference's four geometry structs with its
constructor keywords (nect/sampling/ct_sampling.cu:650-749) and one call of
``sample`` (:756-807).  They cover the benchmark geometries (parallel unit
cube with a 128x128 detector; cone beam DSO 500 / DSD 1000 on a 512x512
detector over a 256^3 volume), detector offsets and tilt, centre-of-rotation
shifts, cylindrical clipping with top/bottom removal, non-uniform spacing,
batches that run past the end of the permutation, and out-of-range pixel
indices.
"""
from __future__ import annotations

import math

PAR_C1 = dict(kind="ParallelGeometryVoxel", nDetector=(128, 128), dDetector=(1 / 128, 1 / 128),
              sVoxel=(1.0, 1.0, 1.0), dVoxel=(1 / 128, 1 / 128, 1 / 128))
CONE_C2 = dict(kind="ConeGeometryVoxel", distance_source_to_origin=500.0, distance_origin_to_detector=500.0,
               nDetector=(512, 512), dDetector=(1.0, 1.0), sVoxel=(256.0, 256.0, 256.0), dVoxel=(1.0, 1.0, 1.0))
CONE_TILT = dict(kind="ConeGeometryVoxel", distance_source_to_origin=410.0, distance_origin_to_detector=290.0,
                 nDetector=(96, 160), dDetector=(1.3, 0.9), offDetector=(3.25, -7.5), rotDetector=(0.02, -0.015, 0.01),
                 COR=1.75, sVoxel=(120.0, 150.0, 150.0), dVoxel=(1.0, 1.0, 1.0))
CONE_CYL = dict(kind="ConeGeometryCylindrical", distance_source_to_origin=500.0, distance_origin_to_detector=500.0,
                nDetector=(256, 256), dDetector=(2.0, 2.0), COR=0.5, object_radius=110.0, object_height=230.0,
                remove_factor_top=0.05, remove_factor_bottom=0.02)
PAR_CYL = dict(kind="ParallelGeometryCylindrical", nDetector=(64, 96), dDetector=(1.0, 1.0), object_radius=40.0,
               object_height=60.0, offDetector=(0.5, 0.0))
PAR_ANISO = dict(kind="ParallelGeometryVoxel", nDetector=(80, 120), dDetector=(0.5, 0.75), COR=-2.0,
                 sVoxel=(30.0, 64.0, 48.0), dVoxel=(0.5, 1.0, 0.75), offDetector=(-1.0, 2.0))


def max_distance(g: dict) -> float:
    """Geometry.max_distance_traveled for these dicts (nect/sampling/geometry.py:156-174)."""
    if g["kind"] == "ConeGeometryVoxel":
        sv, dv = g["sVoxel"], g["dVoxel"]
        length = ((sv[1] - dv[1]) ** 2 + (sv[2] - dv[2]) ** 2) ** 0.5
        theta = math.atan(((sv[0] - dv[0]) / 2) / (g["distance_source_to_origin"] + length / 2))
        return length / math.cos(theta)
    if g["kind"] == "ParallelGeometryVoxel":
        sv, dv = g["sVoxel"], g["dVoxel"]
        return ((sv[1] - dv[1]) ** 2 + (sv[2] - dv[2]) ** 2) ** 0.5
    if g["kind"] == "ConeGeometryCylindrical":
        length = 2 * g["object_radius"]
        theta = math.atan((g["object_height"] / 2) / (g["distance_source_to_origin"] + length / 2))
        return length / math.cos(theta)
    return 2 * g["object_radius"]


# (name, geometry, angle, S, num_rays, start, uniform, random_detector_offset, perm_mode)
# perm_mode: "perm" = randperm of all pixels; "tail" = batch runs past the end;
# "bad" = some indices beyond nDetector[0]*nDetector[1].
CASES = [
    ("par_c1_a0", PAR_C1, 0.0, 256, 192, 0, True, 0.0, "perm"),
    ("par_c1_a07", PAR_C1, 0.7, 256, 192, 64, True, 0.0, "perm"),
    ("par_c1_ahalfpi", PAR_C1, math.pi / 2, 256, 192, 0, True, 0.5, "perm"),
    ("par_c1_a29_nonuni", PAR_C1, 2.9, 200, 160, 0, False, 0.0, "perm"),
    ("cone_c2_a0", CONE_C2, 0.0, 512, 128, 0, True, 0.0, "perm"),
    ("cone_c2_a1", CONE_C2, 1.234, 512, 128, 1000, True, 0.5, "perm"),
    ("cone_c2_a5", CONE_C2, 5.5, 512, 128, 0, True, 0.0, "tail"),
    ("cone_tilt", CONE_TILT, 0.4, 300, 160, 0, True, 0.25, "perm"),
    ("cone_tilt_nonuni", CONE_TILT, 2.2, 300, 160, 0, False, 0.0, "bad"),
    ("cone_cyl", CONE_CYL, 0.9, 384, 160, 0, True, 0.5, "perm"),
    ("par_cyl", PAR_CYL, 1.1, 128, 160, 0, True, 0.0, "perm"),
    ("par_aniso", PAR_ANISO, 3.7, 160, 160, 0, True, 0.3, "perm"),
]


def make_geometry(module, g: dict):
    """Instantiate a geometry dict with a ct_sampling-like module (the
    reference extension or nect_b200.sampling.ct_sampling)."""
    kw = {k: v for k, v in g.items() if k != "kind"}
    return getattr(module, g["kind"])(**kw)


def make_perm(torch, n_pixels: int, num_rays: int, start: int, mode: str, device, seed: int):
    gen = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(n_pixels, generator=gen, dtype=torch.int64)
    if mode == "tail":
        perm = perm[: start + num_rays // 2]
    elif mode == "bad":
        idx = torch.arange(0, perm.numel(), 7)
        perm[idx] = n_pixels + idx
    return perm.to(device)
