"""CPU tests of the sampling oracle: pinned against the reference kernel's own
outputs (tests/golden/sampling_golden.npz) and checked on hand-computed rays."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import sampling as osamp

GOLDEN = Path(__file__).resolve().parent / "golden" / "sampling_golden.npz"

KIND = {"ConeGeometryVoxel": 0, "ConeGeometryCylindrical": 1, "ParallelGeometryVoxel": 2,
        "ParallelGeometryCylindrical": 3}


def struct_from_dict(g):
    d = dict(kind=KIND[g["kind"]], nDetector=g["nDetector"], dDetector=g["dDetector"],
             offOrigin=g.get("offOrigin", (0.0, 0.0, 0.0)), offDetector=g.get("offDetector", (0.0, 0.0)),
             rotDetector=g.get("rotDetector", (0.0, 0.0, 0.0)), COR=g.get("COR", 0.0),
             distance_source_to_origin=g.get("distance_source_to_origin", 0.0),
             distance_origin_to_detector=g.get("distance_origin_to_detector", 0.0),
             sVoxel=g.get("sVoxel", (0.0, 0.0, 0.0)), dVoxel=g.get("dVoxel", (0.0, 0.0, 0.0)),
             object_radius=g.get("object_radius", 0.0), object_height=g.get("object_height", 0.0),
             remove_factor_top=g.get("remove_factor_top", 0.0), remove_factor_bottom=g.get("remove_factor_bottom", 0.0))
    return osamp.to_struct(d)


def golden_cases():
    if not GOLDEN.exists():
        return []
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    return [(m, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(m["name"] + "/")}) for m in meta]


CASES = golden_cases()


@pytest.mark.skipif(not CASES, reason="golden fixture not generated yet")
@pytest.mark.parametrize("case", CASES, ids=[c[0]["name"] for c in CASES])
def test_oracle_matches_reference_kernel_bit_for_bit(case):
    m, a = case
    g = struct_from_dict(m["geometry"])
    pts, dist, counts = osamp.oracle_sample(g, a["perm"], m["start"], m["R"], m["S"], m["angle"], m["maxd"],
                                            m["uniform"], a["jitter"], a["det_off"], trig=a["trig"])
    ref_pts, ref_dist = a["points"], a["distances"]
    # per-ray counts: the reference writes a prefix of each ray
    nz = np.any(ref_pts != 0, axis=2)
    ref_counts = np.where(nz.any(1), nz.shape[1] - np.argmax(nz[:, ::-1], axis=1), 0)
    np.testing.assert_array_equal(counts, ref_counts)
    np.testing.assert_array_equal(dist.view(np.uint32), ref_dist.view(np.uint32))
    np.testing.assert_array_equal(pts.view(np.uint32), ref_pts.view(np.uint32))


def parallel_unit_cube():
    return osamp.to_struct(dict(kind=2, nDetector=(128, 128), dDetector=(1 / 128, 1 / 128), offOrigin=(0, 0, 0),
                                offDetector=(0, 0), rotDetector=(0, 0, 0), COR=0.0, distance_source_to_origin=0.0,
                                distance_origin_to_detector=0.0, sVoxel=(1.0, 1.0, 1.0),
                                dVoxel=(1 / 128, 1 / 128, 1 / 128), object_radius=0.0, object_height=0.0,
                                remove_factor_top=0.0, remove_factor_bottom=0.0))


def test_axis_aligned_ray_known_answer():
    """Angle 0, pixel (row 64, col 64), no jitter: the ray runs along +x at
    y = -0.5/128 (the detector column maps to -y), z = +0.5/128, entering the
    box half-size (1 - 1/256)/2 = 0.498046875 (ct_sampling.cu:339-343)."""
    g = parallel_unit_cube()
    S = 256
    maxd = math.sqrt(2) * (1 - 1 / 128) / S
    perm = np.array([64 * 128 + 64], np.int64)
    pts, dist, counts = osamp.oracle_sample(g, perm, 0, 1, S, 0.0, maxd, True, np.zeros(1, np.float32),
                                            np.zeros((1, 2), np.float32))
    n = int(counts[0])
    step = np.float32(maxd)
    x0 = 0.5 - 0.498046875
    # positions advance by `step` along x; y, z stay put
    assert np.allclose(pts[0, :n, 2], x0 + np.arange(n) * float(step), atol=1e-6)
    assert np.all(pts[0, :n, 1] == np.float32(0.5 - 0.5 / 128))
    assert np.all(pts[0, :n, 0] == np.float32(0.5 + 0.5 / 128))
    # break when pos_x - 1e-5 exceeds end.x = min(1, 0.998046875 + step)
    end = min(1.0, 0.5 + 0.498046875 + float(step))
    expect = sum(1 for i in range(S) if (x0 + i * float(step)) - 1e-5 <= end)
    assert n == expect == 183
    assert np.all(pts[0, n:] == 0)
    assert dist[0] == np.float32(maxd)


def test_ray_missing_the_box_writes_nothing():
    """Cone beam pixel far outside the shadow of the box: count 0, distance 0."""
    g = osamp.to_struct(dict(kind=0, nDetector=(512, 512), dDetector=(1.0, 1.0), offOrigin=(0, 0, 0),
                             offDetector=(0, 0), rotDetector=(0, 0, 0), COR=0.0, distance_source_to_origin=500.0,
                             distance_origin_to_detector=500.0, sVoxel=(64.0, 64.0, 64.0), dVoxel=(1.0, 1.0, 1.0),
                             object_radius=0.0, object_height=0.0, remove_factor_top=0.0, remove_factor_bottom=0.0))
    perm = np.array([0, 511, 512 * 511], np.int64)  # detector corners
    pts, dist, counts = osamp.oracle_sample(g, perm, 0, 3, 64, 0.3, 0.5, True, np.zeros(3, np.float32),
                                            np.zeros((3, 2), np.float32))
    assert counts.tolist() == [0, 0, 0] and dist.tolist() == [0, 0, 0] and not pts.any()


def test_out_of_range_rays_are_skipped():
    g = parallel_unit_cube()
    perm = np.array([5, 128 * 128 + 3], np.int64)
    pts, dist, counts = osamp.oracle_sample(g, perm, 0, 3, 32, 0.1, 0.01, True, np.zeros(3, np.float32),
                                            np.zeros((3, 2), np.float32))
    assert counts[0] > 0 and counts[1] == 0 and counts[2] == 0  # 2nd: index too large; 3rd: past perm end
