"""Generate tests/golden/sampling_golden.npz from the REFERENCE sampling kernel.

Run on a CUDA machine where ``oracle/_ref/ct_sampling.so`` (built from the
reference's nect/sampling/ct_sampling.cu by ``oracle/ref_build.py``) exists:

    python tests/golden/make_sampling_golden.py

For every case in sampling_cases.CASES it seeds torch, calls the reference
``sample`` (which draws its jitter and detector offsets from the CUDA default
generator, ct_sampling.cu:619-622), then re-seeds and re-draws the same random
numbers so the fixture holds every input of the call.  It also stores the
device's cosf/sinf of the angles (the oracle uses them in place of the host
libm values).  The CPU tests check the C oracle against this file bit for bit.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from oracle import ref_build  # noqa: E402
from sampling_cases import CASES, make_geometry, make_perm, max_distance  # noqa: E402


def device_trig(g: dict, angle: float, dev) -> np.ndarray:
    rot = g.get("rotDetector", (0.0, 0.0, 0.0))
    a = torch.tensor([angle, -rot[2], -rot[1], -rot[0]], dtype=torch.float32, device=dev)
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    return np.array([c[0], s[0], c[1], c[2], c[3], s[1], s[2], s[3]], np.float32)


KEEP_EVERY = 3  # rays kept per case: every third, to keep the fixture small


def compact(arrays: dict, meta: list, n_pixels: dict) -> tuple[dict, list]:
    """Keep every KEEP_EVERY-th ray of each case.  Rays are independent, so a
    subset stays a valid call: each kept ray is stored with its own pixel index
    (perm[start + tid], or n_pixels when the reference skips it because the
    index is past the permutation or past the detector) and starting index 0."""
    out, new_meta = {}, []
    for m in meta:
        name = m["name"]
        perm = arrays[f"{name}/perm"]
        R, start = m["R"], m["start"]
        tids = np.arange(0, R, KEEP_EVERY)
        pos = start + tids
        idx = np.where(pos < perm.size, perm[np.minimum(pos, perm.size - 1)], n_pixels[name])
        idx = np.where(idx >= n_pixels[name], n_pixels[name], idx).astype(np.int64)
        out[f"{name}/perm"] = idx
        for k in ("jitter", "det_off", "points", "distances"):
            out[f"{name}/{k}"] = arrays[f"{name}/{k}"][tids]
        out[f"{name}/trig"] = arrays[f"{name}/trig"]
        new_meta.append(dict(m, R=int(tids.size), start=0))
    return out, new_meta


def main(out: Path = HERE / "sampling_golden.npz") -> None:
    ref = ref_build.load()
    dev = torch.device("cuda", 0)
    arrays = {}
    meta = []
    for k, (name, g, angle, S, R, start, uniform, offset, mode) in enumerate(CASES):
        n_pix = g["nDetector"][0] * g["nDetector"][1]
        perm = make_perm(torch, n_pix, R, start, mode, dev, seed=100 + k)
        geom = make_geometry(ref, g)
        maxd = max_distance(g) / S
        torch.manual_seed(1234 + k)
        points, distances = ref.sample(random_ray_index=perm, geometry=geom, angle_rad=angle, num_points_per_ray=S,
                                       num_rays=R, starting_ray_index=start, max_ray_distance_per_point=maxd,
                                       uniform_ray_spacing=uniform, random_detector_offset=offset, device=0)
        torch.manual_seed(1234 + k)
        jitter = torch.rand(R, device=dev) - 0.5
        det_off = (torch.rand(R, 2, device=dev) - 0.5) * offset
        arrays[f"{name}/perm"] = perm.cpu().numpy()
        arrays[f"{name}/jitter"] = jitter.cpu().numpy()
        arrays[f"{name}/det_off"] = det_off.cpu().numpy()
        arrays[f"{name}/trig"] = device_trig(g, angle, dev)
        arrays[f"{name}/points"] = points.cpu().numpy()
        arrays[f"{name}/distances"] = distances.cpu().numpy()
        meta.append(dict(name=name, geometry=g, angle=angle, S=S, R=R, start=start, uniform=uniform, offset=offset,
                         maxd=maxd))
    n_pixels = {m["name"]: m["geometry"]["nDetector"][0] * m["geometry"]["nDetector"][1] for m in meta}
    arrays, meta = compact(arrays, meta, n_pixels)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(out, **arrays)
    print(f"wrote {out} ({out.stat().st_size} bytes, {len(meta)} cases)")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "sampling_golden.npz")
