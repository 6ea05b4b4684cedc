"""GPU parity of the sampling kernel (through the C ABI) against the
reference's own kernel (compiled from nect/sampling/ct_sampling.cu into
oracle/_ref) and against the C oracle: bit-exact points, distances and
per-ray counts."""

import numpy as np
import pytest
import torch

from sampling_cases import CASES, CONE_C2, PAR_C1, make_geometry, make_perm, max_distance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_module(cuda_device):
    from oracle import ref_build

    try:
        return ref_build.load()
    except FileNotFoundError as e:
        pytest.skip(str(e))


@pytest.fixture(scope="module")
def mine():
    from nect_b200.sampling import ct_sampling

    return ct_sampling


def bits_equal(a: torch.Tensor, b: torch.Tensor) -> bool:
    return a.shape == b.shape and torch.equal(a.contiguous().view(torch.int32), b.contiguous().view(torch.int32))


def run_pair(ref, mine, g, angle, S, R, start, uniform, offset, perm, seed):
    maxd = max_distance(g) / S
    torch.manual_seed(seed)
    rp, rd = ref.sample(random_ray_index=perm, geometry=make_geometry(ref, g), angle_rad=angle, num_points_per_ray=S,
                        num_rays=R, starting_ray_index=start, max_ray_distance_per_point=maxd,
                        uniform_ray_spacing=uniform, random_detector_offset=offset, device=0)
    torch.manual_seed(seed)
    mp, md = mine.sample(random_ray_index=perm, geometry=make_geometry(mine, g), angle_rad=angle,
                         num_points_per_ray=S, num_rays=R, starting_ray_index=start, max_ray_distance_per_point=maxd,
                         uniform_ray_spacing=uniform, random_detector_offset=offset, device=0)
    torch.cuda.synchronize()
    return rp, rd, mp, md


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_kernel_matches_reference_kernel(ref_module, mine, cuda_device, case):
    name, g, angle, S, R, start, uniform, offset, mode = case
    k = [c[0] for c in CASES].index(name)
    perm = make_perm(torch, g["nDetector"][0] * g["nDetector"][1], R, start, mode, cuda_device, seed=100 + k)
    rp, rd, mp, md = run_pair(ref_module, mine, g, angle, S, R, start, uniform, offset, perm, 1234 + k)
    assert bits_equal(rd, md)
    assert bits_equal(rp, mp)


@pytest.mark.parametrize("geom,angles,S", [(CONE_C2, [0.0, 0.8, 2.6, 4.4], 512), (PAR_C1, [0.0, 1.0, 2.5], 256)],
                         ids=["cone_c2_full_projection", "parallel_c1_full_projection"])
def test_full_projection_bit_exact(ref_module, mine, cuda_device, geom, angles, S):
    """Every pixel of a full-size benchmark projection in one batch (R = P)."""
    n = geom["nDetector"][0] * geom["nDetector"][1]
    perm = torch.randperm(n, device=cuda_device)
    for j, ang in enumerate(angles):
        rp, rd, mp, md = run_pair(ref_module, mine, geom, ang, S, n, 0, True, 0.0, perm, 77 + j)
        assert bits_equal(rd, md), f"distances differ at angle {ang}"
        assert bits_equal(rp, mp), f"points differ at angle {ang}"
        del rp, mp
        torch.cuda.empty_cache()


def test_counts_match_c_oracle(mine, cuda_device):
    """Per-ray counts and positions of the kernel vs the C oracle (device trig)."""
    from oracle import sampling as osamp

    g = CONE_C2
    S, R = 512, 8192
    n = g["nDetector"][0] * g["nDetector"][1]
    perm = torch.randperm(n, device=cuda_device)
    angle = 2.1
    geom = make_geometry(mine, g)
    maxd = max_distance(g) / S
    torch.manual_seed(5)
    jitter, det_off = mine.draw_ray_randoms(R, 0.5, cuda_device)
    pts, dist, counts = mine.sample_with_draws(perm, geom, angle, S, R, 0, maxd, True, jitter, det_off,
                                               want_counts=True)
    a = torch.tensor([angle, 0.0], dtype=torch.float32, device=cuda_device)
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
    opts, odist, ocounts = osamp.oracle_sample(osamp.to_struct(geom), perm.cpu().numpy(), 0, R, S, angle, maxd, True,
                                               jitter.cpu().numpy(), det_off.cpu().numpy(), trig=trig)
    np.testing.assert_array_equal(counts.cpu().numpy(), ocounts)
    np.testing.assert_array_equal(dist.cpu().numpy().view(np.uint32), odist.view(np.uint32))
    np.testing.assert_array_equal(pts.cpu().numpy().view(np.uint32), opts.view(np.uint32))


def test_projector_clamps_and_gathers(cuda_device):
    from nect_b200.sampling import Geometry, Projector

    geo = Geometry(nDetector=[128, 128], dDetector=[1 / 128, 1 / 128], mode="parallel", nVoxel=[128, 128, 128],
                   dVoxel=[1 / 128] * 3)
    pr = Projector(geo, points_per_batch=4096 * 256, points_per_ray=256, device=0)
    pr.update(angle=0.3)
    proj = torch.rand(128 * 128, device=cuda_device)
    pts, y = pr(0, proj)
    assert pts.shape == (4096, 256, 3) and y.shape == (4096,)
    assert float(pts.min()) >= 0.0 and float(pts.max()) <= 1.0
    assert torch.equal(y, proj[pr.random_indexes[:4096]])
    assert pr.batch_per_epoch == 4
    assert pr(4, proj) == (None, None)
