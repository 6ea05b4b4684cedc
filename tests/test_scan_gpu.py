"""The fused continuous-scan step (every sub-angle's rays in one launch of
each kernel, nectb_train_scan_*) against the per-sub-angle version (one
forward and backward per sub-angle through the split step) and against the
fp64 oracle's sub-angle average (nect/trainers/continous_scanning_trainer.py:
85-140, oracle.hashgrid.averaged_step).

Tolerances: fused vs per-sub-angle on the same draws, y_pred to 1e-6 of the
largest (the average is summed in another order), gradients to 1e-5 (plain)
and 1e-3 (mixed) of the largest entry (the split step's tolerances); against
the oracle the fused step's: plain y_pred and loss 1e-4, gradients 1e-3 of
the largest entry; mixed y_pred 2e-2, gradient cosine > 0.99 and max
deviation < 5e-2.
"""
import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg
from oracle import sampling as osamp
from test_split_step_gpu import rel_max, setup

pytestmark = pytest.mark.gpu


def scan_batch(perm, proj, geo, k, R=500, start=60, S=64, t=0.35, offset=0.0):
    from nect_b200.sampling.ct_sampling import draw_ray_randoms
    from nect_b200.trainer import RayBatch

    draws = [draw_ray_randoms(R, offset, torch.device("cuda")) for _ in range(k)]
    batch = RayBatch(perm=perm, start=start, num_rays=R, points_per_ray=S, angle=0.0,
                     max_ray_distance_per_point=geo.max_distance_traveled / S,
                     jitter=torch.cat([d[0] for d in draws]), detector_offset=torch.cat([d[1] for d in draws]),
                     projection=proj, t=t)
    return batch, draws


def sub_batch(batch, draws, j, angle):
    from nect_b200.trainer import RayBatch

    return RayBatch(perm=batch.perm, start=batch.start, num_rays=batch.num_rays, points_per_ray=batch.points_per_ray,
                    angle=angle, max_ray_distance_per_point=batch.max_ray_distance_per_point, jitter=draws[j][0],
                    detector_offset=draws[j][1], projection=batch.projection, t=batch.t)


def cosine(a, b):
    a, b = a.flatten(), b.flatten()
    return float((a @ b) / (a.norm() * b.norm()).clamp(min=1e-30))


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (3, "mixed"), (4, "mixed")])
def test_fused_scan_matches_per_sub_angle_launches(cuda_device, n_dims, precision):
    from nect_b200.trainer import Workspace, projection_loss, ray_integral, scan_integral

    geo, m, enc, perm, proj = setup(n_dims, precision)
    cg = geo.get_c_geometry()
    k = 4
    edges = np.linspace(0.4, 0.75, k + 1)
    angles = [float((edges[j] + edges[j + 1]) / 2) for j in range(k)]
    batch, draws = scan_batch(perm, proj, geo, k, offset=0.3)
    meas = proj[perm[60:560]]
    y1 = scan_integral(m, cg, batch, angles, geo.max_distance_traveled, Workspace())
    g1 = torch.autograd.grad(projection_loss(y1, meas, "l2"), [m.table, m.mlp])
    y2 = None
    for j in range(k):
        yj = ray_integral(m, cg, sub_batch(batch, draws, j, angles[j]), geo.max_distance_traveled, Workspace()) / k
        y2 = yj if y2 is None else y2 + yj
    g2 = torch.autograd.grad(projection_loss(y2, meas, "l2"), [m.table, m.mlp])
    torch.cuda.synchronize()
    assert rel_max(y1, y2) < 1e-6, rel_max(y1, y2)
    tol = 1e-5 if precision == "plain_fp32" else 1e-3
    assert rel_max(g1[0], g2[0]) < tol and rel_max(g1[1], g2[1]) < tol, (rel_max(g1[0], g2[0]), rel_max(g1[1], g2[1]))


@pytest.mark.parametrize("n_dims,precision,loss", [(3, "plain_fp32", "l2"), (4, "plain_fp32", "l1"),
                                                   (3, "mixed", "l2"), (4, "mixed", "l2")])
def test_fused_scan_step_matches_oracle(cuda_device, n_dims, precision, loss):
    from nect_b200.trainer import Workspace, scan_step

    geo, m, enc, perm, proj = setup(n_dims, precision)
    cg = geo.get_c_geometry()
    k, t = 3, 0.35
    edges = np.linspace(1.1, 1.4, k + 1)
    angles = [float((edges[j] + edges[j + 1]) / 2) for j in range(k)]
    batch, draws = scan_batch(perm, proj, geo, k, t=t)
    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    ws = Workspace()
    L, y = scan_step(m, cg, batch, angles, geo.max_distance_traveled, tg, mg, ws, loss)
    torch.cuda.synchronize()
    assert ws.error_word(cg) == 0
    samples = []
    for j, a in enumerate(angles):
        ang = torch.tensor([a, 0.0], dtype=torch.float32, device="cuda")
        c, s = torch.cos(ang).cpu().numpy(), torch.sin(ang).cpu().numpy()
        trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
        pts, dist, _ = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), batch.start, batch.num_rays,
                                           batch.points_per_ray, a, batch.max_ray_distance_per_point, True,
                                           draws[j][0].cpu().numpy(), draws[j][1].cpu().numpy(), trig=trig)
        samples.append((pts, dist))
    levels, _ = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale),
                           float(enc.base_resolution_t or enc.base_resolution))
    meas = proj[perm[60:560]].cpu().numpy().astype(np.float64)
    yo, Lo, gto, gmo = ohg.averaged_step(samples, meas, m.grid_table.detach().cpu(), m.mlp.detach().cpu(), levels,
                                         enc.log2_hashmap_size, 32, 64, 2, geo.max_distance_traveled, loss=loss,
                                         t=t if n_dims == 4 else None)
    y, gt, gm = y.cpu().double(), tg.cpu().double(), mg.cpu().double()
    if precision == "plain_fp32":
        assert rel_max(y, yo) < 1e-4
        assert abs(float(L) - float(Lo)) <= 1e-4 * abs(float(Lo))
        assert rel_max(gt, gto) < 1e-3, rel_max(gt, gto)
        assert rel_max(gm, gmo) < 1e-3, rel_max(gm, gmo)
    else:
        assert rel_max(y, yo) < 2e-2
        assert abs(float(L) - float(Lo)) <= 5e-2 * abs(float(Lo))
        assert cosine(gt, gto) > 0.99 and cosine(gm, gmo) > 0.99, (cosine(gt, gto), cosine(gm, gmo))
        assert rel_max(gt, gto) < 5e-2 and rel_max(gm, gmo) < 5e-2


def test_trainer_fused_and_per_sub_angle_steps_agree(cuda_device):
    """Trainer.continuous_step draws the same random numbers in the same order
    whether fused or not, so both give the same loss."""
    from nect_b200.trainer import Trainer

    losses = []
    for fused in (True, False):
        geo, m, enc, perm, proj = setup(4, "mixed")
        tr = Trainer(m, geo, points_per_batch=500 * 64, points_per_ray=64, loss="l2", device="cuda",
                     random_offset_detector=0.25)
        torch.manual_seed(123)
        losses.append(float(tr.continuous_step(perm, 0, 0.2, 0.5, proj, t=0.5, accumulation_steps=4, fused=fused)))
    assert abs(losses[0] - losses[1]) <= 1e-5 * abs(losses[1]), losses
