"""The training step in two halves (nectb_train_forward / nectb_train_backward
through trainer.RayIntegral, loss computed by torch) against the fused step,
and the continuous-rotation step (y_pred averaged over sub-angles) against
the fp64 oracle.

Tolerances: split vs fused on the same batch, y_pred to 1e-6 and loss to
1e-5 relative; gradients to 1e-5 (plain) and 1e-3 (mixed) of the largest
entry: torch's loss gradient and the kernel's differ in the last fp32 bit,
which the mixed path rounds to bf16 before its tensor-core products, so a
sample's contribution can move by one bf16 step;
continuous-scan plain fp32 vs the oracle as the fused plain step (y_pred and
loss 1e-4, gradients 1e-3 of the largest entry); mixed vs the oracle on the
same fp16 table, gradient cosine > 0.99 and max deviation < 5e-2."""
import math

import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu


def make_model(n_dims, precision, seed=0):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=12, base_resolution=4,
                            finest_resolution=128, base_resolution_t=2 if n_dims == 4 else None)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=64, activation="ReLU", output_activation="Softplus")
    m = (HashGrid if n_dims == 3 else HashGrid4D)(enc, net, precision=precision, device="cuda", seed=seed)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(seed + 1)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.5)
        m.refresh_half()
    return m, enc


def setup(n_dims, precision):
    from nect_b200.sampling import Geometry

    torch.manual_seed(7)
    geo = Geometry(nDetector=[40, 48], dDetector=[1.5, 1.5], mode="cone", DSD=300.0, DSO=200.0,
                   nVoxel=[32, 32, 32], dVoxel=[1.0] * 3)
    m, enc = make_model(n_dims, precision)
    P = geo.nDetector[0] * geo.nDetector[1]
    perm = torch.randperm(P, device="cuda")
    proj = torch.rand(P, device="cuda")
    return geo, m, enc, perm, proj


def batch_for(perm, proj, angle, jitter, geo, S=64, R=500, start=60, t=0.35):
    from nect_b200.trainer import RayBatch

    return RayBatch(perm=perm, start=start, num_rays=R, points_per_ray=S, angle=angle,
                    max_ray_distance_per_point=geo.max_distance_traveled / S, jitter=jitter,
                    detector_offset=torch.zeros(R, 2, device="cuda"), projection=proj, t=t)


def rel_max(a, b):
    a, b = a.detach(), b.detach()
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (3, "mixed"), (4, "mixed")])
def test_split_step_matches_fused_step(cuda_device, n_dims, precision):
    from nect_b200.trainer import Workspace, projection_loss, ray_integral, train_step

    geo, m, enc, perm, proj = setup(n_dims, precision)
    cg = geo.get_c_geometry()
    batch = batch_for(perm, proj, 0.9, torch.rand(500, device="cuda") - 0.5, geo)
    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    L, y = train_step(m, cg, batch, geo.max_distance_traveled, tg, mg, Workspace(), "l2")
    y2 = ray_integral(m, cg, batch, geo.max_distance_traveled, Workspace())
    L2 = projection_loss(y2, proj[perm[batch.start:batch.start + batch.num_rays]], "l2")
    gt, gm = torch.autograd.grad(L2, [m.table, m.mlp])
    torch.cuda.synchronize()
    assert rel_max(y2, y) < 1e-6
    assert abs(float(L2.detach()) - float(L)) <= 1e-5 * abs(float(L))
    tol = 1e-5 if precision == "plain_fp32" else 1e-3
    assert rel_max(gt, tg) < tol, rel_max(gt, tg)
    assert rel_max(gm, mg) < tol, rel_max(gm, mg)


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (4, "mixed")])
def test_continuous_scan_step_matches_oracle(cuda_device, n_dims, precision):
    from nect_b200.trainer import Workspace, projection_loss, ray_integral

    geo, m, enc, perm, proj = setup(n_dims, precision)
    cg = geo.get_c_geometry()
    k, a0, a1, t = 3, 0.4, 0.7, 0.35
    edges = np.linspace(a0, a1, k + 1)
    angles = [float((edges[j] + edges[j + 1]) / 2) for j in range(k)]
    jitters = [torch.rand(500, device="cuda") - 0.5 for _ in range(k)]
    batches = [batch_for(perm, proj, a, jt, geo, t=t) for a, jt in zip(angles, jitters)]
    y = sum(ray_integral(m, cg, b, geo.max_distance_traveled, Workspace()) for b in batches) / k
    meas = proj[perm[60:560]]
    L = projection_loss(y, meas, "l2")
    gt, gm = torch.autograd.grad(L, [m.table, m.mlp])
    torch.cuda.synchronize()

    samples = []
    for a, jt, b in zip(angles, jitters, batches):
        ang = torch.tensor([a, 0.0], dtype=torch.float32, device="cuda")
        c, s = torch.cos(ang).cpu().numpy(), torch.sin(ang).cpu().numpy()
        trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
        pts, dist, _ = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), b.start, b.num_rays,
                                           b.points_per_ray, a, b.max_ray_distance_per_point, True,
                                           jt.cpu().numpy(), np.zeros((b.num_rays, 2), np.float32), trig=trig)
        samples.append((pts, dist))
    levels, _ = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale),
                           float(enc.base_resolution_t or enc.base_resolution))
    yo, Lo, gto, gmo = ohg.averaged_step(samples, meas.cpu().numpy().astype(np.float64), m.grid_table.detach().cpu(),
                                         m.mlp.detach().cpu(), levels, enc.log2_hashmap_size, 32, 64, 2,
                                         geo.max_distance_traveled, t=t if n_dims == 4 else None)
    y, gt, gm = y.detach().cpu().double(), gt.cpu().double(), gm.cpu().double()
    if precision == "plain_fp32":
        assert rel_max(y, yo) < 1e-4
        assert abs(float(L.detach()) - float(Lo)) <= 1e-4 * abs(float(Lo))
        assert rel_max(gt, gto) < 1e-3, rel_max(gt, gto)
        assert rel_max(gm, gmo) < 1e-3, rel_max(gm, gmo)
    else:
        cos = lambda a, b: float((a.flatten() @ b.flatten()) / (a.norm() * b.norm()))  # noqa: E731
        assert rel_max(y, yo) < 2e-2
        assert cos(gt, gto) > 0.99 and cos(gm, gmo) > 0.99
        assert rel_max(gt, gto) < 5e-2 and rel_max(gm, gmo) < 5e-2


def test_trainer_continuous_step_runs(cuda_device):
    from nect_b200.trainer import Trainer

    geo, m, enc, perm, proj = setup(4, "mixed")
    tr = Trainer(m, geo, points_per_batch=500 * 64, points_per_ray=64, loss="l2", device="cuda")
    losses = [float(tr.continuous_step(perm, 0, 0.2, 0.5, proj, t=0.5, accumulation_steps=4, add_poisson=True))
              for _ in range(3)]
    assert all(math.isfinite(v) for v in losses)
    assert tr.step_count == 3
