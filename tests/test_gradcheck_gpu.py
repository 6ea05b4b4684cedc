"""Gradients of the fused training kernels (called through the C ABI) against
FP64 central finite differences of the same network's loss on 1,000 seeded
parameters: 900 table values among the entries the batch touches and 100 MLP
weights (numpy default_rng(2024)).

Tolerances: plain fp32 path, every sampled gradient within 1e-3 of the
largest sampled gradient (table and MLP separately); mixed path (fp16 table,
bf16 tensor-core MLP) against the finite differences of the fp64 network on
the same fp16 table values, cosine similarity > 0.99 and every entry within
5e-2 of the largest.  The reference's own gradient (tiny-cuda-nn) cannot be
computed here: tiny-cuda-nn is not part of the reference tree."""

import numpy as np
import pytest
import torch

from oracle import gradcheck as ogc
from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu


def make_model(n_dims, precision, seed=0):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=12, base_resolution=4,
                            finest_resolution=128, base_resolution_t=2 if n_dims == 4 else None)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=64, activation="ReLU", output_activation="Softplus")
    cls = HashGrid if n_dims == 3 else HashGrid4D
    m = cls(enc, net, precision=precision, device="cuda", seed=seed)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(seed + 1)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.5)
        m.refresh_half()
    return m, enc


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (4, "mixed")])
def test_kernel_gradients_match_finite_differences(cuda_device, n_dims, precision):
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import RayBatch, Workspace, train_step

    torch.manual_seed(21)
    geo = Geometry(nDetector=[40, 48], dDetector=[1.5, 1.5], mode="cone", DSD=300.0, DSO=200.0,
                   nVoxel=[32, 32, 32], dVoxel=[1.0] * 3)
    m, enc = make_model(n_dims, precision)
    cg = geo.get_c_geometry()
    P = geo.nDetector[0] * geo.nDetector[1]
    S, R, start = 64, 300, 40
    perm = torch.randperm(P, device="cuda")
    jitter = torch.rand(R, device="cuda") - 0.5
    det_off = torch.zeros(R, 2, device="cuda")
    proj = torch.rand(P, device="cuda")
    angle, t = 1.1, 0.6
    maxd = geo.max_distance_traveled / S
    batch = RayBatch(perm=perm, start=start, num_rays=R, points_per_ray=S, angle=angle,
                     max_ray_distance_per_point=maxd, jitter=jitter, detector_offset=det_off, projection=proj, t=t)
    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    train_step(m, cg, batch, geo.max_distance_traveled, tg, mg, Workspace(), "l2")
    torch.cuda.synchronize()
    tg, mg = tg.cpu().double(), mg.cpu().double()

    a = torch.tensor([angle, 0.0], dtype=torch.float32, device="cuda")
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
    pts, dist, _ = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), start, R, S, angle, maxd, True,
                                       jitter.cpu().numpy(), det_off.cpu().numpy(), trig=trig)
    levels, _ = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale),
                           float(enc.base_resolution_t or enc.base_resolution))
    measured = proj.cpu().numpy()[perm.cpu().numpy()[start:start + R]].astype(np.float64)
    bl = ogc.BatchLoss(pts, dist, measured, m.grid_table.detach().cpu(), m.mlp.detach().cpu(), levels,
                       enc.log2_hashmap_size, 32, 64, 2, geo.max_distance_traveled, loss="l2",
                       t=t if n_dims == 4 else None)
    tab, mlp_idx = ogc.seeded_parameters(bl, 900, 100, seed=2024)
    assert len(tab) + len(mlp_idx) == 1000
    h = 1e-6
    fd_t = np.array([bl.table_fd(e, f, h) for e, f in tab])
    fd_m = np.array([bl.mlp_fd(i, h) for i in mlp_idx])
    g_t = np.array([float(tg[e, f]) for e, f in tab])
    g_m = np.array([float(mg[i]) for i in mlp_idx])
    st, sm = np.abs(fd_t).max(), np.abs(fd_m).max()
    err_t, err_m = np.abs(g_t - fd_t).max() / st, np.abs(g_m - fd_m).max() / sm
    if precision == "plain_fp32":
        assert err_t < 1e-3, err_t
        assert err_m < 1e-3, err_m
    else:
        cos_t = float(g_t @ fd_t / (np.linalg.norm(g_t) * np.linalg.norm(fd_t)))
        cos_m = float(g_m @ fd_m / (np.linalg.norm(g_m) * np.linalg.norm(fd_m)))
        assert cos_t > 0.99 and cos_m > 0.99, (cos_t, cos_m)
        assert err_t < 5e-2 and err_m < 5e-2, (err_t, err_m)
