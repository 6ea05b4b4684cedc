"""nectb_model_backward (through trainer.ModelPoints) against the fp64 oracle's
autograd: L = sum_i dsigma_i * sigma(x_i) at random points, including cell
vertices and the 0/1 faces.  Both table precisions run fp32 SIMT arithmetic:
sigma within 1e-5 and gradients within 1e-3 of the largest entry (the
mixed-precision model against the oracle on its fp16 table values).  Then the
total-variation term end to end."""
import math

import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg

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


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (3, "mixed"), (4, "mixed")])
def test_model_backward_matches_oracle(cuda_device, n_dims, precision):
    from nect_b200.trainer import model_points

    m, enc = make_model(n_dims, precision)
    g = torch.Generator(device="cpu").manual_seed(9)
    x = torch.rand(3000, 3, generator=g)
    x[:40] = torch.round(x[:40] * 8) / 8
    x[40:50] = 1.0
    x[50:60] = 0.0
    ds = torch.randn(3000, generator=g)
    t = 0.42
    sig = model_points(m, x.cuda(), t)
    gt, gm = torch.autograd.grad((sig * ds.cuda()).sum(), [m.table, m.mlp])
    torch.cuda.synchronize()

    levels, _ = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale),
                           float(enc.base_resolution_t or enc.base_resolution))
    tab = m.grid_table.detach().cpu().double().requires_grad_(True)
    wf = m.mlp.detach().cpu().double().requires_grad_(True)
    xin = x if n_dims == 3 else torch.cat([x, torch.full((3000, 1), t)], 1)
    so = ohg.mlp(ohg.encode(xin, tab, levels, enc.log2_hashmap_size), ohg.split_mlp_params(wf, 32, 64, 2)).squeeze(-1)
    (so * ds.double()).sum().backward()
    assert rel_max(sig.detach().cpu().double(), so.detach()) < 1e-5
    assert rel_max(gt.cpu().double(), tab.grad) < 1e-3, rel_max(gt.cpu().double(), tab.grad)
    assert rel_max(gm.cpu().double(), wf.grad) < 1e-3, rel_max(gm.cpu().double(), wf.grad)


def test_fit_with_total_variation(cuda_device):
    from nect_b200 import phantoms
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig
    from nect_b200.reconstruct import fit, psnr
    from nect_b200.sampling import Geometry

    n = 48
    geo = Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3, dVoxel=[1 / n] * 3)
    ph = phantoms.ellipsoid_phantom(20, 0)
    angles = np.linspace(0, math.pi, 40, endpoint=False)
    projs = torch.stack([phantoms.ellipsoid_projection(ph, geo, float(a), "cuda") for a in angles])
    truth = phantoms.ellipsoid_volume(ph, n, "cuda")
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=16, base_resolution=8,
                            finest_resolution=4 * n)
    cfg = ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "mixed")
    rec = fit(geo, projs, angles, model_cfg=cfg, niter=300, lr=2e-3, points_per_ray=96, tv=1e-3,
              evaluate=lambda r: {"psnr": psnr(r.volume(), truth)}, eval_every=300)
    assert rec.trainer.step_count == 300
    assert rec.history[-1][2]["psnr"] > rec.history[0][2]["psnr"] + 8
