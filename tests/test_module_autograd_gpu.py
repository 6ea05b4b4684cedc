"""HashGrid / HashGrid4D as differentiable modules, the way the reference's
trainer uses its model: ``points, y = projector(...)``, drop the all-zero
points, ``model(points)``, ``y_pred = sum * distances / max_distance_traveled``,
loss, ``loss.backward()``, ``optim.step()`` (nect/trainers/base_trainer.py:
520-568, 650-654), with the B200 modules in place of the tiny-cuda-nn ones.

Tolerances: sigma within 1e-5 of the fp64 oracle (both table precisions run
fp32 arithmetic in the module forward), gradients within 1e-3 of the
largest entry (fp32 atomics against fp64 autograd).
"""
import pytest
import torch

from oracle import hashgrid as ohg

pytestmark = pytest.mark.gpu


def make_model(n_dims, precision, seed=0):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=13, base_resolution=4,
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


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (3, "mixed"), (4, "plain_fp32"), (4, "mixed")])
def test_module_forward_is_differentiable(cuda_device, n_dims, precision):
    m, enc = make_model(n_dims, precision)
    gen = torch.Generator(device="cpu").manual_seed(4)
    x = torch.rand(4000, 3, generator=gen)
    target = torch.rand(4000, 1, generator=gen)
    t = torch.tensor(0.63, device=cuda_device)   # a device tensor, as the reference passes timesteps
    out = m(x.cuda()) if n_dims == 3 else m(x.cuda(), t)
    assert out.shape == (4000, 1) and out.grad_fn is not None
    loss = torch.nn.functional.mse_loss(out, target.cuda())
    loss.backward()
    torch.cuda.synchronize()

    levels, _ = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale),
                           float(enc.base_resolution_t or enc.base_resolution))
    tab = m.grid_table.detach().cpu().double().requires_grad_(True)
    wf = m.mlp.detach().cpu().double().requires_grad_(True)
    xin = x if n_dims == 3 else torch.cat([x, torch.full((4000, 1), 0.63, dtype=torch.float32)], 1)
    so = ohg.mlp(ohg.encode(xin, tab, levels, enc.log2_hashmap_size), ohg.split_mlp_params(wf, 32, 64, 2))
    torch.nn.functional.mse_loss(so, target.double()).backward()
    assert rel_max(out.detach().cpu().double(), so.detach()) < 1e-5
    assert rel_max(m.table.grad.cpu().double(), tab.grad) < 1e-3, rel_max(m.table.grad.cpu().double(), tab.grad)
    assert rel_max(m.mlp.grad.cpu().double(), wf.grad) < 1e-3, rel_max(m.mlp.grad.cpu().double(), wf.grad)


def test_timestep_tensor_stays_on_device(cuda_device):
    """A CUDA timestep is read by the kernels: forward and backward make no
    host synchronisation (torch's sync debug mode raises on one)."""
    m, _ = make_model(4, "mixed")
    x = torch.rand(2000, 3, device=cuda_device)
    t = torch.rand((), device=cuda_device)
    ref = m(x, float(t)).detach()          # host float (synchronises before the check below)
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode("error")
    try:
        out = m(x, t)
        out.sum().backward()
        with torch.no_grad():
            inf = m(x, t)
    finally:
        torch.cuda.set_sync_debug_mode("default")
    torch.cuda.synchronize()
    assert torch.equal(out.detach(), ref) and torch.equal(inf, ref)


def test_no_graph_under_no_grad(cuda_device):
    m, _ = make_model(3, "mixed")
    with torch.no_grad():
        out = m(torch.rand(100, 3, device=cuda_device))
    assert out.grad_fn is None and out.shape == (100, 1)


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_reference_style_training_loop(cuda_device, precision):
    """The reference's inner loop, written as it is there, with the module
    and the Projector of this package: the loss falls over 60 steps."""
    from nect_b200 import phantoms
    from nect_b200.sampling import Geometry, Projector

    n = 32
    geo = Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3, dVoxel=[1 / n] * 3)
    ph = phantoms.ellipsoid_phantom(20, 0)
    m, _ = make_model(3, precision)
    with torch.no_grad():
        m.table.mul_(1e-3)
        m.refresh_half()
    optim = torch.optim.Adam(m.parameters(), lr=3e-3)
    projector = Projector(geo, points_per_batch=512 * 48, points_per_ray=48, device=0)
    losses = []
    for k in range(60):
        angle = 3.14159 * (k % 16) / 16
        proj = phantoms.ellipsoid_projection(ph, geo, angle, "cuda").flatten()
        projector.update(angle)
        optim.zero_grad()
        points, y = projector(0, proj)
        mask = torch.all(points.view(-1, 3) == 0, dim=-1)
        shape = points.shape
        sig = m(points.view(-1, 3)[~mask])
        full = torch.zeros(shape[0] * shape[1], 1, device="cuda")
        full[~mask] = sig
        y_pred = full.view(shape[0], shape[1]).sum(1) * (projector.distances / geo.max_distance_traveled)
        loss = torch.nn.functional.mse_loss(y_pred, y)
        loss.backward()
        optim.step()
        if precision == "mixed":
            m.refresh_half()
        losses.append(float(loss))
    assert sum(losses[-10:]) < 0.2 * sum(losses[:10]), losses
