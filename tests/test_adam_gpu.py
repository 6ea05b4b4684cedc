"""nectb_adam_step (through the C ABI) against torch.optim.Adam on the GPU.

The fused update stands in for the optimizer the reference builds from its
configuration (nect/config.py:400-414: torch.optim.Adam with betas and weight
decay; the lr schedule is applied outside the step).  Several steps with fresh
gradients exercise the bias corrections; the fp16 shadow the mixed path
gathers from must equal the updated fp32 parameters rounded to fp16, and the
gradient must read zero afterwards when zero_grad is set.

Tolerances: parameters within 1e-6 relative + 1e-8 absolute, moments within
1e-6 of their largest entry (the kernel follows torch's order of operations;
what remains is fp32 contraction inside either kernel); the fp16 shadow bit
for bit.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _adam(p, g, m, v, step, lr, betas, eps, wd, half=None, zero_grad=1):
    from nect_b200 import _lib

    rc = _lib.lib.nectb_adam_step(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), lr, betas[0],
                                  betas[1], eps, wd, step, half.data_ptr() if half is not None else None, zero_grad,
                                  _lib.stream_ptr())
    _lib.check(rc, "nectb_adam_step")


@pytest.mark.parametrize("betas,wd,lr", [((0.9, 0.999), 0.0, 1e-3), ((0.8, 0.95), 1e-2, 5e-3),
                                         ((0.9, 0.99), 1e-6, 2e-4)])
def test_adam_matches_torch_optim_adam(cuda_device, betas, wd, lr):
    gen = torch.Generator(device="cpu").manual_seed(3)
    n = 1_000_003   # not a multiple of the block size: the grid-stride tail
    start = (torch.rand(n, generator=gen) * 2 - 1).to(cuda_device)
    ref = start.clone().requires_grad_(True)
    opt = torch.optim.Adam([ref], lr=lr, betas=betas, eps=1e-15 if wd == 1e-6 else 1e-8, weight_decay=wd)
    eps = opt.param_groups[0]["eps"]
    p = start.clone()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    half = torch.empty(n, dtype=torch.float16, device=cuda_device)
    for step in range(1, 7):
        g = torch.randn(n, generator=gen).to(cuda_device) * (10.0 ** (step % 3 - 1))
        g[::97] = 0.0   # untouched entries still decay their moments
        ref.grad = g.clone()
        opt.step()
        gk = g.clone()
        _adam(p, gk, m, v, step, lr, betas, eps, wd, half=half)
        torch.cuda.synchronize()
        assert not gk.any(), "zero_grad left gradient entries"
        st = opt.state[ref]
        torch.testing.assert_close(p, ref.detach(), rtol=1e-6, atol=1e-8)
        for mine, theirs in ((m, st["exp_avg"]), (v, st["exp_avg_sq"])):
            assert float((mine - theirs).abs().max()) <= 1e-6 * float(theirs.abs().max())
        assert torch.equal(half.view(torch.int16), p.half().view(torch.int16)), "fp16 shadow != table.half()"


def test_adam_keeps_gradient_without_zero_grad(cuda_device):
    p = torch.ones(1000, device=cuda_device)
    g = torch.full_like(p, 0.5)
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    _adam(p, g, m, v, 1, 1e-3, (0.9, 0.999), 1e-8, 0.0, zero_grad=0)
    torch.cuda.synchronize()
    assert torch.equal(g, torch.full_like(p, 0.5))
    # first step of Adam moves every entry by lr against the gradient's sign
    torch.testing.assert_close(p, torch.full_like(p, 1.0 - 1e-3), rtol=0, atol=1e-7)


def test_trainer_update_matches_torch_adam(cuda_device):
    """The Trainer's update (fused Adam over the table and the MLP, fp16 copy
    refreshed) equals torch.optim.Adam over the same two parameters."""
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    geo = Geometry(nDetector=[32, 32], dDetector=[1 / 32, 1 / 32], mode="parallel", nVoxel=[32] * 3,
                   dVoxel=[1 / 32] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=12, base_resolution=4,
                            finest_resolution=128)
    m = HashGrid(enc, MLPNetConfig(), precision="mixed", device=cuda_device)
    tr = Trainer(m, geo, points_per_batch=512 * 32, points_per_ray=32, loss="l2", lr=2e-3, device=cuda_device,
                 betas=(0.85, 0.99), weight_decay=1e-3)
    ref_t = m.table.detach().clone().requires_grad_(True)
    ref_m = m.mlp.detach().clone().requires_grad_(True)
    opt = torch.optim.Adam([ref_t, ref_m], lr=2e-3, betas=(0.85, 0.99), weight_decay=1e-3)
    gen = torch.Generator(device="cpu").manual_seed(9)
    for _ in range(3):
        gt = torch.randn(m.table.shape, generator=gen).to(cuda_device)
        gm = torch.randn(m.mlp.shape, generator=gen).to(cuda_device)
        ref_t.grad, ref_m.grad = gt.clone(), gm.clone()
        opt.step()
        tr.table_grad.copy_(gt)
        tr.mlp_grad.copy_(gm)
        tr._update(tr.table_grad, tr.mlp_grad)
    torch.cuda.synchronize()
    torch.testing.assert_close(m.table.detach(), ref_t.detach(), rtol=1e-6, atol=1e-8)
    torch.testing.assert_close(m.mlp.detach(), ref_m.detach(), rtol=1e-6, atol=1e-8)
    assert torch.equal(m.table_half.view(torch.int16), m.table.detach().half().view(torch.int16))
    assert not tr.table_grad.any() and not tr.mlp_grad.any()


def test_adam_vector_and_scalar_paths_agree(cuda_device):
    """Buffers 16-byte aligned take the four-element path; the same data one
    element off that alignment take the one-element path: bit-identical."""
    gen = torch.Generator(device="cpu").manual_seed(11)
    n = 4099
    bufs = [torch.randn(n + 1, generator=gen).to(cuda_device) for _ in range(4)]
    bufs[3] = bufs[3].abs()
    a = [b[:n].clone() for b in bufs]                       # aligned
    u = [torch.zeros(n + 1, device=cuda_device) for _ in range(4)]
    for dst, b in zip(u, bufs):
        dst[1:] = b[:n]
    u = [b[1:] for b in u]                                  # 4 bytes past alignment
    ha = torch.empty(n, dtype=torch.float16, device=cuda_device)
    hu = torch.empty(n + 1, dtype=torch.float16, device=cuda_device)[1:]
    for step in (1, 2):
        _adam(a[0], a[1], a[2], a[3], step, 1e-3, (0.9, 0.999), 1e-8, 1e-2, half=ha, zero_grad=0)
        _adam(u[0], u[1], u[2], u[3], step, 1e-3, (0.9, 0.999), 1e-8, 1e-2, half=hu, zero_grad=0)
    torch.cuda.synchronize()
    for x, y in zip(a + [ha], u + [hu]):
        assert torch.equal(x, y)
