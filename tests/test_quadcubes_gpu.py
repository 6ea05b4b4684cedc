"""The reference's default dynamic model, QuadCubes (nect/network/networks.py:
392-449): forward and backward against an fp64 restatement built from the
oracle's hash-grid encoding (four 3D grids over (z,y,x), (y,x,t), (x,z,t),
(z,y,t), the raw inputs appended, a bias-free MLP), the encoder backward
kernel against autograd through the oracle, and fit() training it on a
small dynamic scan through the module loop.

Tolerances: plain fp32 forward within 1e-5 of the largest output, gradients
within 1e-4 of the largest entry of each parameter."""
import math

import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg

pytestmark = pytest.mark.gpu


def make(precision="plain_fp32", identity=True, F=4, hidden=2):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.quadcubes import QuadCubes

    enc = HashEncoderConfig(n_levels=6, n_features_per_level=F, log2_hashmap_size=11, base_resolution=4,
                            finest_resolution=48)
    net = MLPNetConfig(n_hidden_layers=hidden, n_neurons=128, activation="LeakyReLU", output_activation="None",
                       include_identity=identity)
    m = QuadCubes(enc, net, precision=precision, device="cuda", seed=3)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(5)
        for tab in m.tables:
            tab.copy_((torch.rand(tab.shape, generator=g) * 2 - 1) * 0.5)
    levels, _ = ohg.layout(3, 6, 11, 4.0, float(enc.per_level_scale))
    return m, levels


def oracle_forward(m, levels, x, t, tables=None, weights=None):
    """fp64 QuadCubes: the four grids' oracle encodings, the raw inputs, the MLP."""
    x = x.double()
    tcol = torch.full((x.shape[0], 1), float(t), dtype=torch.float64)
    ins = [x, torch.cat([x[:, [1, 2]], tcol], 1), torch.cat([x[:, [2, 0]], tcol], 1),
           torch.cat([x[:, [0, 1]], tcol], 1)]
    tables = tables if tables is not None else [tab.detach().cpu().double() for tab in m.tables]
    feats = [ohg.encode(inp.float(), tab, levels, 11) for inp, tab in zip(ins, tables)]
    if m.include_identity:
        feats.append(torch.cat([x, tcol], 1))
    weights = weights if weights is not None else [lin.weight.detach().cpu().double() for lin in m.layers]
    return ohg.mlp(torch.cat(feats, 1), weights, act="leakyrelu", out_act="none")


def rel(a, b):
    a, b = torch.as_tensor(a).double().flatten(), torch.as_tensor(b).double().flatten()
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("identity", [True, False])
def test_forward_matches_oracle(cuda_device, identity):
    m, levels = make(identity=identity)
    gen = torch.Generator(device="cpu").manual_seed(1)
    x = torch.rand(3000, 3, generator=gen)
    for t in (0.0, 0.37, 1.0):
        y = m(x.cuda(), t)
        assert y.shape == (3000, 1)
        assert rel(y.detach().cpu(), oracle_forward(m, levels, x, t)) < 1e-5
    # a CUDA timestep gives the same values
    y_dev = m(x.cuda(), torch.tensor(0.37, device="cuda"))
    assert torch.equal(y_dev, m(x.cuda(), 0.37))


def test_backward_matches_fp64_autograd(cuda_device):
    m, levels = make()
    gen = torch.Generator(device="cpu").manual_seed(2)
    x = torch.rand(2000, 3, generator=gen)
    g = torch.randn(2000, 1, generator=gen)
    t = 0.61
    (m(x.cuda(), t) * g.cuda()).sum().backward()
    tables = [tab.detach().cpu().double().requires_grad_() for tab in m.tables]
    weights = [lin.weight.detach().cpu().double().requires_grad_() for lin in m.layers]
    (oracle_forward(m, levels, x, t, tables, weights) * g.double()).sum().backward()
    for tab, ref in zip(m.tables, tables):
        assert rel(tab.grad.cpu(), ref.grad) < 1e-4, rel(tab.grad.cpu(), ref.grad)
    for lin, ref in zip(m.layers, weights):
        assert rel(lin.weight.grad.cpu(), ref.grad) < 1e-4, rel(lin.weight.grad.cpu(), ref.grad)


def test_encoder_backward_kernel_against_autograd(cuda_device):
    """nectb_hashgrid_encode_backward alone: the table gradient of
    sum(encode(x) * dout) against autograd through the oracle's encoding."""
    m, levels = make(F=2)
    gen = torch.Generator(device="cpu").manual_seed(4)
    x = torch.rand(5000, 3, generator=gen)
    from nect_b200.quadcubes import GridEncode

    tab = m.tables[0]
    out = GridEncode.apply(tab, m.desc, m.n_enc, x.cuda())
    dout = torch.randn(out.shape, generator=gen)
    (out * dout.cuda()).sum().backward()
    ref_tab = tab.detach().cpu().double().requires_grad_()
    (ohg.encode(x, ref_tab, levels, 11) * dout.double()).sum().backward()
    assert rel(tab.grad.cpu(), ref_tab.grad) < 1e-5


def test_fit_trains_quadcubes_on_a_dynamic_scan(cuda_device):
    """fit() on dynamic data builds the reference's default dynamic model
    (here at a small size) and trains it by the module loop: the volume error
    at t = 0.5 falls."""
    from nect_b200 import phantoms
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig
    from nect_b200.quadcubes import ModuleTrainer, QuadCubes
    from nect_b200.reconstruct import fit, psnr
    from nect_b200.sampling import Geometry

    n = 32
    geo = Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3, dVoxel=[1 / n] * 3)
    ph = phantoms.ellipsoid_phantom(8, 1)
    angles = np.linspace(0, 4 * math.pi, 80, endpoint=False)
    projs = torch.stack([phantoms.ellipsoid_projection(ph, geo, float(a), "cuda") for a in angles])
    truth = phantoms.ellipsoid_volume(ph, n, "cuda")
    ts = list(np.linspace(0, 1, len(angles)))
    enc = HashEncoderConfig(n_levels=8, n_features_per_level=4, log2_hashmap_size=14, base_resolution=4,
                            finest_resolution=64)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=128, activation="LeakyReLU", output_activation="None",
                       include_identity=True)
    rec = fit(geo, projs, list(angles), timesteps=ts, model_cfg=ModelConfig("quadcubes", enc, net, "plain_fp32"),
              niter=400, lr=2e-3, rays_per_batch=1024, points_per_ray=64, seed=0,
              evaluate=lambda r: {"psnr": psnr(r.volume(0.5), truth)}, eval_every=400)
    assert isinstance(rec.model, QuadCubes) and isinstance(rec.trainer, ModuleTrainer)
    first, last = rec.history[0][2]["psnr"], rec.history[-1][2]["psnr"]
    assert math.isfinite(last) and last > first + 5, (first, last)


def _rows(m, x, t, dtype):
    from nect_b200.quadcubes import QuadEncode

    m.precision = "mixed" if dtype == torch.bfloat16 else "plain_fp32"
    m.row_width = -(-m.n_in // 64) * 64 if dtype == torch.bfloat16 else -(-m.n_in // 4) * 4
    return QuadEncode.apply(*m.tables, m, x, torch.full((1,), t, device="cuda"))


@pytest.mark.parametrize("F", [2, 4])
def test_composite_rows_match_the_3d_grids(cuda_device, F):
    """nectb_quadcubes_encode against the per-grid 3D encoder
    (nectb_hashgrid_encode): the planes at t equal the trilinear grids up to
    fp32 reassociation (fp32 rows, 1e-5 of the largest entry) and one fp16 +
    one bf16 rounding (bf16
    rows); identity columns exact, padding zero.  The small table puts levels
    in all three plane forms (dense 3D, dense plane of a hashed level, hashed
    plane)."""
    from nect_b200.quadcubes import GridEncode

    m, _ = make(F=F)
    forms = set()
    for r in ohg.layout(3, 6, 11, 4.0, float(m.encoding_config.per_level_scale))[0]:
        v = r.res[0] + 1
        forms.add("dense" if v ** 3 <= 2048 else ("plane" if v ** 2 <= 2048 else "hashed"))
    assert forms == {"dense", "plane", "hashed"}, forms
    gen = torch.Generator(device="cpu").manual_seed(7)
    x = torch.rand(4000, 3, generator=gen).cuda()
    x[:7] = torch.tensor([[0, 0, 0], [1, 1, 1], [1, 0, 1], [0.5, 0.5, 0.5], [0, 1, 0], [1e-7, 1, 0.999999], [0.25, 0.75, 1]],
                         device="cuda")
    for t in (0.0, 0.43, 1.0):
        tcol = torch.full((x.shape[0], 1), t, device="cuda")
        ins = (x, torch.cat([x[:, [1, 2]], tcol], 1), torch.cat([x[:, [2, 0]], tcol], 1),
               torch.cat([x[:, [0, 1]], tcol], 1))
        ref = torch.cat([GridEncode.apply(tab, m.desc, m.n_enc, i.contiguous()) for tab, i in zip(m.tables, ins)]
                        + [x, tcol], 1).detach()
        rows = _rows(m, x, t, torch.float32).detach()
        assert rows.shape == (x.shape[0], m.row_width)
        assert rel(rows[:, :m.n_in].cpu(), ref.cpu()) < 1e-5
        assert torch.equal(rows[:, 4 * m.n_enc:m.n_in], ref[:, 4 * m.n_enc:])
        rows16 = _rows(m, x, t, torch.bfloat16).detach()
        assert rows16.dtype == torch.bfloat16 and rows16.shape[1] % 64 == 0
        assert rel(rows16[:, :m.n_in].float().cpu(), ref.cpu()) < 8e-3
        assert not rows16[:, m.n_in:].any()


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_composite_backward_matches_the_3d_grids(cuda_device, dtype):
    """nectb_quadcubes_encode_backward (planes' gradients spread to the two
    time vertices) against nectb_hashgrid_encode_backward of each 3D grid on
    the same dL/d(rows), fp32 or bf16 rows."""
    from nect_b200.quadcubes import GridEncode

    m, _ = make(F=4)
    gen = torch.Generator(device="cpu").manual_seed(8)
    x = torch.rand(6000, 3, generator=gen).cuda()
    t = 0.71
    rows = _rows(m, x, t, dtype)
    dout = torch.randn(rows.shape, generator=gen).to(device="cuda", dtype=dtype)
    got = torch.autograd.grad((rows.float() * dout.float()).sum(), list(m.tables))
    tcol = torch.full((x.shape[0], 1), t, device="cuda")
    ins = (x, torch.cat([x[:, [1, 2]], tcol], 1), torch.cat([x[:, [2, 0]], tcol], 1),
           torch.cat([x[:, [0, 1]], tcol], 1))
    for k, (tab, i) in enumerate(zip(m.tables, ins)):
        out = GridEncode.apply(tab, m.desc, m.n_enc, i.contiguous())
        d = dout[:, k * m.n_enc:(k + 1) * m.n_enc].float()
        (ref,) = torch.autograd.grad((out * d).sum(), [tab])
        assert rel(got[k].cpu(), ref.cpu()) < 1e-5, (k, rel(got[k].cpu(), ref.cpu()))


def test_mixed_forward_and_backward_match_the_oracle(cuda_device):
    """The mixed path (fp16 planes, bf16 rows and MLP, fp32 accumulation)
    against the fp64 oracle: outputs within 2e-2 of the largest, gradients
    with cosine > 0.99 and within 1e-1 of each parameter's largest entry (the
    128-wide bf16 GEMMs' backward rounds dL/d(rows) to bf16; measured 6e-2)."""
    m, levels = make(precision="mixed")
    gen = torch.Generator(device="cpu").manual_seed(9)
    x = torch.rand(3000, 3, generator=gen)
    g = torch.randn(3000, 1, generator=gen)
    t = 0.29
    y = m(x.cuda(), t)
    (y * g.cuda()).sum().backward()
    tables = [tab.detach().cpu().double().requires_grad_() for tab in m.tables]
    weights = [lin.weight.detach().cpu().double().requires_grad_() for lin in m.layers]
    ref = oracle_forward(m, levels, x, t, tables, weights)
    assert rel(y.detach().cpu(), ref.detach()) < 2e-2
    (ref * g.double()).sum().backward()
    for p, r in [(tab, rt) for tab, rt in zip(m.tables, tables)] + [(lin.weight, rw) for lin, rw in
                                                                     zip(m.layers, weights)]:
        a, b = p.grad.cpu().double().flatten(), r.grad.flatten()
        assert float(torch.dot(a, b) / (a.norm() * b.norm())) > 0.99
        assert rel(a, b) < 1e-1, rel(a, b)


def test_composite_encoder_at_the_preset_size(cuda_device):
    """The reference's preset (quadcubes.yaml: 23 levels x 4 features, 2^23
    entries, base 16) on a 512^2 detector's finest resolution 1024: planes of
    up to 1024^2 vertices on hashed levels.  Rows (fp32) and table gradients
    of 200,000 points against the per-grid 3D kernels, within 2e-5 of the
    largest entry (fp32 reassociation)."""
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.quadcubes import GridEncode, QuadCubes

    enc = HashEncoderConfig(n_levels=23, n_features_per_level=4, log2_hashmap_size=23, base_resolution=16,
                            finest_resolution=1024)
    net = MLPNetConfig(n_hidden_layers=4, n_neurons=128, activation="LeakyReLU", output_activation="None",
                       include_identity=True)
    m = QuadCubes(enc, net, device="cuda", seed=4)
    with torch.no_grad():
        for tab in m.tables:
            tab.mul_(5000.0)   # U(-0.5, 0.5)
    gen = torch.Generator(device="cpu").manual_seed(12)
    x = torch.rand(200_000, 3, generator=gen).cuda()
    t = 0.57
    tcol = torch.full((x.shape[0], 1), t, device="cuda")
    ins = (x, torch.cat([x[:, [1, 2]], tcol], 1), torch.cat([x[:, [2, 0]], tcol], 1),
           torch.cat([x[:, [0, 1]], tcol], 1))
    rows = _rows(m, x, t, torch.float32)
    dout = torch.randn(rows.shape, generator=gen).cuda()
    got = torch.autograd.grad((rows * dout).sum(), list(m.tables))
    for k, (tab, i) in enumerate(zip(m.tables, ins)):
        out = GridEncode.apply(tab, m.desc, m.n_enc, i.contiguous())
        cols = slice(k * m.n_enc, (k + 1) * m.n_enc)
        assert rel(rows[:, cols].detach().cpu(), out.detach().cpu()) < 2e-5, k
        (ref,) = torch.autograd.grad((out * dout[:, cols]).sum(), [tab])
        assert rel(got[k].cpu(), ref.cpu()) < 2e-5, (k, rel(got[k].cpu(), ref.cpu()))
        del out, ref
