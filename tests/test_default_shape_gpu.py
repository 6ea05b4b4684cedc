"""The reference's default static model (nect/cfg/static/hash_grid.yaml:1-13):
19 levels x 4 features, base resolution 8, finest 2 x the detector extent,
6 hidden layers of 64 LeakyReLU with a ReLU output, on the kernels of both
precisions, against the fp64 oracle: corner indices, the module forward and
backward, the fused training step, the two-pass backward against the single
pass, queries, and training through fit().

Its 76 inputs take two bf16 tiles on the tensor-core path (layer 0 runs K
over 80, dX is an N = 128 product and the layer-0 weight gradient is taken
transposed), and the plain backward reads the PyTorch-layout weights from
global memory (both copies do not fit shared memory).

Tolerances: hash indices bit-exact; module forward (fp32 arithmetic in both
precisions) 1e-5 of the largest; module backward 1e-3 of the largest
gradient entry; plain training step y_pred 1e-4, gradients within 1e-2 of
the largest entry and 2e-3 in relative L2 norm (LeakyReLU's kink: a sample
whose pre-activation sits within fp32 rounding of 0 takes slope 1 or 0.01,
in fp32 arithmetic of either order); mixed step y_pred 3e-2 of the largest,
gradient cosine > 0.99 and max deviation < 8e-2 of the largest entry (bf16
operands through seven layers).
"""
import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu

L, F, H = 19, 4, 6


def make_model(precision, out_act="ReLU", n_dims=3, seed=0, log2_T=14):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid

    enc = HashEncoderConfig(n_levels=L, n_features_per_level=F, log2_hashmap_size=log2_T, base_resolution=8,
                            max_resolution_factor=2.0, nDetector=[40, 48])
    net = MLPNetConfig(n_hidden_layers=H, n_neurons=64, activation="LeakyReLU", output_activation=out_act)
    m = HashGrid(enc, net, precision=precision, device="cuda", seed=seed)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(seed + 1)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.5)
        m.refresh_half()
    return m, enc


def levels_of(enc):
    return ohg.layout(3, L, enc.log2_hashmap_size, float(enc.base_resolution), float(enc.per_level_scale))[0]


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


def rel_l2(a, b):
    return float((a - b).norm() / b.norm().clamp(min=1e-30))


def cosine(a, b):
    a, b = a.flatten(), b.flatten()
    return float((a @ b) / (a.norm() * b.norm()).clamp(min=1e-30))


def test_corner_indices_bit_exact(cuda_device):
    m, enc = make_model("plain_fp32")
    levels = levels_of(enc)
    assert m.table.shape[0] == sum(lv.entries for lv in levels)
    assert any(lv.hashed for lv in levels) and not all(lv.hashed for lv in levels)
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.rand(4096, 3, generator=g)
    x[:64] = torch.round(x[:64] * 8) / 8
    x[64:80] = 1.0
    idx, w = m.corners(x.cuda())
    idx, w = idx.cpu(), w.cpu()
    for l, lv in enumerate(levels):
        oi, ow = ohg.corner_indices(x, lv, enc.log2_hashmap_size)
        assert torch.equal(idx[:, l].to(torch.int64), oi), f"level {l}"
        assert torch.equal(w[:, l], ow)


@pytest.mark.parametrize("precision,out_act", [("plain_fp32", "ReLU"), ("mixed", "ReLU"), ("mixed", "Softplus")])
def test_module_forward_and_backward(cuda_device, precision, out_act):
    m, enc = make_model(precision, out_act)
    g = torch.Generator(device="cpu").manual_seed(4)
    x = torch.rand(3000, 3, generator=g)
    target = torch.rand(3000, 1, generator=g)
    out = m(x.cuda())
    torch.nn.functional.mse_loss(out, target.cuda()).backward()
    torch.cuda.synchronize()
    tab = m.grid_table.detach().cpu().double().requires_grad_(True)
    wf = m.mlp.detach().cpu().double().requires_grad_(True)
    ref = ohg.mlp(ohg.encode(x, tab, levels_of(enc), enc.log2_hashmap_size),
                  ohg.split_mlp_params(wf, L * F, 64, H), "leakyrelu", out_act.lower())
    torch.nn.functional.mse_loss(ref, target.double()).backward()
    assert rel_max(out.detach().cpu().double(), ref.detach()) < 1e-5
    assert rel_max(m.table.grad.cpu().double(), tab.grad) < 1e-3, rel_max(m.table.grad.cpu().double(), tab.grad)
    assert rel_max(m.mlp.grad.cpu().double(), wf.grad) < 1e-3, rel_max(m.mlp.grad.cpu().double(), wf.grad)


def run_step(precision, loss, out_act, ws=None):
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import RayBatch, Workspace, train_step

    torch.manual_seed(11)
    geo = Geometry(nDetector=[40, 48], dDetector=[1.5, 1.5], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[32] * 3,
                   dVoxel=[1.0] * 3)
    m, enc = make_model(precision, out_act)
    cg = geo.get_c_geometry()
    P = 40 * 48
    S, R, start = 64, 700, 100
    perm = torch.randperm(P, device="cuda")
    jitter = torch.rand(R, device="cuda") - 0.5
    det_off = torch.zeros(R, 2, device="cuda")
    proj = torch.rand(P, device="cuda")
    angle = 0.7
    maxd = geo.max_distance_traveled / S
    batch = RayBatch(perm=perm, start=start, num_rays=R, points_per_ray=S, angle=angle,
                     max_ray_distance_per_point=maxd, jitter=jitter, detector_offset=det_off, projection=proj)
    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    work = ws if ws is not None else Workspace()
    Lk, y = train_step(m, cg, batch, geo.max_distance_traveled, tg, mg, work, loss)
    torch.cuda.synchronize()
    assert work.error_word(cg) == 0
    a = torch.tensor([angle, 0.0], dtype=torch.float32, device="cuda")
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
    pts, dist, counts = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), start, R, S, angle, maxd, True,
                                            jitter.cpu().numpy(), det_off.cpu().numpy(), trig=trig)
    meas = proj.cpu().numpy()[perm.cpu().numpy()[start:start + R]]
    yo, Lo, gto, gmo = ohg.train_step(pts, counts, dist, meas, m.grid_table.detach().cpu(), m.mlp.detach().cpu(),
                                      levels_of(enc), enc.log2_hashmap_size, L * F, 64, H, geo.max_distance_traveled,
                                      loss=loss, act="leakyrelu", out_act=out_act.lower())
    return (y.cpu().double(), float(Lk), tg.cpu().double(), mg.cpu().double()), (yo, float(Lo), gto, gmo)


@pytest.mark.parametrize("precision,loss,out_act", [("plain_fp32", "l2", "Softplus"), ("plain_fp32", "l1", "ReLU"),
                                                    ("mixed", "l2", "Softplus"), ("mixed", "l2", "ReLU")])
def test_train_step_matches_oracle(cuda_device, precision, loss, out_act):
    (y, Lk, gt, gm), (yo, Lo, gto, gmo) = run_step(precision, loss, out_act)
    assert (y != 0).sum() > 100 and gto.abs().sum() > 0
    if precision == "plain_fp32":
        assert rel_max(y, yo) < 1e-4
        assert abs(Lk - Lo) <= 1e-4 * abs(Lo)
        for a, b in ((gt, gto), (gm, gmo)):
            assert rel_max(a, b) < 1e-2 and rel_l2(a, b) < 2e-3, (rel_max(a, b), rel_l2(a, b))
    else:
        assert rel_max(y, yo) < 3e-2, rel_max(y, yo)
        for a, b in ((gt, gto), (gm, gmo)):
            assert cosine(a, b) > 0.99 and rel_max(a, b) < 8e-2, (cosine(a, b), rel_max(a, b))


@pytest.mark.parametrize("store", [1, 0])
def test_two_pass_backward_matches_single_pass(cuda_device, store):
    """The staged backward (tensor-core pass + scatter passes, with or
    without the encoding store of 160-byte rows) against the single fused
    pass: the same gradients up to fp32 reassociation."""
    from nect_b200 import autotune
    from nect_b200.trainer import Workspace

    before = autotune.get_tuning()
    autotune.set_tuning(dict(before, encoding_store=store))
    try:
        (y1, L1, gt1, gm1), _ = run_step("mixed", "l2", "Softplus", ws=Workspace(staging=True))
    finally:
        autotune.set_tuning(before)
    (y2, L2, gt2, gm2), _ = run_step("mixed", "l2", "Softplus", ws=Workspace(staging=False))
    assert torch.equal(y1, y2)
    assert rel_max(gt1, gt2) < 1e-5 and rel_max(gm1, gm2) < 1e-5, (rel_max(gt1, gt2), rel_max(gm1, gm2))


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_volume_query_matches_module(cuda_device, precision):
    from nect_b200.serving import query_points, volume_items

    m, enc = make_model(precision, "Softplus")
    shape = (24, 20, 28)
    out = torch.empty(shape, device="cuda")
    query_points(m, volume_items(out, shape, 0.0))
    z, y, x = torch.meshgrid(*[(torch.arange(n, device="cuda") + 0.5) / n for n in shape], indexing="ij")
    pts = torch.stack((z.flatten(), y.flatten(), x.flatten()), 1)
    with torch.no_grad():
        ref = m(pts).view(shape)
    tol = 1e-4 if precision == "plain_fp32" else 3e-2   # the mixed query runs the bf16 tensor-core MLP
    assert rel_max(out, ref) < tol, rel_max(out, ref)


def test_fit_trains_the_reference_default_model(cuda_device):
    """fit() with the reference's default static model (the model reconstruct()
    builds for a static scan) learns the volume: PSNR rises well above the
    untrained network's."""
    import math

    from nect_b200 import phantoms
    from nect_b200.reconstruct import default_model_config, fit, psnr
    from nect_b200.sampling import Geometry

    n = 48
    geo = Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3, dVoxel=[1 / n] * 3)
    cfg = default_model_config(geo, "static", "mixed", log2_hashmap_size=17)
    assert (cfg.encoder.n_levels, cfg.encoder.n_features_per_level, cfg.net.n_hidden_layers) == (19, 4, 6)
    ph = phantoms.ellipsoid_phantom(20, 0)
    angles = np.linspace(0, math.pi, 40, endpoint=False)
    projs = torch.stack([phantoms.ellipsoid_projection(ph, geo, float(a), "cuda") for a in angles])
    truth = phantoms.ellipsoid_volume(ph, n, "cuda")
    rec = fit(geo, projs, angles, model_cfg=cfg, niter=300, lr=2e-3, points_per_ray=96,
              evaluate=lambda r: {"psnr": psnr(r.volume(), truth)}, eval_every=300)
    assert rec.history[-1][2]["psnr"] > rec.history[0][2]["psnr"] + 8, rec.history
