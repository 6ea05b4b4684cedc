"""GPU parity of the hash-grid encoding, the model forward and the fused
training step (called through the C ABI) against the fp64 oracle.

Tolerances (plain fp32 path vs fp64 oracle): hash indices bit-exact;
interpolation weights bit-exact (the oracle's fp32 weights: the rounded
position's fraction, products in axis order); encodings and sigma rel
1e-5; y_pred and loss rel 1e-4; gradients within 1e-3 of the largest
gradient entry.
"""
import contextlib
import math

import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def tuning(**values):
    """The library's tuning with ``values`` set, restored afterwards."""
    from nect_b200 import autotune

    before = autotune.get_tuning()
    autotune.set_tuning(dict(before, **values))
    try:
        yield
    finally:
        autotune.set_tuning(before)


def make_model(n_dims, log2_T=12, base=4, finest=128, precision="plain_fp32", table_scale=0.5, seed=0,
               out_act="Softplus"):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=log2_T, base_resolution=base,
                            finest_resolution=finest, base_resolution_t=2 if n_dims == 4 else None)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=64, activation="ReLU", output_activation=out_act)
    cls = HashGrid if n_dims == 3 else HashGrid4D
    m = cls(enc, net, precision=precision, device="cuda", seed=seed)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(seed + 1)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * table_scale)
        m.refresh_half()
    return m, enc


def oracle_levels(m, enc, n_dims):
    levels, total = ohg.layout(n_dims, 16, enc.log2_hashmap_size, float(enc.base_resolution),
                               float(enc.per_level_scale), float(enc.base_resolution_t or enc.base_resolution))
    return levels, total


@pytest.mark.parametrize("n_dims", [3, 4])
def test_layout_matches_oracle(cuda_device, n_dims):
    m, enc = make_model(n_dims)
    levels, total = oracle_levels(m, enc, n_dims)
    assert m.table.shape[0] == total
    assert [lv.offset for lv in levels] == m.level_offset
    assert [lv.hashed for lv in levels] == m.level_hashed
    assert any(m.level_hashed) and not all(m.level_hashed)


@pytest.mark.parametrize("n_dims", [3, 4])
def test_corner_indices_bit_exact(cuda_device, n_dims):
    m, enc = make_model(n_dims)
    levels, _ = oracle_levels(m, enc, n_dims)
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.rand(4096, n_dims, generator=g)
    x[:64] = torch.round(x[:64] * 8) / 8          # exact vertices
    x[64:80] = 1.0                                # upper boundary
    x[80:96] = 0.0
    idx, w = m.corners(x.cuda())
    idx, w = idx.cpu(), w.cpu()
    for l, lv in enumerate(levels):
        oi, ow = ohg.corner_indices(x, lv, enc.log2_hashmap_size)
        assert torch.equal(idx[:, l].to(torch.int64), oi), f"level {l} indices differ"
        assert torch.equal(w[:, l], ow), f"level {l} weights differ"


@pytest.mark.parametrize("n_dims,precision", [(3, "plain_fp32"), (4, "plain_fp32"), (3, "mixed"), (4, "mixed")])
def test_model_forward_matches_oracle(cuda_device, n_dims, precision):
    m, enc = make_model(n_dims, precision=precision)
    levels, _ = oracle_levels(m, enc, n_dims)
    g = torch.Generator(device="cpu").manual_seed(4)
    x = torch.rand(3000, 3, generator=g)
    t = 0.37
    out = (m(x.cuda()) if n_dims == 3 else m(x.cuda(), t)).cpu().double()
    xin = x if n_dims == 3 else torch.cat([x, torch.full((x.shape[0], 1), t)], 1)
    table = m.grid_table.detach().cpu().double()
    Ws = ohg.split_mlp_params(m.mlp.detach().cpu().double(), 32, 64, 2)
    ref = ohg.mlp(ohg.encode(xin, table, levels, enc.log2_hashmap_size), Ws, "relu", "softplus")
    assert torch.allclose(out, ref, rtol=1e-5, atol=1e-6), (out - ref).abs().max()


def run_train_case(n_dims, precision, loss, geom_kind="parallel", duplicates=False, ws=None, t=0.45):
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import RayBatch, Workspace, train_step

    torch.manual_seed(11)
    if geom_kind == "parallel":
        geo = Geometry(nDetector=[32, 32], dDetector=[1 / 32, 1 / 32], mode="parallel", nVoxel=[32, 32, 32],
                       dVoxel=[1 / 32] * 3)
    else:
        geo = Geometry(nDetector=[40, 48], dDetector=[1.5, 1.5], mode="cone", DSD=300.0, DSO=200.0,
                       nVoxel=[32, 32, 32], dVoxel=[1.0] * 3)
    m, enc = make_model(n_dims, precision=precision)
    cg = geo.get_c_geometry()
    P = geo.nDetector[0] * geo.nDetector[1]
    S, R, start = 64, 700, 100
    perm = torch.randperm(P, device="cuda")
    if duplicates:  # a batch that repeats pixels (scheduler falls back to batch order)
        perm[start + 1:start + 40] = perm[start]
    jitter = torch.rand(R, device="cuda") - 0.5
    det_off = torch.zeros(R, 2, device="cuda")
    proj = torch.rand(P, device="cuda")
    angle = 0.7
    maxd = geo.max_distance_traveled / S
    batch = RayBatch(perm=perm, start=start, num_rays=R, points_per_ray=S, angle=angle,
                     max_ray_distance_per_point=maxd, jitter=jitter, detector_offset=det_off, projection=proj, t=t)
    tg = torch.zeros_like(m.table)
    mg = torch.zeros_like(m.mlp)
    L, y_pred = train_step(m, cg, batch, geo.max_distance_traveled, tg, mg, ws if ws is not None else Workspace(),
                           loss)
    torch.cuda.synchronize()
    # oracle: same samples (C oracle with the device's trig values), fp64 network
    a = torch.tensor([angle, 0.0], dtype=torch.float32, device="cuda")
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
    pts, dist, counts = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), start, R, S, angle, maxd, True,
                                            jitter.cpu().numpy(), det_off.cpu().numpy(), trig=trig)
    levels, _ = oracle_levels(m, enc, n_dims)
    measured = proj.cpu().numpy()[perm.cpu().numpy()[start:start + R]]
    yo, Lo, gto, gmo = ohg.train_step(pts, counts, dist, measured, m.grid_table.detach().cpu(),
                                      m.mlp.detach().cpu(), levels, enc.log2_hashmap_size, 32, 64, 2,
                                      geo.max_distance_traveled, loss=loss, t=t if n_dims == 4 else None)
    return (y_pred.cpu().double(), float(L.item()), tg.cpu().double(), mg.cpu().double()), (yo, float(Lo), gto, gmo)


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


@pytest.mark.parametrize("n_dims,loss,geom", [(3, "l2", "parallel"), (3, "l1", "cone"), (4, "l2", "cone")])
def test_fused_plain_step_matches_oracle(cuda_device, n_dims, loss, geom):
    (y, L, gt, gm), (yo, Lo, gto, gmo) = run_train_case(n_dims, "plain_fp32", loss, geom)
    assert rel_max(y, yo) < 1e-4
    assert abs(L - Lo) / abs(Lo) < 1e-4
    assert rel_max(gm, gmo) < 1e-3, rel_max(gm, gmo)
    assert rel_max(gt, gto) < 1e-3, rel_max(gt, gto)


def cosine(a, b):
    a, b = a.flatten(), b.flatten()
    return float((a @ b) / (a.norm() * b.norm()).clamp(min=1e-30))


@pytest.mark.parametrize("n_dims,loss,geom", [(3, "l2", "parallel"), (3, "l2", "cone"), (4, "l1", "cone")])
def test_fused_mixed_step_matches_oracle(cuda_device, n_dims, loss, geom):
    """Mixed path (fp16 table, bf16 tensor-core MLP, fp32 accumulation) vs the
    fp64 oracle evaluated on the same fp16 table values.  Tolerances: y_pred
    within 2e-2 of max|y_pred|; gradients with cosine similarity > 0.99 and
    max deviation < 5e-2 of the largest entry (bf16 operands carry 8 bits of
    mantissa)."""
    (y, L, gt, gm), (yo, Lo, gto, gmo) = run_train_case(n_dims, "mixed", loss, geom)
    assert rel_max(y, yo) < 2e-2, rel_max(y, yo)
    assert abs(L - Lo) / abs(Lo) < 5e-2
    assert cosine(gm, gmo) > 0.99, cosine(gm, gmo)
    assert cosine(gt, gto) > 0.99, cosine(gt, gto)
    assert rel_max(gm, gmo) < 5e-2, rel_max(gm, gmo)
    assert rel_max(gt, gto) < 5e-2, rel_max(gt, gto)


def test_mixed_error_word_clear(cuda_device):
    """The bounded mbarrier waits of the tensor-core kernels never time out."""
    from nect_b200.trainer import Workspace

    for n_dims in (3, 4):
        ws = Workspace()
        run_train_case(n_dims, "mixed", "l2", "cone", ws=ws)
        assert ws.error_word() == 0


@pytest.mark.parametrize("n_dims,duplicates", [(3, False), (4, False), (4, True)])
def test_staged_and_fused_backward_agree(cuda_device, n_dims, duplicates):
    """The two-pass backward (tensor-core pass staging dL/d(encoding), scatter
    passes per level group, 8 rounds) and the single fused pass give the same
    gradients up to fp32 reassociation of the reductions.  In 4D the time
    slice is off here: it is compared with the 4D kernels below."""
    from nect_b200.trainer import Workspace

    with tuning(time_slice=0):
        (y1, L1, gt1, gm1), _ = run_train_case(n_dims, "mixed", "l2", "cone", duplicates, ws=Workspace(staging=True))
    (y2, L2, gt2, gm2), _ = run_train_case(n_dims, "mixed", "l2", "cone", duplicates, ws=Workspace(staging=False))
    assert torch.equal(y1, y2)
    assert abs(L1 - L2) <= 1e-5 * abs(L2)   # the loss is an fp32 atomic sum over blocks
    assert rel_max(gt1, gt2) < 1e-5, rel_max(gt1, gt2)
    assert rel_max(gm1, gm2) < 1e-5, rel_max(gm1, gm2)


@pytest.mark.parametrize("n_dims,duplicates,store_rows", [(3, False, 5600), (4, True, 5600), (3, False, 0),
                                                           (4, False, 0)])
def test_encoding_store_partial_and_absent(cuda_device, n_dims, duplicates, store_rows):
    """The staged backward reads the rows the forward stored and gathers the
    rest: a store smaller than the batch's samples (rays beyond it recompute)
    and no store at all give the single fused pass's results."""
    from nect_b200.trainer import Workspace

    R, S, row_bytes = 700, 64, 32 * 2

    class Trimmed(Workspace):
        # passes the C ABI a workspace smaller than the recommended one by the
        # store rows it should not have
        def get(self, model, c_geometry, num_rays, device, points_per_ray=0):
            ptr, n = super().get(model, c_geometry, num_rays, device, points_per_ray)
            return ptr, n - (R * S - store_rows) * row_bytes - (256 if store_rows == 0 else 0)

    ws = Trimmed(staging=True)
    with tuning(time_slice=0):   # the exact comparison; the time slice is tested on its own
        (y1, L1, gt1, gm1), _ = run_train_case(n_dims, "mixed", "l2", "cone", duplicates, ws=ws)
    assert ws.error_word() == 0
    (y2, L2, gt2, gm2), _ = run_train_case(n_dims, "mixed", "l2", "cone", duplicates, ws=Workspace(staging=False))
    assert torch.equal(y1, y2)
    assert abs(L1 - L2) <= 1e-5 * abs(L2)
    assert rel_max(gt1, gt2) < 1e-5, rel_max(gt1, gt2)
    assert rel_max(gm1, gm2) < 1e-5, rel_max(gm1, gm2)


@pytest.mark.parametrize("duplicates,t", [(False, 0.45), (True, 0.45), (False, 0.0), (False, 1.0)])
def test_time_slice_matches_4d_kernels(cuda_device, duplicates, t):
    """A 4D mixed step on the time slice at the batch's t (8-corner 3D
    kernels, gradients spread back to the two time vertices) against the same
    step on the 16-corner 4D kernels.  The slice is fp16, so its values carry
    one more fp16 rounding (2^-11) before the bf16 rounding (2^-8) of the MLP
    input, and a bf16 rounding can flip: y_pred within 1e-2 of the largest,
    gradients with cosine > 0.999 and within 5e-2 of the largest entry (the
    mixed path's tolerance against the oracle).  The same step against the fp64
    oracle is test_fused_mixed_step_matches_oracle (4D, default tuning)."""
    from nect_b200.trainer import Workspace

    (y1, L1, gt1, gm1), (yo, Lo, gto, gmo) = run_train_case(4, "mixed", "l2", "cone", duplicates, ws=Workspace(), t=t)
    with tuning(time_slice=0):
        (y2, L2, gt2, gm2), _ = run_train_case(4, "mixed", "l2", "cone", duplicates, ws=Workspace(), t=t)
    # t = 0 and t = 1 put the blend on the first and the last time vertex
    assert cosine(gt1, gto) > 0.99 and rel_max(y1, yo) < 2e-2, (cosine(gt1, gto), rel_max(y1, yo))
    assert rel_max(y1, y2) < 1e-2, rel_max(y1, y2)
    assert abs(L1 - L2) <= 1e-2 * abs(L2)
    assert cosine(gt1, gt2) > 0.999 and cosine(gm1, gm2) > 0.999, (cosine(gt1, gt2), cosine(gm1, gm2))
    assert rel_max(gt1, gt2) < 5e-2 and rel_max(gm1, gm2) < 5e-2, (rel_max(gt1, gt2), rel_max(gm1, gm2))


@pytest.mark.parametrize("fraction", [0.3, 0.05])
def test_partial_staging_budget(cuda_device, fraction):
    """A workspace with a share of the recommended staging (fewer store rows,
    or no store and more rounds) gives the single fused pass's results."""
    from nect_b200.trainer import Workspace

    (y1, L1, gt1, gm1), _ = run_train_case(3, "mixed", "l2", "cone", ws=Workspace(staging_fraction=fraction))
    (y2, L2, gt2, gm2), _ = run_train_case(3, "mixed", "l2", "cone", ws=Workspace(staging=False))
    assert torch.equal(y1, y2)
    assert rel_max(gt1, gt2) < 1e-5, rel_max(gt1, gt2)
    assert rel_max(gm1, gm2) < 1e-5, rel_max(gm1, gm2)


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_batch_with_repeated_pixels(cuda_device, precision):
    """Every ray of the batch is processed when pixels repeat (the pixel-order
    scheduler's fallback), with the same tolerances as above."""
    (y, L, gt, gm), (yo, Lo, gto, gmo) = run_train_case(3, precision, "l2", "cone", duplicates=True)
    tol = 1e-4 if precision == "plain_fp32" else 2e-2
    assert rel_max(y, yo) < tol
    assert cosine(gt, gto) > 0.99


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_edge_batches(cuda_device, precision):
    """Empty batch; a batch whose rays all miss the object (detector shifted
    off the volume: no samples, y_pred 0, loss from the measured values only,
    no gradient); one sample per ray."""
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import RayBatch, Workspace, train_step

    m, enc = make_model(3, precision=precision)
    P = 32 * 32
    perm = torch.randperm(P, device="cuda")
    proj = torch.rand(P, device="cuda")

    def step(geo, R, S):
        batch = RayBatch(perm=perm, start=0, num_rays=R, points_per_ray=S, angle=0.3,
                         max_ray_distance_per_point=geo.max_distance_traveled / S,
                         jitter=torch.zeros(max(R, 1), device="cuda"),
                         detector_offset=torch.zeros(max(R, 1), 2, device="cuda"), projection=proj)
        tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
        L, y = train_step(m, geo.get_c_geometry(), batch, geo.max_distance_traveled, tg, mg, Workspace(), "l2")
        torch.cuda.synchronize()
        return float(L), y, tg, mg

    geo = Geometry(nDetector=[32, 32], dDetector=[1 / 32, 1 / 32], mode="parallel", nVoxel=[32] * 3,
                   dVoxel=[1 / 32] * 3)
    L, y, tg, mg = step(geo, 0, 16)
    assert L == 0.0 and y.numel() == 0 and not tg.any() and not mg.any()

    off = Geometry(nDetector=[32, 32], dDetector=[1 / 32, 1 / 32], mode="parallel", nVoxel=[32] * 3,
                   dVoxel=[1 / 32] * 3, offDetector=(5.0, 5.0))
    L, y, tg, mg = step(off, 300, 16)
    meas = proj[perm[:300]]
    assert not y.any() and not tg.any() and not mg.any()
    assert abs(L - float((meas * meas).mean())) <= 1e-6 * float((meas * meas).mean())

    L, y, tg, mg = step(geo, 300, 1)
    assert math.isfinite(L) and (y != 0).sum() > 100 and tg.abs().sum() > 0
