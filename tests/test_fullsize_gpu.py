"""Parity at the benchmark workloads' full sizes.

The small parity tests use 2^12-2^14 entry tables and detectors of 64^2 or
less.  Here the fused path runs the benchmark shapes themselves:

* static parallel 128^2, S 256, 16 x 2 fp32 features, 2^19 entries (one
  projection = 16,384 rays);
* static cone 512^2 (DSO 500, DSD 1000, 256^3 volume), S 512, 16 x 2
  features, 2^20 entries (one projection = 262,144 rays);
* 4D cone 512^2, S 512, 16 x 2 features, 2^21 entries, temporal base 4;
* large 4D cylindrical cone 2048^2 (a batch of 2^20 of its 4,194,304
  pixels), S 1024, 16 x 4 features, 2^22 entries, finest 4096, 3 x 64 MLP.

1. Sampling inside the fused path: the per-ray sample counts, integral scales
   and regenerated positions a training step prepares (nectb_train_rays) are
   bit-identical with the reference's own sampler (nect/sampling/
   ct_sampling.cu:475-576, built from its source into oracle/_ref) on the
   same random draws, and the counts with the C oracle (device trig values).
2. One training step per workload and precision against the fp64 oracle on a
   seeded subset of rays.  The step runs on the whole batch (full workspace,
   staging rounds, encoding store or recompute, time slice), in two halves:
   the forward's y_pred is compared on the subset; the backward gets
   dL/dy_pred nonzero on the subset only, so every other ray contributes an
   exact zero and the table and MLP gradients must equal the oracle's
   gradient of sum(dL/dy * y_pred) over the subset.  The fused single-call
   step on the same batch must give the split step's y_pred bit for bit, its
   loss within fp32 summation error, and its gradients within fp32
   reassociation.

Tolerances.  Plain fp32 with a smooth network (no hidden activation,
softplus output): y_pred 1e-4 and gradients 1e-4 of the largest entry,
5e-5 in relative L2 norm (measured: about 2e-6 and 5e-7, as plain fp32
arithmetic on the CPU).  Plain fp32 with ReLU hidden layers: y_pred 1e-4;
gradients within 1e-2 of the largest entry and 3e-3 in relative L2 norm,
because with a million samples some pre-activations sit within fp32
rounding of the kink, where either order of fp32 arithmetic may take the
other side (plain fp32 on the CPU deviates from fp64 by up to 1.7e-3 of
the largest entry on the same batch).  Mixed: y_pred 2e-2, gradients cosine
> 0.99 and max deviation < 5e-2 of the largest entry.
"""
import contextlib
import ctypes

import numpy as np
import pytest
import torch

from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu

WORKLOADS = {
    "c1_parallel": dict(geo=dict(nDetector=[128, 128], dDetector=[1 / 128, 1 / 128], mode="parallel",
                                 nVoxel=[128] * 3, dVoxel=[1 / 128] * 3),
                        n_dims=3, F=2, H=2, log2_T=19, base=16, finest=1024, base_t=None, S=256, rays=16384),
    "c2_cone": dict(geo=dict(nDetector=[512, 512], dDetector=[1.0, 1.0], mode="cone", DSD=1000.0, DSO=500.0,
                             nVoxel=[256] * 3, dVoxel=[1.0] * 3),
                    n_dims=3, F=2, H=2, log2_T=20, base=16, finest=None, base_t=None, S=512, rays=1 << 18),
    "c3_cone_4d": dict(geo=dict(nDetector=[512, 512], dDetector=[1.0, 1.0], mode="cone", DSD=1000.0, DSO=500.0,
                                nVoxel=[256] * 3, dVoxel=[1.0] * 3),
                       n_dims=4, F=2, H=2, log2_T=21, base=16, finest=None, base_t=4, S=512, rays=1 << 18),
    "c5_large_4d": dict(geo=dict(nDetector=[2048, 2048], dDetector=[1.0, 1.0], mode="cone", DSD=4000.0,
                                 DSO=2000.0, nVoxel=[1024] * 3, dVoxel=[1.0] * 3, reconstruction_mode="cylindrical"),
                        n_dims=4, F=4, H=3, log2_T=22, base=16, finest=4096, base_t=4, S=1024, rays=1 << 20),
}


@contextlib.contextmanager
def tuning(**values):
    from nect_b200 import autotune

    before = autotune.get_tuning()
    autotune.set_tuning(dict(before, **values))
    try:
        yield
    finally:
        autotune.set_tuning(before)


def build(name, precision, table_scale=0.5, seed=0, act="ReLU"):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D
    from nect_b200.sampling import Geometry

    w = WORKLOADS[name]
    geo = Geometry(**w["geo"])
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=w["F"], log2_hashmap_size=w["log2_T"],
                            base_resolution=w["base"], max_resolution_factor=2.0, nDetector=w["geo"]["nDetector"],
                            finest_resolution=w["finest"], base_resolution_t=w["base_t"])
    net = MLPNetConfig(n_hidden_layers=w["H"], n_neurons=64, activation=act, output_activation="Softplus")
    m = (HashGrid if w["n_dims"] == 3 else HashGrid4D)(enc, net, precision=precision, device="cuda", seed=seed)
    with torch.no_grad():
        g = torch.Generator(device="cuda").manual_seed(seed + 1)
        m.table.copy_((torch.rand(m.table.shape, generator=g, device="cuda") * 2 - 1) * table_scale)
        m.refresh_half()
    return w, geo, m, enc


def device_trig(angle):
    a = torch.tensor([angle, 0.0], dtype=torch.float32, device="cuda")
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    return np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)


def ref_geometry(ref, cg):
    kw = {f: getattr(cg, f) for f in cg._fields}
    return getattr(ref, type(cg).__name__)(**kw)


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


def rel_l2(a, b):
    return float((a - b).norm() / b.norm().clamp(min=1e-30))


def cosine(a, b):
    a, b = a.flatten(), b.flatten()
    return float((a @ b) / (a.norm() * b.norm()).clamp(min=1e-30))


def train_rays(cg, R, S, ws_ptr, points=True):
    from nect_b200 import _lib

    counts = torch.empty(R, dtype=torch.int32, device="cuda")
    scale = torch.empty(R, dtype=torch.float32, device="cuda")
    pts = torch.empty(R, S, 3, dtype=torch.float32, device="cuda") if points else None
    rc = _lib.lib.nectb_train_rays(ctypes.byref(cg.c_struct), R, S, ws_ptr, counts.data_ptr(), scale.data_ptr(),
                                   _lib.ptr(pts), _lib.stream_ptr())
    _lib.check(rc, "nectb_train_rays")
    return counts, scale, pts


def forward_half(m, cg, batch, max_dist, ws):
    from nect_b200 import _lib
    from nect_b200.trainer import c_batch

    y = torch.empty(batch.num_rays, device="cuda")
    ptr, size = ws.get(m, cg, batch.num_rays, "cuda", batch.points_per_ray)
    cb = c_batch(batch, max_dist, "l2")
    rc = _lib.lib.nectb_train_forward(ctypes.byref(cg.c_struct), ctypes.byref(m.grid_desc), ctypes.byref(m.mlp_desc),
                                      m.grid_table.data_ptr(), m.mlp.data_ptr(), ctypes.byref(cb), y.data_ptr(), ptr,
                                      size, _lib.stream_ptr())
    _lib.check(rc, "nectb_train_forward")
    return y, cb, ptr, size


def backward_half(m, cg, cb, dy, ptr, size):
    from nect_b200 import _lib

    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    rc = _lib.lib.nectb_train_backward(ctypes.byref(cg.c_struct), ctypes.byref(m.grid_desc),
                                       ctypes.byref(m.mlp_desc), m.grid_table.data_ptr(), m.mlp.data_ptr(),
                                       ctypes.byref(cb), dy.data_ptr(), tg.data_ptr(), mg.data_ptr(), ptr, size,
                                       _lib.stream_ptr())
    _lib.check(rc, "nectb_train_backward")
    return tg, mg


# ---------------------------------------------------------------- sampling
@pytest.fixture(scope="module")
def ref_sampler(cuda_device):
    from oracle import ref_build

    try:
        return ref_build.load()
    except FileNotFoundError as e:
        pytest.skip(str(e))


@pytest.mark.parametrize("name,angle,chunk", [("c1_parallel", 2.3, 1 << 14), ("c2_cone", 0.8, 1 << 18),
                                              ("c5_large_4d", 4.1, 1 << 17)])
def test_fused_path_sampling_is_the_reference_sampler(ref_sampler, name, angle, chunk):
    from nect_b200.sampling import ct_sampling
    from nect_b200.trainer import RayBatch, Workspace

    w, geo, m, _ = build(name, "mixed")
    cg = geo.get_c_geometry()
    P = geo.nDetector[0] * geo.nDetector[1]
    R, S = w["rays"], w["S"]
    maxd = geo.max_distance_traveled / S
    torch.manual_seed(21)
    perm = torch.randperm(P, device="cuda")
    # the reference draws its jitter inside sample(); chunk k's draws are replayed from seed 500 + k
    jit, off = [], []
    for k, lo in enumerate(range(0, R, chunk)):
        torch.manual_seed(500 + k)
        j, o = ct_sampling.draw_ray_randoms(min(chunk, R - lo), 0.0, torch.device("cuda"))
        jit.append(j)
        off.append(o)
    jitter, det_off = torch.cat(jit), torch.cat(off)
    batch = RayBatch(perm=perm, start=0, num_rays=R, points_per_ray=S, angle=angle, max_ray_distance_per_point=maxd,
                     jitter=jitter, detector_offset=det_off, projection=torch.rand(P, device="cuda"), t=0.5)
    ws = Workspace(staging=False)
    forward_half(m, cg, batch, geo.max_distance_traveled, ws)
    counts, scale, pts = train_rays(cg, R, S, ws.buf.data_ptr())
    # the sampler entry point on the same draws
    _, sd, sc = ct_sampling.sample_with_draws(perm, cg, angle, S, R, 0, maxd, True, jitter, det_off, want_points=False,
                                              want_counts=True)
    assert torch.equal(counts, sc)
    maxdist = torch.tensor(geo.max_distance_traveled, dtype=torch.float32, device="cuda")
    assert torch.equal(scale, sd / maxdist)
    rgeom = ref_geometry(ref_sampler, cg)
    idx = torch.arange(S, device="cuda")
    for k, lo in enumerate(range(0, R, chunk)):
        n = min(chunk, R - lo)
        torch.manual_seed(500 + k)
        rp, rd = ref_sampler.sample(random_ray_index=perm, geometry=rgeom, angle_rad=angle, num_points_per_ray=S,
                                    num_rays=n, starting_ray_index=lo, max_ray_distance_per_point=maxd,
                                    uniform_ray_spacing=True, random_detector_offset=0.0, device=0)
        written = (rp != 0).any(-1)
        ref_counts = (torch.where(written, idx, -1).max(1).values + 1).to(torch.int32)
        assert torch.equal(counts[lo:lo + n], ref_counts), f"counts differ in rays {lo}..{lo + n}"
        assert torch.equal(sd[lo:lo + n].view(torch.int32), rd.view(torch.int32))
        assert torch.equal(pts[lo:lo + n], rp.clamp_(0.0, 1.0)), f"positions differ in rays {lo}..{lo + n}"
        del rp, rd, written
    assert int(counts.min()) >= 0 and int(counts.max()) <= S and int((counts > 0).sum()) > R // 4
    # the C oracle (host arithmetic, device trig values) on the counts
    n_or = min(R, 1 << 18)
    _, _, oc = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy(), 0, n_or, S, angle, maxd, True,
                                   jitter[:n_or].cpu().numpy(), det_off[:n_or].cpu().numpy(), trig=device_trig(angle),
                                   want_points=False)
    np.testing.assert_array_equal(counts[:n_or].cpu().numpy(), oc)
    del pts
    torch.cuda.empty_cache()


# ---------------------------------------------------------- training step
CASES = [("c2_cone", "mixed", 1, 2048, "ReLU"), ("c2_cone", "mixed", 0, 2048, "ReLU"),
         ("c2_cone", "plain_fp32", 1, 2048, "None"), ("c2_cone", "plain_fp32", 1, 2048, "ReLU"),
         ("c3_cone_4d", "mixed", 1, 2048, "ReLU"), ("c3_cone_4d", "plain_fp32", 1, 2048, "None"),
         ("c3_cone_4d", "plain_fp32", 1, 2048, "ReLU"), ("c5_large_4d", "mixed", 0, 1024, "ReLU"),
         ("c5_large_4d", "plain_fp32", 0, 1024, "None"), ("c5_large_4d", "plain_fp32", 0, 1024, "ReLU")]


@pytest.mark.parametrize("name,precision,store,n_check,act", CASES,
                         ids=[f"{c[0]}-{c[1]}-{'store' if c[2] else 'recompute'}-{c[4]}" for c in CASES])
def test_fullsize_step_matches_oracle(cuda_device, name, precision, store, n_check, act):
    from nect_b200.sampling import ct_sampling
    from nect_b200.trainer import RayBatch, Workspace, train_step

    torch.cuda.empty_cache()
    w, geo, m, enc = build(name, precision, act=act)
    cg = geo.get_c_geometry()
    P = geo.nDetector[0] * geo.nDetector[1]
    S = w["S"]
    # the plain path runs the large workload on a 65,536-ray batch (same table, detector and S)
    R = w["rays"] if not (precision == "plain_fp32" and name == "c5_large_4d") else 1 << 16
    maxd = geo.max_distance_traveled / S
    angle, t = 1.9, 0.37
    torch.manual_seed(7)
    perm = torch.randperm(P, device="cuda")
    jitter, det_off = ct_sampling.draw_ray_randoms(R, 0.0, torch.device("cuda"))
    proj = torch.rand(P, device="cuda")
    batch = RayBatch(perm=perm, start=0, num_rays=R, points_per_ray=S, angle=angle, max_ray_distance_per_point=maxd,
                     jitter=jitter, detector_offset=det_off, projection=proj, t=t)
    gen = torch.Generator(device="cpu").manual_seed(11)
    sub = torch.randperm(R, generator=gen)[:n_check].sort().values
    dy = torch.zeros(R)
    dy[sub] = torch.randn(n_check, generator=gen) / n_check
    with tuning(encoding_store=store):
        ws = Workspace()
        y, cb, ptr, size = forward_half(m, cg, batch, geo.max_distance_traveled, ws)
        tg, mg = backward_half(m, cg, cb, dy.cuda(), ptr, size)
        torch.cuda.synchronize()
        assert ws.error_word(cg) == 0
        # the fused step on the same batch, built-in L2 loss
        tg2, mg2 = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
        loss, y2 = train_step(m, cg, batch, geo.max_distance_traveled, tg2, mg2, ws, "l2")
        torch.cuda.synchronize()
        assert ws.error_word(cg) == 0
        # the backward half with the L2 loss's dL/dy_pred on the fused step's workspace
        tg3, mg3 = backward_half(m, cg, cb, (2 * (y - proj[perm[:R]]) / R).contiguous(), ptr, size)
        torch.cuda.synchronize()
    assert torch.equal(y2, y)
    meas = proj[perm[:R]].double()
    lref = float(((y.double() - meas) ** 2).mean())
    assert abs(float(loss) - lref) <= 1e-5 * lref
    tol_split = 1e-3 if precision == "mixed" else 1e-4
    assert rel_max(tg2, tg3) < tol_split and rel_max(mg2, mg3) < tol_split, (rel_max(tg2, tg3), rel_max(mg2, mg3))
    del tg2, mg2, tg3, mg3, ws
    torch.cuda.empty_cache()

    # fp64 oracle on the subset: positions from the C oracle with the device's trig values
    sub_np = sub.numpy()
    pts, dist, counts = osamp.oracle_sample(osamp.to_struct(cg), perm.cpu().numpy()[sub_np], 0, n_check, S, angle,
                                            maxd, True, jitter.cpu().numpy()[sub_np],
                                            det_off.cpu().numpy()[sub_np], trig=device_trig(angle))
    levels, _ = ohg.layout(w["n_dims"], 16, enc.log2_hashmap_size, float(enc.base_resolution),
                           float(enc.per_level_scale), float(enc.base_resolution_t or enc.base_resolution))
    n_in = 16 * w["F"]
    tab = m.grid_table.detach().cpu().double().requires_grad_(True)
    wf = m.mlp.detach().cpu().double().requires_grad_(True)
    yo = ohg.line_integrals(pts, dist, tab, wf, levels, enc.log2_hashmap_size, n_in, 64, w["H"],
                            geo.max_distance_traveled, act=act.lower(), t=t if w["n_dims"] == 4 else None)
    (yo * dy[sub].double()).sum().backward()
    ys = y[sub.cuda()].cpu().double()
    assert int((torch.from_numpy(counts) > 0).sum()) > n_check // 4
    if precision == "mixed":
        assert rel_max(ys, yo.detach()) < 2e-2, rel_max(ys, yo.detach())
        gt, gm = tg.cpu().double(), mg.cpu().double()
        assert cosine(gt, tab.grad) > 0.99 and cosine(gm, wf.grad) > 0.99, (cosine(gt, tab.grad), cosine(gm, wf.grad))
        assert rel_max(gt, tab.grad) < 5e-2 and rel_max(gm, wf.grad) < 5e-2, (rel_max(gt, tab.grad),
                                                                             rel_max(gm, wf.grad))
    else:
        assert rel_max(ys, yo.detach()) < 1e-4, rel_max(ys, yo.detach())
        gt, gm = tg.cpu().double(), mg.cpu().double()
        tol_max, tol_l2 = (1e-4, 5e-5) if act == "None" else (1e-2, 3e-3)
        for a, b in ((gt, tab.grad), (gm, wf.grad)):
            assert rel_max(a, b) < tol_max and rel_l2(a, b) < tol_l2, (rel_max(a, b), rel_l2(a, b))
