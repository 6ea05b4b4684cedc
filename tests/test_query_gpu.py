"""GPU parity of the query paths (C ABI: nectb_query_points,
nectb_query_reproject) against the oracle, and of the continuous-batching
server: every result served in a concurrent mix equals the same request
served alone (bit for bit).

Tolerances vs the fp64 oracle: plain fp32 model 1e-5 relative to the largest
value; mixed model (bf16 tensor-core MLP) 2e-2.
"""

import ctypes

import numpy as np
import pytest
import torch

from nect_b200 import _lib

from oracle import hashgrid as ohg
from oracle import sampling as osamp

pytestmark = pytest.mark.gpu

TOL = {"plain_fp32": 1e-5, "mixed": 2e-2}


def model_and_geometry(precision, n_dims=4):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D
    from nect_b200.sampling import Geometry

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=13, base_resolution=4,
                            finest_resolution=160, base_resolution_t=2 if n_dims == 4 else None)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=64, activation="ReLU", output_activation="Softplus")
    m = (HashGrid4D if n_dims == 4 else HashGrid)(enc, net, precision=precision, device="cuda")
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(7)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.4)
        m.refresh_half()
    geo = Geometry(nDetector=[48, 40], dDetector=[1.2, 1.2], mode="cone", DSD=250.0, DSO=160.0, nVoxel=[32] * 3,
                   dVoxel=[1.0] * 3)
    levels, _ = ohg.layout(n_dims, 16, 13, 4.0, float(enc.per_level_scale), float(enc.base_resolution_t or 4))
    return m, geo, levels


def oracle_sigma(m, levels, pts, t=None):
    x = torch.as_tensor(pts, dtype=torch.float32)
    if t is not None:
        x = torch.cat([x, torch.full((x.shape[0], 1), float(t))], 1)
    Ws = ohg.split_mlp_params(m.mlp.detach().cpu().double(), 32, 64, 2)
    return ohg.mlp(ohg.encode(x, m.grid_table.detach().cpu().double(), levels, 13), Ws).squeeze(-1)


def rel(a, b):
    a, b = torch.as_tensor(a).double().flatten(), torch.as_tensor(b).double().flatten()
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_volume_and_slices_match_oracle(cuda_device, precision):
    from nect_b200 import serving

    m, geo, levels = model_and_geometry(precision)
    t = 0.3
    vol = torch.empty(12, 16, 20, device="cuda")
    sl = torch.empty(33, 47, device="cuda")
    ob = torch.empty(40, 40, device="cuda")
    it_sl = serving.slice_items(sl, sl.shape, t, centre=(0.4, 0.5, 0.6))
    it_ob = serving.slice_items(ob, ob.shape, t, centre=(0.5, 0.5, 0.5), u=(0.2, 0.7, 0.3), v=(0.0, -0.3, 0.9),
                                rows_per_item=7)
    serving.query_points(m, np.concatenate([serving.volume_items(vol, vol.shape, t), it_sl, it_ob]))
    torch.cuda.synchronize()
    z, y, x = [serving.centres(n) for n in (12, 16, 20)]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    ref = oracle_sigma(m, levels, np.stack([Z, Y, X], -1).reshape(-1, 3), t)
    assert rel(vol.cpu(), ref) < TOL[precision]
    for out, items in ((sl, it_sl), (ob, it_ob)):
        pts = []
        for it in items:
            o, du, dv = it["origin"], it["du"], it["dv"]
            for j in range(int(it["nv"])):
                for i in range(int(it["nu"])):
                    pts.append(np.clip(o + np.float32(i) * du + np.float32(j) * dv, 0, 1))
        assert rel(out.cpu(), oracle_sigma(m, levels, np.array(pts, np.float32), t)) < TOL[precision]


def test_slice_queries_match_4d_queries_and_oracle(cuda_device):
    """Volume and slice items of a 4D mixed model evaluated on its time slice
    at t (nectb_time_slice + nectb_query_points_slice, 8 corners per level)
    agree with the 16-corner 4D queries within 1e-2 and with the oracle within
    the mixed tolerance; slices at two t differ where the model does."""
    from nect_b200 import serving

    m, geo, levels = model_and_geometry("mixed")
    for t in (0.0, 0.3, 0.77, 1.0):
        vol4, vols = torch.empty(12, 16, 20, device="cuda"), torch.empty(12, 16, 20, device="cuda")
        sl4, sls = torch.empty(33, 47, device="cuda"), torch.empty(33, 47, device="cuda")
        serving.query_points(m, np.concatenate([serving.volume_items(vol4, vol4.shape, t),
                                                serving.slice_items(sl4, sl4.shape, t, centre=(0.4, 0.5, 0.6))]))
        slc = serving.time_slice(m, t)
        serving.query_points(m, np.concatenate([serving.volume_items(vols, vols.shape, 0.123),   # t ignored
                                                serving.slice_items(sls, sls.shape, t, centre=(0.4, 0.5, 0.6))]),
                             slice=slc)
        torch.cuda.synchronize()
        assert rel(vols.cpu(), vol4.cpu()) < 1e-2, t
        assert rel(sls.cpu(), sl4.cpu()) < 1e-2, t
        z, y, x = [serving.centres(n) for n in (12, 16, 20)]
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        ref = oracle_sigma(m, levels, np.stack([Z, Y, X], -1).reshape(-1, 3), t)
        assert rel(vols.cpu(), ref) < TOL["mixed"], t


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_reprojection_matches_oracle(cuda_device, precision):
    from nect_b200 import serving

    m, geo, levels = model_and_geometry(precision)
    angle, t, S = 0.8, 0.6, 64
    view = serving.reproject(m, geo, angle, t, S)
    torch.cuda.synchronize()
    assert rel(view.cpu(), oracle_view(m, geo, levels, angle, t, S)) < TOL[precision]


def oracle_view(m, geo, levels, angle, t, S):
    """The re-projection from the oracle's sampler and fp64 model."""
    cg = geo.get_c_geometry()
    P = geo.nDetector[0] * geo.nDetector[1]
    a = torch.tensor([angle, 0.0], dtype=torch.float32, device="cuda")
    c, s = torch.cos(a).cpu().numpy(), torch.sin(a).cpu().numpy()
    trig = np.array([c[0], s[0], c[1], c[1], c[1], s[1], s[1], s[1]], np.float32)
    maxd = geo.max_distance_traveled / S
    pts, dist, counts = osamp.oracle_sample(osamp.to_struct(cg), np.arange(P), 0, P, S, angle, maxd, True,
                                            np.zeros(P, np.float32), np.zeros((P, 2), np.float32), trig=trig)
    keep = ~np.all(np.clip(pts, 0, 1).reshape(-1, 3) == 0, axis=1)
    sig = np.zeros(P * S)
    sig[keep] = oracle_sigma(m, levels, np.clip(pts, 0, 1).reshape(-1, 3)[keep], t).numpy()
    return sig.reshape(P, S).sum(1) * dist / geo.max_distance_traveled


@pytest.mark.parametrize("precision,n_dims", [("plain_fp32", 4), ("mixed", 3), ("mixed", 4)])
def test_reprojection_pieces_match_the_whole_view(cuda_device, precision, n_dims):
    """A view computed in pieces (nectb_query_reproject_range, 1, 3 and 4
    warpgroups per SM) equals the whole view bit for bit where both gather the
    same table.  With room for a time slice a 4D mixed model gathers 8 corners
    on the slice at t: that view agrees with the 16-corner one within 1e-2 and
    with the oracle within the mixed tolerance."""
    from nect_b200 import serving

    m, geo, levels = model_and_geometry(precision, n_dims)
    angle, t, S = 0.8, 0.6, 64
    whole = serving.reproject(m, geo, angle, t, S).flatten().clone()
    P = whole.numel()
    piece = 500
    sliced = n_dims == 4 and precision == "mixed"
    cg = geo.get_c_geometry()
    base = _lib.lib.nectb_train_workspace_bytes(ctypes.byref(cg.c_struct), None, None, piece)
    for wg in (1, 3, 4):
        for room in ((False, True) if sliced else (False,)):
            nbytes = serving.reproject_workspace_bytes(m, geo, piece) if room else base
            ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            out = torch.full((P,), float("nan"), device="cuda")
            for b in range(0, P, piece):
                serving.reproject(m, geo, angle, t, S, out=out, workspace=ws, pixels=(b, min(piece, P - b)),
                                  warpgroups=wg)
            torch.cuda.synchronize()
            assert not torch.isnan(out).any()
            if room:
                assert rel(out.cpu(), whole.cpu()) < 1e-2
            else:
                assert torch.equal(out, whole), (wg, room)
    if sliced:
        one = serving.reproject(m, geo, angle, t, S, warpgroups=3).flatten()   # one piece, slice room included
        torch.cuda.synchronize()
        assert rel(one.cpu(), whole.cpu()) < 1e-2
        assert rel(one.cpu(), oracle_view(m, geo, levels, angle, t, S)) < TOL[precision]


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_server_results_same_alone_and_in_mix(cuda_device, precision):
    from nect_b200.serving import QueryServer, Request

    m, geo, _ = model_and_geometry(precision)
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(24):
        kind = ["slice", "slice", "reproject", "volume"][k % 4]
        reqs.append(dict(kind=kind, t=float(rng.random()), size=int(rng.choice([40, 64, 96])) if kind != "volume"
                         else 24, angle=float(rng.random() * 6.28),
                         centre=tuple(rng.random(3) * 0.4 + 0.3), u=(0.0, 0.0, 1.0), v=(0.0, 1.0, 0.0)))
    srv = QueryServer(m, geo, memory_budget=256 << 20, points_per_ray=64, piece_pixels=700)   # 3 pieces a view
    alone = []
    for d in reqs:  # one at a time
        r = srv.submit(Request(**d))
        r.event.wait(60)
        alone.append(r.result.copy())
    mixed = [srv.submit(Request(**d)) for d in reqs]  # all at once
    for r in mixed:
        assert r.event.wait(60)
    srv.close()
    for a, r in zip(alone, mixed):
        assert np.array_equal(a, r.result), f"{r.kind} differs between alone and mixed"
    stats = srv.latency_stats()
    assert set(stats) == {"slice", "reproject", "volume"}
