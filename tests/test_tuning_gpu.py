"""Launch shapes and scheduling do not change results: gradients of the mixed
step under extreme tunings (one block per SM everywhere, 16 rounds, 1 MiB
level groups, no run merging / merging every level) against the defaults
within 1e-5 of the largest entry (fp32 reassociation); and the autotuner on a
small workload restores the model and returns a valid tuning."""
import json

import pytest
import torch

pytestmark = pytest.mark.gpu


def setup(n_dims=4):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid, HashGrid4D
    from nect_b200.sampling import Geometry

    torch.manual_seed(3)
    geo = Geometry(nDetector=[40, 48], dDetector=[1.5, 1.5], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[32] * 3,
                   dVoxel=[1.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=12, base_resolution=4,
                            finest_resolution=128, base_resolution_t=2 if n_dims == 4 else None)
    m = (HashGrid if n_dims == 3 else HashGrid4D)(enc, MLPNetConfig(n_hidden_layers=2), precision="mixed",
                                                  device="cuda", seed=0)
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(1)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.5)
        m.refresh_half()
    return geo, m


def grads(geo, m, seed=5):
    from nect_b200.trainer import RayBatch, Workspace, train_step

    P = 40 * 48
    gen = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(P, device="cuda", generator=gen)
    batch = RayBatch(perm=perm, start=0, num_rays=1200, points_per_ray=64, angle=0.5,
                     max_ray_distance_per_point=geo.max_distance_traveled / 64,
                     jitter=torch.rand(1200, device="cuda", generator=gen) - 0.5,
                     detector_offset=torch.zeros(1200, 2, device="cuda"),
                     projection=torch.rand(P, device="cuda", generator=gen), t=0.4)
    tg, mg = torch.zeros_like(m.table), torch.zeros_like(m.mlp)
    train_step(m, geo.get_c_geometry(), batch, geo.max_distance_traveled, tg, mg, Workspace(), "l2")
    torch.cuda.synchronize()
    return tg, mg


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


@pytest.mark.parametrize("n_dims", [3, 4])
def test_tunings_give_the_same_gradients(cuda_device, n_dims):
    from nect_b200 import autotune

    geo, m = setup(n_dims)
    default = autotune.get_tuning()
    try:
        tg0, mg0 = grads(geo, m)
        for t in ({"forward_blocks_per_sm": 1, "backward_blocks_per_sm": 1, "scatter_blocks_per_sm": 1},
                  {"staged_rounds": 16, "scatter_group_bytes": 1 << 20},
                  {"run_threshold_3d": 0.0, "run_threshold_4d": 0.0},
                  {"run_threshold_3d": 64.0, "run_threshold_4d": 64.0}):
            autotune.set_tuning(dict(default, **t))
            tg, mg = grads(geo, m)
            assert rel_max(tg, tg0) < 1e-5 and rel_max(mg, mg0) < 1e-5, (t, rel_max(tg, tg0), rel_max(mg, mg0))
    finally:
        autotune.set_tuning(default)


def test_autotuner_restores_state_and_caches(cuda_device, tmp_path):
    from nect_b200 import autotune
    from nect_b200.trainer import Trainer

    geo, m = setup(4)
    default = autotune.get_tuning()
    tr = Trainer(m, geo, points_per_batch=1200 * 64, points_per_ray=64, device="cuda")
    P = 40 * 48
    proj = torch.rand(P, device="cuda")

    def make_batch(k):
        return tr.make_batch(torch.randperm(P, device="cuda"), 0, 0.1 * k, proj, 0.5)

    table0 = m.table.detach().clone()
    try:
        cache = tmp_path / "tuning.json"
        best = autotune.tune(tr, make_batch, steps=2, warmup=1,
                             space={"forward_blocks_per_sm": (2, 4), "staged_rounds": (4, 8)}, cache=cache)
        assert set(best) == set(autotune.FIELDS)
        assert torch.equal(m.table, table0) and tr.step_count == 0
        stored = json.loads(cache.read_text())
        assert len(stored) == 1 and list(stored.values())[0]["tuning"] == best
        autotune.set_tuning(default)
        assert autotune.tune(tr, make_batch, cache=cache) == best   # served from the cache
    finally:
        autotune.set_tuning(default)
