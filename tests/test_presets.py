"""The reference's quality presets as reconstruct() resolves them (CPU):
the configuration fields of each preset (nect/reconstruct.py:173-208 over
nect/cfg/default.yaml and the mode's model preset), the learning-rate rule
(nect/config.py:398-399) and the schedule and model they give."""
import math

import pytest


def geometry(n=256):
    from nect_b200.sampling import Geometry

    return Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3,
                    dVoxel=[1 / n] * 3)


# (quality, loss, log2 entries, epochs, base lr, warm-up steps, lrf, points_per_ray end), static mode
STATIC = [
    ("poor", "l2", 19, "0.02x", 1e-2, 500, "auto", "auto"),
    ("low", "l2", 19, "0.1x", 5e-3, 500, "auto", "auto"),
    ("medium", "l1", 21, "0.3x", 2e-3, 500, "auto", "auto"),
    ("high", "l1", 21, "1x", 5e-4, 500, "auto", "auto"),
    ("higher", "l1", 21, "2x", 5e-4, 3000, 0.05, "1.5x"),
    ("highest", "l1", 23, "4x", 2e-4, 5000, 0.01, "1.5x"),
]


@pytest.mark.parametrize("quality,loss,log2,epochs,base_lr,warmup,lrf,pend", STATIC)
def test_static_presets(quality, loss, log2, epochs, base_lr, warmup, lrf, pend):
    from nect_b200.reconstruct import preset_config

    cfg = preset_config("static", quality)
    assert (cfg["loss"], cfg["log2_hashmap_size"], cfg["epochs"], cfg["warmup_steps"], cfg["lrf"],
            cfg["points_end"]) == (loss, log2, epochs, warmup, lrf, pend)
    assert cfg["base_lr"] == pytest.approx(base_lr, rel=1e-12)
    assert cfg["warmup_lr0"] == 1e-3


def test_dynamic_defaults_and_overrides():
    from nect_b200.reconstruct import preset_config

    cfg = preset_config("dynamic", "medium")
    assert cfg["base_lr"] == pytest.approx(4e-4) and cfg["warmup_steps"] == 2000 and cfg["warmup_lr0"] == 1e-4
    assert cfg["log2_hashmap_size"] == 23 and cfg["loss"] == "l1"
    cfg = preset_config("static", "poor", niter=7, lr=3e-3)   # niter replaces epochs, lr the base lr
    assert cfg["epochs"] == 7 and cfg["base_lr"] == 3e-3
    with pytest.raises(ValueError, match="quality"):
        preset_config("static", "best")
    with pytest.raises(ValueError, match="mode"):
        preset_config("4d", "high")


def test_learning_rate_rule():
    from nect_b200.reconstruct import learning_rate

    assert learning_rate(1e-3, 1_000_000) == pytest.approx(1e-3)
    assert learning_rate(5e-4, 5_000_000, n_gpus=4) == pytest.approx(5e-4 * math.sqrt(20))


def test_plan_for_high_quality():
    from nect_b200.reconstruct import AUTO_POINTS_PER_BATCH, plan_reconstruction

    geo = geometry(256)
    plan = plan_reconstruction(geo, "static", 100, "high", precision="plain_fp32")
    sch = plan.schedule
    assert sch.epochs == math.ceil(49 / 100 * 256)              # epochs "1x" of the base epochs
    assert sch.total_projections == sch.epochs * 100
    assert sch.lr[0] == pytest.approx(5e-4 * math.sqrt(AUTO_POINTS_PER_BATCH / 1e6))
    assert sch.warmup[:2] == (500, 1e-3)
    assert sch.pts[1] == math.ceil(1.5 * 256)                      # points_per_ray end "auto"
    assert plan.points_per_batch == AUTO_POINTS_PER_BATCH // 2    # the trainer samples half (base_trainer.py:143)
    assert plan.loss == "l1"
    enc = plan.model_cfg.encoder
    assert enc.log2_hashmap_size == 21 and plan.model_cfg.precision == "plain_fp32"
    first = next(iter(sch.steps()))
    assert first.points_per_ray == 100 and first.detector_binning == 2


def test_plan_with_niter_and_points_per_batch():
    from nect_b200.reconstruct import plan_reconstruction

    plan = plan_reconstruction(geometry(64), "dynamic", 30, "poor", niter=3, points_per_batch=1_000_000)
    assert plan.schedule.total_projections == 90 and plan.points_per_batch == 500_000
    assert plan.schedule.lr[0] == pytest.approx(2e-3)
    assert plan.model_cfg.model == "quadcubes" and plan.model_cfg.encoder.log2_hashmap_size == 19


def test_reconstruct_resolves_the_preset_and_turns_the_static_volume(monkeypatch):
    """reconstruct() with fit() stubbed (fit itself runs on the GPU): the preset
    reaches fit, and the static volume comes back turned by 180 degrees in
    (y, x), as nect/reconstruct.py:246-247 returns create_volume."""
    import numpy as np
    import torch

    from nect_b200 import reconstruct as rc

    seen = {}
    vol = torch.arange(2 * 3 * 4, dtype=torch.float32).reshape(2, 3, 4)

    class Rec:
        def volume(self):
            return vol

    def fake_fit(geometry, projections, angles, timesteps=None, **kw):
        seen.update(kw, angles=angles, timesteps=timesteps)
        return Rec()

    monkeypatch.setattr(rc, "fit", fake_fit)
    geo = geometry(32)
    out = rc.reconstruct(geo, np.zeros((10, 32, 32), np.float32), angles=np.arange(10) * 18.0, radians=False,
                         quality="medium", lr=1e-3, verbose=False, flip_projections=True, channel_order="NHW")
    assert np.array_equal(out, vol.flip(1).flip(2).numpy())
    assert seen["loss"] == "l1" and seen["points_per_batch"] == 2_500_000
    assert seen["niter"] == seen["schedule"].total_projections == math.ceil(0.3 * math.ceil(49 / 10 * 32)) * 10
    assert seen["lr"] == pytest.approx(1e-3 * math.sqrt(5))
    assert np.allclose(seen["angles"], np.deg2rad(np.arange(10) * 18.0)) and seen["timesteps"] is None
    assert seen["s3im"] is False and seen["add_poisson"] is False

    seen.clear()
    rc.reconstruct(geo, np.zeros((10, 32, 32), np.float32), angles=np.arange(10) * 0.3, quality="high",
                   verbose=False, config_override={"epochs": 2, "s3im": True, "points_per_batch": 400_000,
                                                   "warmup": {"steps": 7}})
    assert seen["niter"] == 20 and seen["s3im"] is True and seen["points_per_batch"] == 200_000
    assert seen["schedule"].warmup[0] == 7
    assert seen["betas"] == (0.9, 0.999) and seen["weight_decay"] == 0.0
    seen.clear()
    rc.reconstruct(geo, np.zeros((10, 32, 32), np.float32), angles=np.arange(10) * 0.3, verbose=False,
                   config_override={"optimizer": {"otype": "Adam", "beta1": 0.8, "weight_decay": 0.01}})
    assert seen["betas"] == (0.8, 0.999) and seen["weight_decay"] == 0.01
    with pytest.raises(ValueError, match="array"):
        rc.reconstruct(geo, "projections.npy", angles=np.arange(10) * 0.3, verbose=False)


def test_config_override_mapping():
    from nect_b200.reconstruct import preset_config

    cfg = preset_config("static", "high", niter=5, lr=1e-2, config_override={
        "epochs": 9, "base_lr": 3e-3, "loss": "L2", "lr_scheduler": {"otype": "exponential", "lrf": 0.1},
        "points_per_ray": {"start": 64, "end": 512, "linear": False}, "encoder": {"log2_hashmap_size": 18},
        "downsampling_detector": {"start": 4, "update_interval": 50}})
    assert cfg["epochs"] == 9 and cfg["base_lr"] == 3e-3 and cfg["loss"] == "l2"   # the override comes last
    assert (cfg["lr_otype"], cfg["lrf"]) == ("exponential", 0.1)
    assert (cfg["points_start"], cfg["points_end"], cfg["points_linear"]) == (64, 512, False)
    assert cfg["log2_hashmap_size"] == 18 and (cfg["downsampling_start"], cfg["downsampling_update_interval"]) == (4, 50)
    for bad in ({"optimizer": {"otype": "Lion"}}, {"model": "kplanes"}):
        with pytest.raises(ValueError, match="not supported"):
            preset_config("static", "high", config_override=bad)
