"""fit()'s checkpoints and resume (CPU, with the fused step replaced by a stub
that counts steps and moves the table): a run stopped after 12 steps and
resumed from its checkpoint takes the projections an uninterrupted 20-step
run takes at steps 13-20, with the model, Adam step count and position
restored (base_trainer.py:189-212, 297-299); the metrics log, cancel_at and
KeyboardInterrupt handling, several batches per projection, and the batches
Trainer.make_batch cuts from a projection."""
import numpy as np
import pytest
import torch


def run(tmp_path, monkeypatch, niter, **kw):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig
    from nect_b200.reconstruct import fit
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    seen = []

    def fake_step(self, batch):
        self.step_count += 1
        seen.append((self.step_count, round(batch.angle, 6)))
        with torch.no_grad():
            self.model.table.add_(1.0)
        return torch.zeros(1)

    monkeypatch.setattr(Trainer, "step", fake_step)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    geo = Geometry(nDetector=[16, 16], dDetector=[1 / 16] * 2, mode="parallel", nVoxel=[16] * 3, dVoxel=[1 / 16] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=10, base_resolution=4,
                            finest_resolution=32)
    cfg = ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "plain_fp32")
    angles = np.linspace(0, np.pi, 7, endpoint=False)
    projs = torch.rand(7, 16, 16, generator=torch.Generator().manual_seed(0))
    rec = fit(geo, projs, angles, model_cfg=cfg, niter=niter, points_per_ray=8, rays_per_batch=32, seed=5,
              device="cpu", **kw)
    return rec, seen


def test_resumed_fit_continues_the_uninterrupted_run(tmp_path, monkeypatch):
    from nect_b200 import checkpoint

    full, seen_full = run(tmp_path, monkeypatch, 20)
    part, seen_part = run(tmp_path, monkeypatch, 12, checkpoint_dir=tmp_path / "a", checkpoint_interval=1e9)
    ckpt = tmp_path / "a" / "model" / "checkpoints" / "last.ckpt"
    data = torch.load(ckpt, map_location="cpu", weights_only=False)
    assert (data["epoch"], data["angle"]) == (1, 5)          # 12 steps of 7 projections
    prev = torch.load(tmp_path / "a" / "model" / "checkpoints" / "2nd_last.ckpt", map_location="cpu",
                      weights_only=False)
    assert (prev["epoch"], prev["angle"]) == (0, 0)           # the one saved at the start
    assert (tmp_path / "a" / "model" / "geometry.yaml").exists()
    assert seen_part == seen_full[:12]

    resumed, seen_res = run(tmp_path, monkeypatch, 20, resume_from=ckpt, checkpoint_dir=tmp_path / "b")
    assert seen_res == seen_full[12:]                          # steps 13..20, same projections
    assert resumed.trainer.step_count == 20
    assert torch.equal(resumed.model.table, full.model.table)
    data = torch.load(tmp_path / "b" / "model" / "checkpoints" / "last.ckpt", map_location="cpu",
                      weights_only=False)
    assert (data["epoch"], data["angle"]) == (2, 6)
    assert checkpoint.resume(tmp_path / "b" / "model" / "checkpoints" / "last.ckpt", resumed.model) == \
        {"epoch": 2, "angle": 6}


def test_fit_logs_the_reference_keys(tmp_path, monkeypatch):
    logged = []
    run(tmp_path, monkeypatch, 9, log_fn=lambda step, m: logged.append((step, m)))
    assert [s for s, _ in logged] == list(range(1, 10))
    keys = {"loss", "max_mem", "current_mem", "epoch", "downsample_detector_factor", "points_per_ray",
            "distance_between_points", "lr", "num_proj_processed", "rays"}
    assert all(set(m) == keys for _, m in logged)
    step, m = logged[-1]
    assert (m["epoch"], m["num_proj_processed"], m["points_per_ray"], m["downsample_detector_factor"]) == (1, 8, 8, 1)



def test_cancel_at_stops_and_saves(tmp_path, monkeypatch):
    import datetime

    import pytest

    rec, seen = run(tmp_path, monkeypatch, 20, checkpoint_dir=tmp_path / "c", cancel_at="2000-01-01T00:00:00")
    assert rec.stopped == "cancelled" and len(seen) == 1 and rec.trainer.step_count == 1
    data = torch.load(tmp_path / "c" / "model" / "checkpoints" / "last.ckpt", map_location="cpu", weights_only=False)
    assert (data["epoch"], data["angle"]) == (0, 1)
    later = datetime.datetime.now(datetime.timezone.utc) + datetime.timedelta(days=1)
    rec, seen = run(tmp_path, monkeypatch, 5, cancel_at=later)
    assert rec.stopped is None and len(seen) == 5
    with pytest.raises(ValueError, match="ISO"):
        run(tmp_path, monkeypatch, 5, cancel_at="tomorrow")


def test_keyboard_interrupt_ends_training_without_a_save_before_3000_steps(tmp_path, monkeypatch):
    from nect_b200.trainer import Trainer

    rec, seen = run(tmp_path, monkeypatch, 3)          # installs the stub
    stub = Trainer.step

    def interrupting(self, batch):
        if self.step_count == 4:
            raise KeyboardInterrupt
        return stub(self, batch)

    monkeypatch.setattr(Trainer, "step", interrupting)
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig
    from nect_b200.reconstruct import fit
    from nect_b200.sampling import Geometry

    geo = Geometry(nDetector=[16, 16], dDetector=[1 / 16] * 2, mode="parallel", nVoxel=[16] * 3, dVoxel=[1 / 16] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=10, base_resolution=4,
                            finest_resolution=32)
    cfg = ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "plain_fp32")
    rec = fit(geo, torch.rand(7, 16, 16), np.linspace(0, np.pi, 7, endpoint=False), model_cfg=cfg, niter=20,
              points_per_ray=8, rays_per_batch=32, device="cpu", checkpoint_dir=tmp_path / "k")
    assert rec.stopped == "interrupted" and rec.trainer.step_count == 4
    data = torch.load(tmp_path / "k" / "model" / "checkpoints" / "last.ckpt", map_location="cpu", weights_only=False)
    assert (data["epoch"], data["angle"]) == (0, 0)     # only the checkpoint written at the start


def test_batches_per_projection(tmp_path, monkeypatch):
    rec, seen = run(tmp_path, monkeypatch, 5, batch_per_proj=3)
    assert len(seen) == 15 and rec.trainer.step_count == 15
    angles = [a for _, a in seen]
    assert all(angles[3 * i] == angles[3 * i + 1] == angles[3 * i + 2] for i in range(5))
    rec, seen = run(tmp_path, monkeypatch, 2, batch_per_proj="all")   # 256 pixels / 32 rays
    assert len(seen) == 16


@pytest.mark.parametrize("P,bs,expect", [
    (1024, 64, [(0, 64), (64, 64), (960, 64), None]),   # batches 0, 1, 15, 16
    (40, 64, [(0, 40), None, None, None]),               # partial first batch (projector.py:108-112)
    (128, 64, [(0, 64), (64, 64), None, None]),
])
def test_make_batch_follows_the_projector(P, bs, expect):
    """Batches of a projection: full batches of batch_size rays from the
    permutation, the partial first batch when the detector holds fewer, and
    None past the end; jitter in [-0.5, 0.5) and detector offsets scaled by
    random_offset_detector (ct_sampling.cu:619-622)."""
    from nect_b200.trainer import Trainer

    tr = Trainer.__new__(Trainer)
    tr.points_per_batch, tr.points_per_ray, tr.random_offset_detector = bs * 8, 8, 0.5
    tr.device, tr.uniform_ray_spacing = torch.device("cpu"), True

    class Geo:
        max_distance_traveled = 4.0

    tr.geometry = Geo()
    perm = torch.randperm(P)
    got = []
    for batch_num in (0, 1, 15, 16):
        b = tr.make_batch(perm, batch_num, 0.3, torch.zeros(P), t=0.2)
        got.append(None if b is None else (b.start, b.num_rays))
        if b is not None:
            assert b.jitter.shape == (b.num_rays,) and bool((b.jitter.abs() <= 0.5).all())
            assert b.detector_offset.shape == (b.num_rays, 2) and bool((b.detector_offset.abs() <= 0.25).all())
            assert b.max_ray_distance_per_point == 0.5 and (b.angle, b.t) == (0.3, 0.2)
    assert got == expect
