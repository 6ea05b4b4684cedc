"""User entry point: reconstruct a volume from projections on the fused kernels.

Mirrors ``nect.reconstruct`` (nect/reconstruct.py:113-131) for the hot path
this package replaces: a hash-grid model is trained on the projections with
the fused sample -> encode -> MLP -> line integral -> loss -> backward step
(nectb_train_step) and the fused Adam update, then exported on a regular grid
with create_volume's de-normalisation (nect/trainers/base_trainer.py:402-450).

Scheduling follows BaseTrainer.fit (base_trainer.py:492-655) with one batch
per projection visit: each step takes the next projection of a seeded random
order, a device randperm of its pixels and one batch of rays.  ``fit`` takes
the reference's per-projection schedules (detector binning, points-per-ray
ramp, lr warm-up and decay: schedule.Schedule), its S3IM, Poisson and TV
terms; ``reconstruct`` resolves the reference's quality presets into them.
"""
from __future__ import annotations

import datetime
import math
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from .config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
from .network import _HashGridModel
from .sampling import Geometry
from .schedule import Schedule, bin_projection, s3im_patch_size
from .serving import denormalisation, query_points, volume_items
from .quadcubes import ModuleTrainer, QuadCubes
from .trainer import Trainer


@dataclass
class Reconstruction:
    """A trained model with the dataset scaling needed to export volumes."""
    model: _HashGridModel
    geometry: Geometry
    minimum: float
    maximum: float
    trainer: Trainer
    history: list = field(default_factory=list)   # (step, seconds of training, metrics dict)
    stopped: str | None = None                    # "cancelled" (cancel_at) or "interrupted" (KeyboardInterrupt)

    def volume(self, t: float = 0.0, shape: tuple | None = None) -> torch.Tensor:
        """Attenuation on the voxel-centre grid [z, y, x] (create_volume)."""
        shape = tuple(shape or self.geometry.nVoxel)
        scale, offset = denormalisation(self.geometry.max_distance_traveled, self.minimum, self.maximum)
        if isinstance(self.model, QuadCubes):
            return self.model.volume(shape, t, scale, offset)
        out = torch.empty(shape, device=self.model.table.device)
        query_points(self.model, volume_items(out, shape, t, scale, offset))
        return out


def default_model_config(geometry: Geometry, mode: str, precision: str, log2_hashmap_size: int = 21) -> ModelConfig:
    """The reference's default model of the mode.  Static: its hash_grid
    preset (nect/cfg/static/hash_grid.yaml:1-13): 19 levels x 4 features,
    2^21 entries (unless the quality preset sets another size), base
    resolution 8, finest 2 x the largest detector extent, 6 x 64 LeakyReLU
    MLP with a ReLU output.  Dynamic: its quadcubes preset
    (nect/cfg/dynamic/quadcubes.yaml:1-16): four 3D grids of 23 levels x 4
    features, 2^23 entries (or the preset's size), base resolution 16,
    finest 2 x the largest detector extent, the raw inputs appended, 4 x 128
    LeakyReLU MLP without an output activation.  The fused single-4D-grid
    model ("hash_grid_4d") is the fast dynamic model (fused_dynamic_config)."""
    if mode == "dynamic":
        enc = HashEncoderConfig(n_levels=23, n_features_per_level=4, log2_hashmap_size=log2_hashmap_size,
                                base_resolution=16, max_resolution_factor=2.0, nDetector=list(geometry.nDetector),
                                nVoxel=list(geometry.nVoxel))
        net = MLPNetConfig(n_hidden_layers=4, n_neurons=128, activation="LeakyReLU", output_activation="None",
                           include_identity=True)
        return ModelConfig("quadcubes", enc, net, precision)
    enc = HashEncoderConfig(n_levels=19, n_features_per_level=4, log2_hashmap_size=log2_hashmap_size,
                            base_resolution=8, max_resolution_factor=2.0, nDetector=list(geometry.nDetector),
                            nVoxel=list(geometry.nVoxel))
    net = MLPNetConfig(n_hidden_layers=6, n_neurons=64, activation="LeakyReLU", output_activation="ReLU")
    return ModelConfig("hash_grid", enc, net, precision)


def fused_dynamic_config(geometry: Geometry, precision: str, log2_hashmap_size: int = 21) -> ModelConfig:
    """The dynamic model of the fused kernels: one 4D grid of 16 levels x 2
    features, temporal base resolution 4, 2 x 64 ReLU MLP with a softplus
    output (the benchmark's 4D model)."""
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=log2_hashmap_size,
                            base_resolution=16, max_resolution_factor=2.0, nDetector=list(geometry.nDetector),
                            nVoxel=list(geometry.nVoxel), base_resolution_t=4)
    return ModelConfig("hash_grid_4d", enc, MLPNetConfig(n_hidden_layers=2), precision)


# ---------------------------------------------------------- quality presets ----
# The fields the quality presets change, as the reference's configuration
# starts them: nect/cfg/default.yaml (loss L1, base_lr 1e-3, warm-up 500 steps
# from lr0 1e-3, epochs / lrf / points_per_ray.end "auto") overlaid by the
# model preset of each mode (nect/cfg/static/hash_grid.yaml: 2^21 entries;
# nect/cfg/dynamic/quadcubes.yaml: 2^23 entries, base_lr 2e-4, warm-up 2000
# steps from lr0 1e-4).
_COMMON_CONFIG = {"loss": "l1", "epochs": "auto", "lrf": "auto", "lr_otype": "cosine", "warmup_otype": "exponential",
                  "points_start": 100, "points_end": "auto", "points_update_interval": "auto", "points_linear": True,
                  "downsampling_start": 2, "downsampling_end": 1, "downsampling_update_interval": 1000,
                  "points_per_batch": "auto", "s3im": False, "add_poisson": False, "batch_per_proj": 1,
                  "clip_grad_value": None, "optimizer": "Adam", "beta1": 0.9, "beta2": 0.999, "weight_decay": 0.0}
_BASE_CONFIG = {
    "static": dict(_COMMON_CONFIG, base_lr=1e-3, warmup_steps=500, warmup_lr0=1e-3, log2_hashmap_size=21),
    "dynamic": dict(_COMMON_CONFIG, base_lr=2e-4, warmup_steps=2000, warmup_lr0=1e-4, log2_hashmap_size=23),
}

# config_override keys (the reference's configuration schema, nect/config.py)
# -> the fields above; nested sections map key by key.
_OVERRIDE_KEYS = {
    "epochs": "epochs", "base_lr": "base_lr", "loss": "loss", "points_per_batch": "points_per_batch",
    "s3im": "s3im", "add_poisson": "add_poisson", "batch_per_proj": "batch_per_proj",
    "clip_grad_value": "clip_grad_value",
    ("warmup", "steps"): "warmup_steps", ("warmup", "lr0"): "warmup_lr0", ("warmup", "otype"): "warmup_otype",
    ("lr_scheduler", "otype"): "lr_otype", ("lr_scheduler", "lrf"): "lrf",
    ("points_per_ray", "start"): "points_start", ("points_per_ray", "end"): "points_end",
    ("points_per_ray", "update_interval"): "points_update_interval", ("points_per_ray", "linear"): "points_linear",
    ("downsampling_detector", "start"): "downsampling_start", ("downsampling_detector", "end"): "downsampling_end",
    ("downsampling_detector", "update_interval"): "downsampling_update_interval",
    ("encoder", "log2_hashmap_size"): "log2_hashmap_size",
    ("optimizer", "otype"): "optimizer", ("optimizer", "beta1"): "beta1", ("optimizer", "beta2"): "beta2",
    ("optimizer", "weight_decay"): "weight_decay",
}

# nect/reconstruct.py:173-204: per quality, the fields set and the factor the
# base learning rate is multiplied ("mul") or divided ("div") by.
QUALITY_PRESETS = {
    "poor": {"set": {"loss": "l2", "log2_hashmap_size": 19, "epochs": "0.02x"}, "lr": ("mul", 10)},
    "low": {"set": {"loss": "l2", "log2_hashmap_size": 19, "epochs": "0.1x"}, "lr": ("mul", 5)},
    "medium": {"set": {"epochs": "0.3x"}, "lr": ("mul", 2)},
    "high": {"set": {"epochs": "1x", "warmup_steps": 500}, "lr": ("div", 2)},
    "higher": {"set": {"epochs": "2x", "warmup_steps": 3000, "lrf": 0.05, "points_end": "1.5x"}, "lr": ("div", 2)},
    "highest": {"set": {"epochs": "4x", "warmup_steps": 5000, "lrf": 0.01, "points_end": "1.5x",
                        "log2_hashmap_size": 23}, "lr": ("div", 5)},
}

# points_per_batch "auto" fills free device memory up to this cap
# (nect/config.py:380-388); a B200's 180 GB always reaches it.
AUTO_POINTS_PER_BATCH = 5_000_000


def apply_override(cfg: dict, override: dict) -> dict:
    """``config_override`` (keys of the reference's configuration, e.g.
    {"epochs": 3, "warmup": {"steps": 10}}) applied to the fields; keys this
    path has no use for raise ValueError."""
    out = dict(cfg)
    for key, value in override.items():
        if isinstance(value, dict):
            for sub, v in value.items():
                if (key, sub) not in _OVERRIDE_KEYS:
                    raise ValueError(f"config_override: {key}.{sub} is not supported here")
                out[_OVERRIDE_KEYS[(key, sub)]] = v
        elif key in _OVERRIDE_KEYS:
            out[_OVERRIDE_KEYS[key]] = value
        else:
            raise ValueError(f"config_override: {key} is not supported here")
    if isinstance(out["loss"], str):
        out["loss"] = out["loss"].lower()
    if str(out["optimizer"]).casefold() != "adam":
        raise ValueError(f"config_override: optimizer {out['optimizer']} is not supported here (the fused "
                         "update is Adam)")
    return out


def preset_config(mode: str, quality: str = "high", niter=None, lr: float | None = None,
                  config_override: dict | None = None) -> dict:
    """The configuration fields of ``reconstruct(mode, quality, niter, lr,
    config_override)``: the preset applied to the mode's defaults, then
    ``niter`` replacing the epochs and ``lr`` the base learning rate, then the
    override (nect/reconstruct.py:205-216)."""
    if quality not in QUALITY_PRESETS:
        raise ValueError(f"quality must be one of {list(QUALITY_PRESETS)} (got {quality!r})")
    if mode not in _BASE_CONFIG:
        raise ValueError(f"mode must be 'static' or 'dynamic' (got {mode!r})")
    cfg = dict(_BASE_CONFIG[mode])
    preset = QUALITY_PRESETS[quality]
    cfg.update(preset["set"])
    op, k = preset["lr"]
    cfg["base_lr"] = cfg["base_lr"] * k if op == "mul" else cfg["base_lr"] / k
    if niter is not None:
        cfg["epochs"] = niter
    if lr is not None:
        cfg["base_lr"] = lr
    if config_override:
        cfg = apply_override(cfg, config_override)
    return cfg


def learning_rate(base_lr: float, points_per_batch: int, n_gpus: int = 1) -> float:
    """base_lr * sqrt(points_per_batch * n_gpus / 10^6) (nect/config.py:398-399)."""
    return base_lr * math.sqrt(points_per_batch * n_gpus / 1_000_000)


@dataclass
class ReconstructionPlan:
    """What ``reconstruct`` trains with: the model configuration, the
    per-projection schedule, the loss and the points per batch the trainer
    samples (half the configured number, base_trainer.py:141-143)."""
    model_cfg: ModelConfig
    schedule: Schedule
    loss: str
    points_per_batch: int
    config: dict


def plan_reconstruction(geometry: Geometry, mode: str, n_projections: int, quality: str = "high", niter=None,
                        lr: float | None = None, precision: str = "mixed", points_per_batch: int | None = None,
                        n_gpus: int = 1, config_override: dict | None = None) -> ReconstructionPlan:
    """The quality preset resolved for this geometry and projection count."""
    cfg = preset_config(mode, quality, niter, lr, config_override)
    if points_per_batch is None:
        points_per_batch = AUTO_POINTS_PER_BATCH if cfg["points_per_batch"] == "auto" else cfg["points_per_batch"]
    ppb = int(points_per_batch)
    schedule = Schedule(list(geometry.nDetector), n_projections, epochs=cfg["epochs"],
                        base_lr=learning_rate(cfg["base_lr"], ppb, n_gpus),
                        downsampling_start=cfg["downsampling_start"], downsampling_end=cfg["downsampling_end"],
                        downsampling_update_interval=cfg["downsampling_update_interval"],
                        points_start=cfg["points_start"], points_end=cfg["points_end"],
                        points_update_interval=cfg["points_update_interval"], points_linear=cfg["points_linear"],
                        warmup_steps=cfg["warmup_steps"], warmup_lr0=cfg["warmup_lr0"],
                        warmup_otype=cfg["warmup_otype"] or "exponential", lr_otype=cfg["lr_otype"],
                        lrf=cfg["lrf"], n_gpus=n_gpus)
    return ReconstructionPlan(default_model_config(geometry, mode, precision, cfg["log2_hashmap_size"]), schedule,
                              cfg["loss"], ppb // 2, cfg)


def step_plan(n_proj: int, seed: int, niter: int, schedule=None, start: int = 0):
    """(step, projection index, schedule settings or None) for steps
    start + 1 .. niter.  Each epoch visits the projections in a seeded random
    order, drawn anew at the end of every epoch (epoch e uses seed + e * n_proj,
    epoch 0 the seed), so a run resumed after ``start`` steps takes the steps
    an uninterrupted run would."""
    settings = iter(schedule.steps(start)) if schedule is not None else None
    epoch = start // n_proj
    order = np.random.default_rng(seed if epoch == 0 else seed + epoch * n_proj).permutation(n_proj)
    for step in range(start + 1, niter + 1):
        k = int(order[(step - 1) % n_proj])
        if (step - 1) % n_proj == n_proj - 1:
            order = np.random.default_rng(seed + step).permutation(n_proj)
        yield step, k, (next(settings) if settings is not None else None)


def fit(geometry: Geometry, projections: torch.Tensor, angles, timesteps=None, *, model_cfg: ModelConfig | None = None,
        precision: str = "mixed", niter: int = 2000, lr: float = 1e-3, rays_per_batch: int = 65536,
        points_per_ray: int | None = None, points_per_batch: int | None = None, loss: str = "l2", seed: int = 0,
        device="cuda",
        evaluate=None, eval_every: int = 0, schedule=None, s3im: bool = False,
        add_poisson: bool = False, tv: float = 0.0, resume_from=None, checkpoint_dir=None,
        checkpoint_interval: float | None = None, log_fn=None, cancel_at=None, batch_per_proj: int | str = 1,
        clip_grad_value: float | None = None, betas=(0.9, 0.999), weight_decay: float = 0.0) -> Reconstruction:
    """Train a model on ``projections`` [N, rows, cols] (raw line integrals) at
    ``angles`` (radians) and optional ``timesteps``.  Projections are min-max
    scaled over the data set (nect/data.py:177-183).  ``evaluate(rec)`` is
    called every ``eval_every`` steps (and at the end) outside the training
    time; its dict is recorded in ``history``.

    With a ``schedule`` (nect_b200.schedule.Schedule) each step takes that
    projection's detector binning (pooled projection, binned geometry, random
    detector offset while binned), points per ray and learning rate, for
    min(niter, schedule.total_projections) steps.  ``s3im`` adds the S3IM
    term after the schedule's warm-up (base_trainer.py:557-566) and
    ``add_poisson`` the reference's Poisson term and ``tv`` > 0 the
    total-variation term of a static model on a random 100^3 sub-grid after
    the warm-up (base_trainer.py:615-649); these run the step as forward
    half, torch loss, backward half.

    ``checkpoint_dir`` gets the run's checkpoint (checkpoint.save: model,
    Adam state, epoch and angle; the previous one kept as 2nd_last.ckpt) at
    the start, every ``checkpoint_interval`` seconds and at the end
    (base_trainer.py:297-299, 452-478).
    ``resume_from`` (a last.ckpt) restores the model, the Adam state and the
    position, and training continues from the next projection with the
    schedule's settings at that point (base_trainer.py:189-212).  Random
    draws (ray permutations, jitter, TV sub-grids) are not replayed.

    ``log_fn(step, metrics)`` is called after every step with the keys the
    reference logs (base_trainer.py:596-609: loss, max_mem, current_mem,
    epoch, downsample_detector_factor, points_per_ray,
    distance_between_points, lr, num_proj_processed) and the batch's rays;
    the loss is the device tensor, so logging adds no synchronisation unless
    ``log_fn`` reads it.

    ``cancel_at`` (an ISO date-time string or datetime; UTC when it names no
    zone) ends training after the first step that finishes later, saving the
    checkpoint; a KeyboardInterrupt ends it too, saving only after more than
    3000 steps (base_trainer.py:281-284, 659-666).  Where the reference then
    exits the process, this returns the Reconstruction with ``stopped`` set.

    ``batch_per_proj`` (an int or "all") batches of rays are taken from each
    projection visit, each an optimizer step with the projection's settings,
    up to the batches the detector holds (base_trainer.py:517-520);
    ``clip_grad_value`` clamps the gradients before each Adam step
    (base_trainer.py:651-652); ``betas`` and ``weight_decay`` are Adam's
    (nect/config.py:409-413).  ``niter``, checkpoints and resume count
    projection visits."""
    dev = torch.device(device)
    proj = torch.as_tensor(projections, dtype=torch.float32, device=dev)
    n_proj = proj.shape[0]
    mn, mx = float(proj.min()), float(proj.max())
    proj = ((proj - mn) / (mx - mn)).reshape(n_proj, -1).contiguous()
    angles = [float(a) for a in angles]
    if timesteps is None:
        ts = [0.0] * n_proj
    else:
        tt = np.asarray(timesteps, np.float64)
        ts = list(tt / tt.max()) if tt.max() > 0 else [0.0] * n_proj   # nect/data.py:78-79
    mode = "static" if timesteps is None else "dynamic"
    cfg = model_cfg or default_model_config(geometry, mode, precision)
    torch.manual_seed(seed)
    model = get_model(cfg, device=dev)
    S = points_per_ray or int(math.ceil(1.5 * max(geometry.nDetector)))
    if isinstance(model, QuadCubes):
        # the module loop, at most the reference's 5 M points per batch (config.py:380-391)
        trainer = ModuleTrainer(model, geometry, points_per_batch=min(points_per_batch or rays_per_batch * S,
                                                                      5_000_000),
                                points_per_ray=S, loss=loss, lr=lr, betas=tuple(betas), weight_decay=weight_decay,
                                device=dev, clip_grad_value=clip_grad_value)
    else:
        trainer = Trainer(model, geometry, points_per_batch=points_per_batch or rays_per_batch * S, points_per_ray=S,
                          loss=loss, lr=lr, betas=tuple(betas), weight_decay=weight_decay, device=dev,
                          clip_grad_value=clip_grad_value)
    n_batches = 10 ** 9 if batch_per_proj == "all" else int(batch_per_proj)
    rec = Reconstruction(model, geometry, mn, mx, trainer)
    if isinstance(cancel_at, str):
        try:
            cancel_at = datetime.datetime.fromisoformat(cancel_at)
        except ValueError:
            raise ValueError(f"cancel_at {cancel_at!r} is not an ISO date-time") from None
    if cancel_at is not None and cancel_at.tzinfo is None:
        cancel_at = cancel_at.replace(tzinfo=datetime.timezone.utc)
    start = 0
    if resume_from is not None:
        from . import checkpoint

        pos = checkpoint.resume(resume_from, model, trainer)
        start = int(pos["epoch"]) * n_proj + int(pos["angle"])
    train_s = 0.0

    def record(step):
        if evaluate is not None:
            torch.cuda.synchronize(dev)
            rec.history.append((step, train_s, evaluate(rec)))

    def save(step, with_geometry=False):
        from . import checkpoint

        checkpoint.save(checkpoint_dir, model, trainer, geometry if with_geometry else None,
                        epoch=step // n_proj, angle=step % n_proj, keep_two=True)

    if schedule is not None:
        niter = min(niter, schedule.total_projections)
        rows, cols = geometry.nDetector
        raw = proj.view(n_proj, rows, cols)
        ppb = trainer.points_per_batch
    binning = 1
    tv_rng = np.random.default_rng(seed + 7)
    if checkpoint_dir is not None:
        save(start, with_geometry=True)   # config and geometry before any detector binning
    last_save = time.perf_counter()
    record(start)
    done, taken = start, 0   # projection visits completed, optimizer steps taken in this call
    try:
        for step, k, st in step_plan(n_proj, seed, niter, schedule, start):
            t0 = time.perf_counter()
            target = proj[k]
            if st is not None:
                if st.detector_binning != binning:
                    binning = st.detector_binning
                    geometry.set_detector_binning(binning)
                    trainer.c_geometry = geometry.get_c_geometry()
                target = bin_projection(raw[k], binning).reshape(-1).contiguous()
                trainer.points_per_ray = st.points_per_ray
                trainer.points_per_batch = ppb
                trainer.random_offset_detector = st.random_offset_detector
                trainer.lr = st.lr
            perm = torch.randperm(target.numel(), dtype=torch.int64, device=dev)
            for batch_num in range(n_batches):
                batch = trainer.make_batch(perm, batch_num, angles[k], target, ts[k])
                if batch is None:   # past the detector's batches (Projector.batch_per_epoch)
                    break
                if s3im or add_poisson or tv > 0:
                    warm = schedule.warmup[0] if schedule is not None else 0
                    patch = s3im_patch_size(target.numel(), trainer.batch_size) if s3im and step > warm else 0
                    tv_w = tv if (tv > 0 and mode == "static" and step > warm) else 0.0
                    loss = trainer.split_step(batch, add_poisson=add_poisson, s3im_patch=patch, tv_weight=tv_w,
                                              tv_origin=tv_rng.random(3) * 0.8 if tv_w else None)
                else:
                    loss = trainer.step(batch)
                taken += 1
                if log_fn is not None:
                    on_gpu = dev.type == "cuda"
                    free, total = torch.cuda.mem_get_info(dev) if on_gpu else (0, 0)
                    log_fn(trainer.step_count, {
                        "loss": loss, "max_mem": torch.cuda.max_memory_allocated(dev) if on_gpu else 0,
                        "current_mem": total - free, "epoch": (step - 1) // n_proj,
                        "downsample_detector_factor": binning, "points_per_ray": trainer.points_per_ray,
                        "distance_between_points": batch.max_ray_distance_per_point, "lr": trainer.lr,
                        "num_proj_processed": step - 1, "rays": batch.num_rays})
            done = step
            if eval_every and (step % eval_every == 0 or step == niter):
                torch.cuda.synchronize(dev)
                train_s += time.perf_counter() - t0
                record(step)
            else:
                train_s += time.perf_counter() - t0
            if checkpoint_interval is not None and checkpoint_dir is not None and \
                    time.perf_counter() - last_save >= checkpoint_interval:
                save(step)
                last_save = time.perf_counter()
            if cancel_at is not None and datetime.datetime.now(datetime.timezone.utc) > cancel_at:
                rec.stopped = "cancelled"
                break
    except KeyboardInterrupt:
        rec.stopped = "interrupted"
    torch.cuda.synchronize(dev)
    if binning != 1:
        geometry.set_detector_binning(1)
        trainer.c_geometry = geometry.get_c_geometry()
    # after an interrupt the reference saves only runs of more than 3000 steps
    if checkpoint_dir is not None and done > start and (rec.stopped != "interrupted" or taken > 3000):
        save(done)
    rec.train_seconds = train_s
    return rec


def reconstruct(geometry: Geometry, projections, mode: str = "static", angles=None, radians: bool = True,
                quality: str = "high", niter: int | None = None, lr: float | None = None, timesteps=None,
                verbose: bool = True, log: bool = False, exp_name: str | None = None,
                flip_projections: bool = False, channel_order: str | None = None,
                config_override: dict | None = None, save_ckpt: bool = False, precision: str = "mixed",
                points_per_batch: int | None = None, **kw):
    """``nect.reconstruct`` (nect/reconstruct.py:113-250) for arrays of
    projections [N, rows, cols]: returns the volume (np.ndarray [z, y, x],
    turned by 180 degrees in (y, x) as the reference returns it) for mode
    "static" and the Reconstruction (export any t with ``.volume(t)``) for
    mode "dynamic".

    As in the reference, ``quality`` picks the preset (epochs, learning rate,
    warm-up, final lr fraction, points per ray, hash-table size and loss),
    ``niter`` replaces the preset's epochs, ``lr`` its base learning rate and
    ``config_override`` any field this path uses (ValueError for others);
    training follows the per-projection schedules (detector binning,
    points-per-ray ramp, warm-up and decay) for epochs x projections steps
    (plan_reconstruction).  ``flip_projections`` and ``channel_order`` act on
    projections read from files, which the reference's in-memory path leaves
    as given, and so do nothing here; ``save_ckpt`` writes the checkpoint and
    its pruned copy under outputs/<exp_name> (checkpoint.save / prune);
    ``verbose`` prints the plan and the training time; ``log`` has no
    effect."""
    if isinstance(projections, (str, bytes)) or hasattr(projections, "__fspath__"):
        raise ValueError("projections must be an array [N, rows, cols]: reading projection files is not part "
                         "of this package")
    if angles is None:
        angles = geometry.angles
    angles = np.asarray(angles, np.float64)
    if not radians:
        angles = np.deg2rad(angles)
    if mode == "dynamic" and timesteps is None:
        timesteps = getattr(geometry, "timesteps", None)
        if timesteps is None:
            timesteps = np.arange(len(angles), dtype=np.float64)
    plan = plan_reconstruction(geometry, mode, len(angles), quality, niter, lr, precision, points_per_batch,
                               config_override=config_override)
    kw.setdefault("s3im", bool(plan.config["s3im"]))
    kw.setdefault("add_poisson", bool(plan.config["add_poisson"]))
    kw.setdefault("batch_per_proj", plan.config["batch_per_proj"])
    kw.setdefault("clip_grad_value", plan.config["clip_grad_value"])
    kw.setdefault("betas", (plan.config["beta1"], plan.config["beta2"]))
    kw.setdefault("weight_decay", plan.config["weight_decay"])
    if verbose:
        sch = plan.schedule
        print(f"nect_b200.reconstruct: {mode}, quality {quality}: {sch.total_projections} steps "
              f"({sch.epochs} epochs x {len(angles)} projections), lr {sch.lr[0]:.3g}, loss {plan.loss}, "
              f"{plan.points_per_batch} points per batch, 2^{plan.model_cfg.encoder.log2_hashmap_size} entries")
    rec = fit(geometry, projections, angles, timesteps if mode == "dynamic" else None, model_cfg=plan.model_cfg,
              precision=precision, niter=plan.schedule.total_projections, lr=plan.schedule.lr[0],
              points_per_batch=plan.points_per_batch, loss=plan.loss, schedule=plan.schedule, **kw)
    if verbose:
        print(f"nect_b200.reconstruct: trained in {rec.train_seconds:.1f} s")
    if save_ckpt:
        from . import checkpoint

        run = Path("outputs") / (exp_name or "reconstruction")
        checkpoint.save(run, rec.model, rec.trainer, geometry)
        checkpoint.prune(run)
    if mode == "static":
        # the reference returns create_volume turned by 180 degrees in (y, x)
        # (nect/reconstruct.py:246-247)
        return torch.rot90(rec.volume(), 2, (1, 2)).contiguous().cpu().numpy()
    return rec


# ------------------------------------------------------------ evaluation ----
def psnr(x: torch.Tensor, y: torch.Tensor) -> float:
    """-10 log10(MSE), as nect/src/evaluation/evaluator.py:17-19."""
    return float(-10 * torch.log10(torch.nn.functional.mse_loss(x.float(), y.float())))


def ssim3d(x: torch.Tensor, y: torch.Tensor, data_range: float | None = None, win: int = 7,
           sigma: float = 1.5) -> float:
    """Structural similarity (Wang et al., IEEE TIP 13(4), 2004) with a
    separable Gaussian window over three dimensions (K1 = 0.01, K2 = 0.03)."""
    x = x.float()[None, None]
    y = y.float()[None, None]
    L = data_range if data_range is not None else float(y.max() - y.min())
    g = torch.exp(-((torch.arange(win, device=x.device) - win // 2) ** 2) / (2 * sigma ** 2))
    g = (g / g.sum()).float()

    def blur(v):
        for dim in range(3):
            shape = [1, 1, 1, 1, 1]
            shape[2 + dim] = win
            v = torch.nn.functional.conv3d(v, g.view(shape))
        return v

    mx, my = blur(x), blur(y)
    sxx = blur(x * x) - mx * mx
    syy = blur(y * y) - my * my
    sxy = blur(x * y) - mx * my
    c1, c2 = (0.01 * L) ** 2, (0.03 * L) ** 2
    s = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    return float(s.mean())


def fbp_parallel(projections: torch.Tensor, geometry: Geometry, angles) -> torch.Tensor:
    """Filtered back-projection (Ram-Lak filter, linear interpolation) of
    parallel-beam projections [N, rows, cols] on the geometry's voxel grid
    [z, y, x]: the classical reconstruction without a learned model that the
    reference runs through tigre (nect/fdk.py).  Angles must cover [0, pi)
    evenly.  Detector conventions as the sampler (ct_sampling.cu:226-256):
    column u maps to world -y before rotation, row v to z, so the ray of
    pixel u at angle a is {x sin a - y cos a = u}."""
    if geometry.mode != "parallel":
        raise ValueError("fbp_parallel needs a parallel-beam geometry")
    dev = projections.device
    p = projections.double()
    n, nr, nc = p.shape
    du = geometry.dDetector[1]
    # Ram-Lak kernel in the spatial domain, zero-padded linear convolution via FFT
    m = 1 << int(math.ceil(math.log2(2 * nc)))
    k = torch.arange(-(nc - 1), nc, device=dev, dtype=torch.float64)
    h = torch.zeros_like(k)
    h[k == 0] = 1.0 / (4 * du * du)
    odd = (k.abs() % 2) == 1
    h[odd] = -1.0 / (math.pi ** 2 * k[odd] ** 2 * du * du)
    H = torch.fft.rfft(h, m)
    q = torch.fft.irfft(torch.fft.rfft(p, m, dim=-1) * H, m, dim=-1)[..., nc - 1:2 * nc - 1] * du
    nz, ny, nx = geometry.nVoxel
    dz, dy, dx = geometry.dVoxel
    xs = (torch.arange(nx, device=dev, dtype=torch.float64) - (nx - 1) / 2) * dx + geometry.offOrigin[2]
    ys = (torch.arange(ny, device=dev, dtype=torch.float64) - (ny - 1) / 2) * dy + geometry.offOrigin[1]
    Y, X = torch.meshgrid(ys, xs, indexing="ij")
    u0 = -(nc - 1) / 2 * du + geometry.offDetector[1]
    zs = (torch.arange(nz, device=dev, dtype=torch.float64) - (nz - 1) / 2) * dz + geometry.offOrigin[0]
    rows = ((zs - geometry.offDetector[0]) / geometry.dDetector[0] + (nr - 1) / 2).round().long().clamp(0, nr - 1)
    vol = torch.zeros(nz, ny, nx, device=dev, dtype=torch.float64)
    for i, a in enumerate(angles):
        u = X * math.sin(a) - (Y - geometry.COR) * math.cos(a)
        f = (u - u0) / du
        j0 = f.floor().long()
        w = f - j0
        ok0 = (j0 >= 0) & (j0 < nc)
        ok1 = (j0 + 1 >= 0) & (j0 + 1 < nc)
        qi = q[i][rows]                                   # [nz, nc]
        v0 = qi[:, j0.clamp(0, nc - 1)] * ok0
        v1 = qi[:, (j0 + 1).clamp(0, nc - 1)] * ok1
        vol += v0 * (1 - w) + v1 * w
    return (vol * math.pi / len(angles)).float()
