"""Checkpoints in the reference's layout.

The reference saves a training run as a directory (nect/trainers/base_trainer.py:452-484,
nect/config.py:499-524, nect/utils.py:132-150):

    <run>/model/config.yaml, <run>/model/geometry.yaml
    <run>/model/checkpoints/last.ckpt   {"model", "optim", "epoch", "angle", "lr_scheduler"}
    <run>/pruned/checkpoints/last.ckpt  {"model"} (plus copies of the two yaml files)

and its export tools read ``torch.load(.../checkpoints/last.ckpt)["model"]``
into the module from ``config.get_model()`` (nect/static_export.py:53-54,
nect/dynamic_export.py:180-183, 338-339).  ``save`` and ``prune`` write the
same files and keys here; "model" is the state dict of this package's module
(keys ``table`` and ``mlp``: the fp32 hash table [entries, features] and the
flat fp32 MLP weights, PyTorch Linear layout), and "optim" is the Adam state in
torch.optim.Adam's own state-dict format (parameter 0 = table, 1 = mlp), so a
stock torch Adam over [model.table, model.mlp] can resume from it as well.
The tiny-cuda-nn flat parameter layout of the reference's own modules is not
written: tiny-cuda-nn is not part of the reference tree and its layout is not
pinned here.
"""
from __future__ import annotations

import shutil
from dataclasses import asdict
from pathlib import Path

import torch
import yaml

from .config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
from .network import _HashGridModel
from .trainer import Trainer


def _adam_state(trainer: Trainer) -> dict:
    state = {}
    for i, (m, v) in enumerate(trainer.optimizer_moments()):
        state[i] = {"step": torch.tensor(float(trainer.step_count)), "exp_avg": m.detach().clone(),
                    "exp_avg_sq": v.detach().clone()}
    group = {"lr": trainer.lr, "betas": tuple(trainer.betas), "eps": trainer.eps,
             "weight_decay": trainer.weight_decay, "amsgrad": False, "maximize": False, "foreach": None,
             "capturable": False, "differentiable": False, "fused": None, "params": sorted(state)}
    return {"state": state, "param_groups": [group]}


def _config_dict(model: _HashGridModel) -> dict:
    enc = asdict(model.encoding_config)
    enc.pop("nDetector", None)   # as Config.save drops them (config.py:504-505)
    enc.pop("nVoxel", None)
    from .quadcubes import QuadCubes

    name = "quadcubes" if isinstance(model, QuadCubes) else ("hash_grid_4d" if model.n_dims == 4 else "hash_grid")
    return {"model": name, "mode": "dynamic" if model.n_dims == 4 else "static", "precision": model.precision,
            "encoder": enc, "net": asdict(model.network_config), "geometry": "SAME_FOLDER"}


def _geometry_dict(geometry) -> dict:
    g = dict(geometry.to_dict())
    for k, v in list(g.items()):
        if hasattr(v, "tolist"):
            g[k] = v.tolist()
        elif isinstance(v, tuple):
            g[k] = list(v)
    return g


def save(run_dir: str | Path, model: _HashGridModel, trainer: Trainer | None = None, geometry=None,
         epoch: int = 0, angle: int = 0, keep_two: bool = False) -> Path:
    """Write ``run_dir/model/{config.yaml, geometry.yaml, checkpoints/last.ckpt}``.
    With ``keep_two`` an existing last.ckpt first becomes 2nd_last.ckpt
    (base_trainer.py:469-475).

    With a trainer whose optimizer is sharded over data-parallel ranks every
    rank calls this (the Adam moments are gathered); rank 0 writes."""
    adam = _adam_state(trainer) if trainer is not None else None
    if trainer is not None and trainer.sharded is not None and trainer.sharded.rank != 0:
        return Path(run_dir) / "model" / "checkpoints" / "last.ckpt"
    base = Path(run_dir) / "model"
    (base / "checkpoints").mkdir(parents=True, exist_ok=True)
    with open(base / "config.yaml", "w") as f:
        yaml.safe_dump(_config_dict(model), f)
    if geometry is not None:
        with open(base / "geometry.yaml", "w") as f:
            yaml.safe_dump(_geometry_dict(geometry), f, default_flow_style=None)
    state = {"model": {k: v.detach().cpu() for k, v in model.state_dict().items()}, "epoch": epoch, "angle": angle}
    if trainer is not None:
        state["optim"] = {"state": {i: {k: (v.cpu() if torch.is_tensor(v) else v) for k, v in s.items()}
                                    for i, s in adam["state"].items()},
                          "param_groups": adam["param_groups"]}
        state["lr_scheduler"] = {"lr": trainer.lr}
    path = base / "checkpoints" / "last.ckpt"
    if keep_two and path.exists():
        path.replace(base / "checkpoints" / "2nd_last.ckpt")
    torch.save(state, path)
    return path


def prune(run_dir: str | Path) -> Path:
    """The model-only copy ``run_dir/pruned/checkpoints/last.ckpt`` (utils.py:132-150)."""
    src = Path(run_dir) / "model"
    data = torch.load(src / "checkpoints" / "last.ckpt", map_location="cpu", weights_only=False)
    dst = Path(run_dir) / "pruned"
    (dst / "checkpoints").mkdir(parents=True, exist_ok=True)
    torch.save({"model": data["model"]}, dst / "checkpoints" / "last.ckpt")
    for name in ("config.yaml", "geometry.yaml"):
        if (src / name).exists():
            shutil.copy(src / name, dst / name)
    return dst / "checkpoints" / "last.ckpt"


def model_from_dir(base: str | Path, device="cuda", precision: str | None = None) -> _HashGridModel:
    """Build the model described by ``base/config.yaml`` and load
    ``base/checkpoints/last.ckpt`` into it (what the export tools do)."""
    base = Path(base)
    with open(base / "config.yaml") as f:
        cfg = yaml.safe_load(f)
    enc = HashEncoderConfig(**cfg["encoder"])
    net = MLPNetConfig(**cfg["net"])
    model = get_model(ModelConfig(cfg["model"], enc, net, precision or cfg.get("precision", "plain_fp32")),
                      device=device)
    data = torch.load(base / "checkpoints" / "last.ckpt", map_location="cpu", weights_only=False)
    model.load_state_dict(data["model"])
    return model


def resume(path: str | Path, model: _HashGridModel, trainer: Trainer | None = None) -> dict:
    """Load a checkpoint file into ``model`` (and the Adam state into
    ``trainer``); returns {"epoch", "angle"} (base_trainer.py:188-198)."""
    data = torch.load(path, map_location="cpu", weights_only=False)
    model.load_state_dict(data["model"])
    if trainer is not None and "optim" in data:
        st = data["optim"]["state"]
        trainer.load_optimizer_moments([(st[i]["exp_avg"], st[i]["exp_avg_sq"]) for i in sorted(st)])
        trainer.step_count = int(float(st[0]["step"]))
    return {"epoch": data.get("epoch", 0), "angle": data.get("angle", 0)}
