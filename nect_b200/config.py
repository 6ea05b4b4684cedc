"""Encoder/network configuration with the reference's fields and rules.

``HashEncoderConfig`` and ``MLPNetConfig`` keep the dataclass fields,
``get_encoder_config``/``get_network_config`` dicts (tiny-cuda-nn schema) and
the ``per_level_scale`` rule of nect/config.py:73-135.  Two keys are added:
``precision`` ("plain_fp32" runs fp32 tables and the fp32 SIMT MLP; "mixed"
runs fp16 tables and the bf16 tensor-core MLP with fp32 accumulation) and
``base_resolution_t`` (temporal base resolution of 4D grids; defaults to
``base_resolution``).  ``get_model`` mirrors Config.get_model
(nect/config.py:288-391) for the hash-grid models this path implements.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Literal, Optional


@dataclass
class HashEncoderConfig:
    otype: str = "HashGrid"
    n_levels: int = 16
    n_features_per_level: int = 2
    log2_hashmap_size: int = 19
    base_resolution: int = 16
    max_resolution_factor: float = 2.0
    nDetector: Optional[list[int] | tuple[int, int]] = None
    nVoxel: Optional[list[int] | tuple[int, int, int]] = None
    sample_outside: Optional[int] = 0
    max_resolution_type: Optional[Literal["nVoxel"] | Literal["nDetector"]] = "nDetector"
    base_resolution_t: Optional[float] = None
    finest_resolution: Optional[int] = None  # overrides the factor rule when set

    def get_encoder_config(self) -> dict:
        return {
            "otype": self.otype,
            "n_levels": self.n_levels,
            "n_features_per_level": self.n_features_per_level,
            "log2_hashmap_size": self.log2_hashmap_size,
            "base_resolution": self.base_resolution,
            "per_level_scale": self.per_level_scale,
        }

    def __str__(self):
        return (f"{self.n_levels}_{self.n_features_per_level}_{self.log2_hashmap_size}_{self.base_resolution}_"
                f"{self.max_resolution_factor}")

    @property
    def per_level_scale(self) -> float:
        """b = (max_resolution_factor * size / base_resolution)^(1/(L-1)) (nect/config.py:99-112)."""
        if self.finest_resolution is not None:
            return (self.finest_resolution / self.base_resolution) ** (1 / (self.n_levels - 1))
        if self.max_resolution_type == "nDetector":
            if self.nDetector is None:
                raise ValueError("nDetector is not provided")
            size = max(self.nDetector)
        elif self.max_resolution_type == "nVoxel":
            if self.nVoxel is None:
                raise ValueError("nVoxel is not provided")
            nVoxel = list(self.nVoxel)
            if self.sample_outside:
                nVoxel = [nVoxel[0], nVoxel[1] + 2 * self.sample_outside, nVoxel[2] + 2 * self.sample_outside]
            size = max(nVoxel)
        else:
            raise ValueError(f"unknown max_resolution_type {self.max_resolution_type}")
        return (self.max_resolution_factor * size / self.base_resolution) ** (1 / (self.n_levels - 1))


@dataclass
class MLPNetConfig:
    otype: str = "FullyFusedMLP"
    n_hidden_layers: int = 2
    n_neurons: int = 64
    activation: str = "ReLU"
    output_activation: str = "Softplus"
    include_adaptive_skip: Optional[bool] = None
    include_identity: Optional[bool] = None

    def get_network_config(self) -> dict:
        return {
            "otype": self.otype,
            "n_hidden_layers": self.n_hidden_layers,
            "n_neurons": self.n_neurons,
            "activation": self.activation,
            "output_activation": self.output_activation,
        }

    def __str__(self):
        return f"{self.n_hidden_layers}_{self.n_neurons}"


PRECISIONS = ("plain_fp32", "mixed")


@dataclass
class ModelConfig:
    """The part of nect.config.Config that selects and builds the model."""
    model: str = "hash_grid"
    encoder: HashEncoderConfig = field(default_factory=HashEncoderConfig)
    net: MLPNetConfig = field(default_factory=MLPNetConfig)
    precision: str = "plain_fp32"

    @property
    def mode(self) -> str:
        return "static" if self.model in ("kplanes", "hash_grid") else "dynamic"


def get_model(cfg: ModelConfig, device="cuda"):
    """Build the model named by ``cfg.model`` (Config.get_model, nect/config.py:288-391).

    "hash_grid" is the static 3D model; "hash_grid_4d" is a single 4D (z,y,x,t)
    hash grid + MLP behind the dynamic ``model(x, t)`` interface (the 4D component
    of HyperCubes, nect/network/networks.py:478-481); "quadcubes" is the
    reference's default dynamic model (networks.py:392-449), four 3D grids
    and a wide MLP, trained by the module loop (quadcubes.ModuleTrainer)."""
    from .network import HashGrid, HashGrid4D

    if cfg.precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {cfg.precision!r}")
    if cfg.model == "hash_grid":
        return HashGrid(cfg.encoder, cfg.net, precision=cfg.precision, device=device)
    if cfg.model in ("hash_grid_4d", "hypercubes_4d"):
        return HashGrid4D(cfg.encoder, cfg.net, precision=cfg.precision, device=device)
    if cfg.model == "quadcubes":
        from .quadcubes import QuadCubes

        return QuadCubes(cfg.encoder, cfg.net, precision=cfg.precision, device=device)
    raise ValueError(f"Model type {cfg.model} is not supported by the B200 path")
