"""Hash-grid models behind the reference's module interface.

``HashGrid(encoding_config, network_config)`` keeps the constructor and the
static ``forward(x) -> [N, 1]`` of nect/network/networks.py:28-65;
``HashGrid4D`` is the dynamic ``forward(x, t) -> [N, 1]`` model with one 4D
(z, y, x, t) grid (the 4D component of HyperCubes, networks.py:478-481, with t
broadcast like networks.py:85).  Parameters are an fp32 table
``[entries, n_features]`` (level after level) and one fp32 MLP weight vector in
PyTorch Linear layout; with ``precision="mixed"`` an fp16 copy of the table is
kept for the gathers and refreshed by the fused Adam step.

Initialisation: table entries U(-1e-4, 1e-4) (Mueller et al. 2022, section 4);
weights Glorot-uniform per layer.  ``forward`` runs the CUDA model kernel
(inference; training goes through ``nect_b200.trainer``).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .config import HashEncoderConfig, MLPNetConfig

_ACT_NAMES = {"none": "none", "relu": "relu", "leakyrelu": "leakyrelu", "softplus": "softplus", "sigmoid": "sigmoid"}


def act_code(name: str | None) -> int:
    key = (name or "None").replace("_", "").lower()
    if key not in _ACT_NAMES:
        raise ValueError(f"activation {name!r} is not supported by the B200 path")
    return _lib.ACT[_ACT_NAMES[key]]


class _HashGridModel(nn.Module):
    n_dims = 3

    def __init__(self, encoding_config: HashEncoderConfig, network_config: MLPNetConfig,
                 precision: str = "plain_fp32", device="cuda", seed: int = 1337):
        super().__init__()
        if network_config.include_identity:
            raise NotImplementedError("include_identity is not supported by the fused B200 path")
        if network_config.n_neurons != 64:
            raise NotImplementedError("the fused B200 path supports n_neurons == 64")
        self.precision = precision
        enc = encoding_config
        self.encoding_config = enc
        self.network_config = network_config
        mixed = precision == "mixed"
        self.grid_desc = _lib.NectbHashGrid(
            n_dims=self.n_dims, n_levels=enc.n_levels, n_features=enc.n_features_per_level,
            log2_hashmap_size=enc.log2_hashmap_size, feature_dtype=_lib.F16 if mixed else _lib.F32,
            base_resolution=float(enc.base_resolution), per_level_scale=float(enc.per_level_scale),
            base_resolution_t=float(enc.base_resolution_t or enc.base_resolution))
        L = enc.n_levels
        res = (ctypes.c_int32 * L)()
        res_t = (ctypes.c_int32 * L)()
        off = (ctypes.c_int64 * L)()
        ent = (ctypes.c_int64 * L)()
        hsh = (ctypes.c_int32 * L)()
        total = _lib.lib.nectb_hashgrid_layout(ctypes.byref(self.grid_desc), ctypes.addressof(res),
                                               ctypes.addressof(res_t), ctypes.addressof(off), ctypes.addressof(ent),
                                               ctypes.addressof(hsh))
        if total <= 0:
            raise ValueError("invalid hash-grid configuration")
        self.level_resolution = list(res)
        self.level_resolution_t = list(res_t)
        self.level_offset = list(off)
        self.level_entries = list(ent)
        self.level_hashed = [bool(h) for h in hsh]
        self.n_input = L * enc.n_features_per_level
        self.mlp_desc = _lib.NectbMLP(n_input=self.n_input, n_hidden_layers=network_config.n_hidden_layers,
                                      width=64, activation=act_code(network_config.activation),
                                      output_activation=act_code(network_config.output_activation),
                                      compute_dtype=_lib.BF16 if mixed else _lib.F32)
        gen = torch.Generator(device="cpu").manual_seed(seed)
        table = (torch.rand(total, enc.n_features_per_level, generator=gen) * 2 - 1) * 1e-4
        self.table = nn.Parameter(table.to(device))
        self.mlp = nn.Parameter(self._init_mlp(gen).to(device))
        self.register_buffer("table_half", self.table.detach().half() if mixed else None, persistent=False)

    def _init_mlp(self, gen) -> torch.Tensor:
        shapes = self.mlp_shapes()
        parts = []
        for out_f, in_f in shapes:
            bound = math.sqrt(6.0 / (in_f + out_f))
            parts.append((torch.rand(out_f * in_f, generator=gen) * 2 - 1) * bound)
        return torch.cat(parts)

    def mlp_shapes(self) -> list[tuple[int, int]]:
        H = self.network_config.n_hidden_layers
        return [(64, self.n_input)] + [(64, 64)] * (H - 1) + [(1, 64)]

    @property
    def grid_table(self) -> torch.Tensor:
        """The table the kernels gather from (fp16 copy on the mixed path)."""
        return self.table_half if self.precision == "mixed" else self.table

    @torch.no_grad()
    def refresh_half(self):
        if self.precision == "mixed":
            self.table_half.copy_(self.table)

    def _load_from_state_dict(self, *args, **kwargs):
        super()._load_from_state_dict(*args, **kwargs)
        self.refresh_half()

    @torch.no_grad()
    def _forward(self, x: torch.Tensor, t: float) -> torch.Tensor:
        _lib.require_cuda(x, "x")
        if x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] != 3:
            raise ValueError("x must be fp32 [N, 3] (z, y, x) in [0, 1]")
        n = x.shape[0]
        out = torch.empty(n, 1, device=x.device, dtype=torch.float32)
        rc = _lib.lib.nectb_model_forward(ctypes.byref(self.grid_desc), ctypes.byref(self.mlp_desc),
                                          self.grid_table.data_ptr(), self.mlp.data_ptr(), x.data_ptr(), n,
                                          float(t), out.data_ptr(), _lib.stream_ptr(x.device))
        _lib.check(rc, "nectb_model_forward")
        return out

    def corners(self, x: torch.Tensor):
        """Per-level corner indices/weights [N, L, 2^d] (diagnostic)."""
        _lib.require_cuda(x, "x")
        n = x.shape[0]
        nc = 1 << self.n_dims
        idx = torch.empty(n, self.encoding_config.n_levels, nc, dtype=torch.int32, device=x.device)
        w = torch.empty(n, self.encoding_config.n_levels, nc, dtype=torch.float32, device=x.device)
        rc = _lib.lib.nectb_hashgrid_corners(ctypes.byref(self.grid_desc), x.data_ptr(), n, idx.data_ptr(),
                                             w.data_ptr(), _lib.stream_ptr(x.device))
        _lib.check(rc, "nectb_hashgrid_corners")
        return idx, w

    def encode(self, x: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(x, "x")
        n = x.shape[0]
        out = torch.empty(n, self.n_input, device=x.device, dtype=torch.float32)
        rc = _lib.lib.nectb_hashgrid_encode(ctypes.byref(self.grid_desc), self.grid_table.data_ptr(), x.data_ptr(),
                                            n, out.data_ptr(), _lib.stream_ptr(x.device))
        _lib.check(rc, "nectb_hashgrid_encode")
        return out


class HashGrid(_HashGridModel):
    """Static model: forward(x [N,3] in (z,y,x)) -> sigma [N,1] (networks.py:28-65)."""
    n_dims = 3

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        return self._forward(x.contiguous(), 0.0)


class HashGrid4D(_HashGridModel):
    """Dynamic model with one 4D grid: forward(x [N,3], t in [0,1]) -> sigma [N,1]."""
    n_dims = 4

    def forward(self, x: torch.Tensor, t) -> torch.Tensor:
        if isinstance(t, torch.Tensor):
            t = float(t.item())
        return self._forward(x.contiguous(), float(t))
