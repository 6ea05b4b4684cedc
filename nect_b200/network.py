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
weights Glorot-uniform per layer.  ``forward`` runs the CUDA model kernel;
when autograd records it is a differentiable node (``ModelPoints``, the
hand-written backward), so ``loss.backward()`` through ``model(points)``
trains the table and the MLP as in the reference's loop.  The fused
training step of ``nect_b200.trainer`` is the fast path for ray batches.
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

    def _forward(self, x: torch.Tensor, t) -> torch.Tensor:
        """sigma [N, 1] at x [N, 3]; differentiable in (table, mlp) whenever
        autograd records (the hand-written backward, ModelPoints), plain
        inference otherwise."""
        if torch.is_grad_enabled() and (self.table.requires_grad or self.mlp.requires_grad):
            sigma = ModelPoints.apply(self.table, self.mlp, self, x, t)
        else:
            sigma = _model_forward(self, x, t)
        return sigma.unsqueeze(1)

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
        return self._forward(x, 0.0)


class HashGrid4D(_HashGridModel):
    """Dynamic model with one 4D grid: forward(x [N,3], t in [0,1]) -> sigma [N,1].

    t is a float or a one-element tensor; a CUDA tensor stays on the device
    (the kernels read it there, as the reference broadcasts it on the device,
    networks.py:85), so a dynamic query never waits for the host."""
    n_dims = 4

    def forward(self, x: torch.Tensor, t) -> torch.Tensor:
        return self._forward(x, t)


def _timestep(t):
    """(host value, device tensor or None) of a timestep argument."""
    if isinstance(t, torch.Tensor):
        if t.numel() != 1:
            raise ValueError(f"t must hold one value, got shape {tuple(t.shape)}")
        if t.is_cuda:
            return 0.0, t.detach().reshape(1).to(torch.float32).contiguous()
        return float(t.reshape(())), None
    return float(t), None


def _check_points(x: torch.Tensor) -> torch.Tensor:
    _lib.require_cuda(x, "x")
    if x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] != 3:
        raise ValueError("x must be fp32 [N, 3] (z, y, x) in [0, 1]")
    return x.detach().contiguous()


def _model_forward(model: _HashGridModel, x: torch.Tensor, t) -> torch.Tensor:
    """sigma [N] = MLP(encode(x, t)) by nectb_model_forward(_t), no autograd."""
    x = _check_points(x)
    tv, td = _timestep(t)
    sigma = torch.empty(x.shape[0], device=x.device, dtype=torch.float32)
    args = (ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
            model.mlp.data_ptr(), x.data_ptr(), x.shape[0])
    if td is None:
        rc = _lib.lib.nectb_model_forward(*args, tv, sigma.data_ptr(), _lib.stream_ptr(x.device))
    else:
        rc = _lib.lib.nectb_model_forward_t(*args, td.data_ptr(), sigma.data_ptr(), _lib.stream_ptr(x.device))
    _lib.check(rc, "nectb_model_forward")
    return sigma


class ModelPoints(torch.autograd.Function):
    """sigma(x) [N] at points x [N, 3], differentiable in (table, mlp):
    forward nectb_model_forward, backward nectb_model_backward (fp32 SIMT for
    both table precisions; the gradient of the fp16 copy is the fp32
    table's).  This is the autograd node behind HashGrid.forward, for the
    reference's loss.backward() through model(points) (base_trainer.py:
    535-542, 650) and for losses on model outputs such as the total-variation
    term (base_trainer.py:615-649).  No gradient flows to x."""

    @staticmethod
    def forward(ctx, table, mlp, model, x, t):
        sigma = _model_forward(model, x, t)
        ctx.model, ctx.x, ctx.t = model, _check_points(x), _timestep(t)
        return sigma

    @staticmethod
    def backward(ctx, dsigma):
        model, x = ctx.model, ctx.x
        tv, td = ctx.t
        g = dsigma.detach().to(torch.float32).contiguous()
        tg, mg = torch.zeros_like(model.table), torch.zeros_like(model.mlp)
        args = (ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                model.mlp.data_ptr(), x.data_ptr(), x.shape[0])
        if td is None:
            rc = _lib.lib.nectb_model_backward(*args, tv, g.data_ptr(), tg.data_ptr(), mg.data_ptr(),
                                               _lib.stream_ptr(x.device))
        else:
            rc = _lib.lib.nectb_model_backward_t(*args, td.data_ptr(), g.data_ptr(), tg.data_ptr(), mg.data_ptr(),
                                                 _lib.stream_ptr(x.device))
        _lib.check(rc, "nectb_model_backward")
        return tg, mg, None, None, None


def model_points(model: _HashGridModel, x: torch.Tensor, t=0.0) -> torch.Tensor:
    """Differentiable sigma [n] of the model at points x [n, 3] ((z, y, x) in [0, 1])."""
    return ModelPoints.apply(model.table, model.mlp, model, x, t)
