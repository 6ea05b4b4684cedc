"""The reference's default dynamic model, QuadCubes (nect/network/networks.py:
392-449, preset nect/cfg/dynamic/quadcubes.yaml), and the training loop for
models the fused ray kernels do not cover.

QuadCubes encodes a point (z, y, x) at time t with four 3D hash grids of the
same configuration over (z, y, x), (y, x, t), (x, z, t) and (z, y, t) (the
reference's input order, networks.py:438-446), concatenates the four
encodings and, with ``include_identity``, the four raw inputs (z, y, x, t),
and runs a FullyFusedMLP without biases (default 4 hidden layers of 128,
LeakyReLU, no output activation).  Here:

- the grids are fp32 tables ``tables[k]`` [entries, features] in the
  library's layout, encoded together by ``nectb_quadcubes_encode`` straight
  into the MLP's input rows (bf16 on the mixed path) and differentiated by
  ``nectb_quadcubes_encode_backward`` (hand-written kernels, one autograd
  node); the three grids over (a, b, t) are evaluated on their plane at the
  call's t, 4 corners a level from an L2-sized blend of the two time
  vertices;
- the MLP is a chain of plain GEMMs (``torch.nn.Linear`` without bias, on
  cuBLAS; bf16 autocast when ``precision="mixed"``), weights Glorot-uniform,
  tables U(-1e-4, 1e-4) as for the hash-grid models.

``ModuleTrainer`` trains any such module the way the reference's loop does
(nect/trainers/base_trainer.py:517-568, 650-654): rays of a batch sampled by
the library's sampler, the clamp and the zero-point mask, the model on the
remaining points, the line integral sum(sigma) * distance / max_distance,
the loss, autograd, and the library's Adam kernel on every parameter.
"""
from __future__ import annotations

import ctypes
import math

import torch
import torch.nn as nn
import torch.nn.functional as F_

from . import _lib
from .config import HashEncoderConfig, MLPNetConfig
from .sampling import batching
from .sampling.ct_sampling import draw_ray_randoms, sample_with_draws
from .trainer import RayBatch, adam_step, projection_loss, reduce_gradients

# the reference's model-call chunk (base_trainer.py:523-551: at most 5 M points per call)
_CHUNK = 5_000_000


def _activation(name: str | None):
    key = (name or "None").replace("_", "").lower()
    table = {"none": lambda h: h, "relu": F_.relu, "leakyrelu": lambda h: F_.leaky_relu(h, 0.01),
             "softplus": F_.softplus, "sigmoid": torch.sigmoid}
    if key not in table:
        raise ValueError(f"activation {name!r} is not supported")
    return table[key]


class GridEncode(torch.autograd.Function):
    """Encoding [N, L * F] of points x [N, 3] by one 3D grid (nectb_hashgrid_encode);
    the backward adds the table gradient (nectb_hashgrid_encode_backward).  No
    gradient flows to x."""

    @staticmethod
    def forward(ctx, table, desc, n_out, x):
        n = x.shape[0]
        out = torch.empty(n, n_out, device=x.device, dtype=torch.float32)
        if n:
            rc = _lib.lib.nectb_hashgrid_encode(ctypes.byref(desc), table.data_ptr(), x.data_ptr(), n,
                                                out.data_ptr(), _lib.stream_ptr(x.device))
            _lib.check(rc, "nectb_hashgrid_encode")
        ctx.desc = desc
        ctx.save_for_backward(x)
        ctx.table_shape = table.shape
        return out

    @staticmethod
    def backward(ctx, dout):
        (x,) = ctx.saved_tensors
        grad = torch.zeros(ctx.table_shape, device=x.device, dtype=torch.float32)
        if x.shape[0]:
            g = dout.detach().to(torch.float32).contiguous()
            rc = _lib.lib.nectb_hashgrid_encode_backward(ctypes.byref(ctx.desc), x.data_ptr(), x.shape[0],
                                                         g.data_ptr(), grad.data_ptr(), _lib.stream_ptr(x.device))
            _lib.check(rc, "nectb_hashgrid_encode_backward")
        return grad, None, None, None


class QuadEncode(torch.autograd.Function):
    """The composite encoding of QuadCubes in one node: rows [N, ld] (fp32, or
    bf16 on the mixed path) holding the four grids' features, the raw inputs
    (z, y, x, t) with ``include_identity`` and zero columns up to ld
    (nectb_quadcubes_encode); the backward adds the four table gradients
    (nectb_quadcubes_encode_backward).  t is a 1-element fp32 CUDA tensor.  No
    gradient flows to zyx or t."""

    @staticmethod
    def forward(ctx, t0, t1, t2, t3, model, zyx, t):
        n = zyx.shape[0]
        dtype = torch.bfloat16 if model.precision == "mixed" else torch.float32
        out = torch.empty(n, model.row_width, device=zyx.device, dtype=dtype)
        if n:
            ws = torch.empty(model.workspace_bytes, device=zyx.device, dtype=torch.uint8)
            ptrs = (ctypes.c_void_p * 4)(*[tab.data_ptr() for tab in (t0, t1, t2, t3)])
            rc = _lib.lib.nectb_quadcubes_encode(
                ctypes.byref(model.desc), ptrs, zyx.data_ptr(), n, t.data_ptr(), int(model.include_identity),
                out.data_ptr(), model.row_width, _lib.BF16 if dtype == torch.bfloat16 else _lib.F32, ws.data_ptr(),
                ws.numel(), _lib.stream_ptr(zyx.device))
            _lib.check(rc, "nectb_quadcubes_encode")
        ctx.model = model
        ctx.save_for_backward(zyx, t)
        return out

    @staticmethod
    def backward(ctx, dout):
        zyx, t = ctx.saved_tensors
        model = ctx.model
        grads = [torch.zeros_like(tab) for tab in model.tables]
        if zyx.shape[0]:
            d = dout.detach()
            if d.dtype not in (torch.float32, torch.bfloat16):
                d = d.float()
            d = d.contiguous()
            ws = torch.empty(model.workspace_bytes, device=zyx.device, dtype=torch.uint8)
            ptrs = (ctypes.c_void_p * 4)(*[g.data_ptr() for g in grads])
            rc = _lib.lib.nectb_quadcubes_encode_backward(
                ctypes.byref(model.desc), zyx.data_ptr(), zyx.shape[0], t.data_ptr(), d.data_ptr(), d.shape[1],
                _lib.BF16 if d.dtype == torch.bfloat16 else _lib.F32, ptrs, ws.data_ptr(), ws.numel(),
                _lib.stream_ptr(zyx.device))
            _lib.check(rc, "nectb_quadcubes_encode_backward")
        return (*grads, None, None, None)


class QuadCubes(nn.Module):
    """forward(zyx [N, 3], t) -> sigma [N, 1] (networks.py:438-449)."""
    n_dims = 4

    def __init__(self, encoding_config: HashEncoderConfig, network_config: MLPNetConfig, prior: bool = False,
                 concat: bool = True, precision: str = "plain_fp32", device="cuda", seed: int = 1337):
        super().__init__()
        if prior:
            raise NotImplementedError("QuadCubes with a prior model is not supported")
        if not concat:
            raise NotImplementedError("QuadCubes with multiplied encodings is not supported")
        enc, net = encoding_config, network_config
        self.encoding_config, self.network_config, self.precision = enc, net, precision
        self.include_identity = bool(net.include_identity)
        self.desc = _lib.NectbHashGrid(n_dims=3, n_levels=enc.n_levels, n_features=enc.n_features_per_level,
                                       log2_hashmap_size=enc.log2_hashmap_size, feature_dtype=_lib.F32,
                                       base_resolution=float(enc.base_resolution),
                                       per_level_scale=float(enc.per_level_scale), base_resolution_t=0.0)
        L = enc.n_levels
        buf = [(ctypes.c_int32 * L)(), (ctypes.c_int32 * L)(), (ctypes.c_int64 * L)(), (ctypes.c_int64 * L)(),
               (ctypes.c_int32 * L)()]
        total = _lib.lib.nectb_hashgrid_layout(ctypes.byref(self.desc), *[ctypes.addressof(b) for b in buf])
        if total <= 0:
            raise ValueError("invalid hash-grid configuration")
        self.n_enc = L * enc.n_features_per_level
        self.n_in = 4 * self.n_enc + (4 if self.include_identity else 0)
        # rows of the encoding matrix: 16-byte aligned (fp32), or a multiple of
        # 64 bf16 columns on the mixed path (aligned GEMM tiles); the padded
        # columns are zero and meet zero weight columns
        self.row_width = -(-self.n_in // 64) * 64 if precision == "mixed" else -(-self.n_in // 4) * 4
        self.workspace_bytes = int(_lib.lib.nectb_quadcubes_workspace_bytes(ctypes.byref(self.desc)))
        if self.workspace_bytes <= 0:
            raise ValueError("invalid QuadCubes grid configuration")
        gen = torch.Generator(device="cpu").manual_seed(seed)
        self.tables = nn.ParameterList([
            nn.Parameter(((torch.rand(total, enc.n_features_per_level, generator=gen) * 2 - 1) * 1e-4).to(device))
            for _ in range(4)])
        widths = [self.n_in] + [net.n_neurons] * net.n_hidden_layers + [1]
        self.layers = nn.ModuleList()
        for a, b in zip(widths[:-1], widths[1:]):
            lin = nn.Linear(a, b, bias=False)
            bound = math.sqrt(6.0 / (a + b))
            with torch.no_grad():
                lin.weight.copy_((torch.rand(b, a, generator=gen) * 2 - 1) * bound)
            self.layers.append(lin.to(device))
        self.act = _activation(net.activation)
        self.out_act = _activation(net.output_activation)

    def forward(self, zyx: torch.Tensor, t) -> torch.Tensor:
        _lib.require_cuda(zyx, "zyx")
        if zyx.dtype != torch.float32 or zyx.dim() != 2 or zyx.shape[1] != 3:
            raise ValueError("zyx must be fp32 [N, 3] (z, y, x) in [0, 1]")
        x = zyx.detach().contiguous()
        if isinstance(t, torch.Tensor):   # stays on the device (no host sync)
            tdev = t.detach().to(device=x.device, dtype=torch.float32).reshape(1).contiguous()
        else:
            tdev = torch.full((1,), float(t), device=x.device, dtype=torch.float32)
        h = QuadEncode.apply(*self.tables, self, x, tdev)
        w0 = self.layers[0].weight
        if self.row_width != self.n_in:
            w0 = F_.pad(w0, (0, self.row_width - self.n_in))
        with torch.autocast("cuda", dtype=torch.bfloat16, enabled=self.precision == "mixed"):
            h = self.act(F_.linear(h, w0))
            for lin in self.layers[1:-1]:
                h = self.act(lin(h))
            out = self.layers[-1](h)
        return self.out_act(out.float())

    @torch.no_grad()
    def volume(self, shape, t, scale: float = 1.0, offset: float = 0.0) -> torch.Tensor:
        """sigma * scale + offset on the voxel-centre grid [z, y, x] (create_volume, base_trainer.py:402-450)."""
        dev = self.tables[0].device
        nz, ny, nx = shape
        c = [(torch.arange(k, device=dev, dtype=torch.float32) + 0.5) / k for k in (nz, ny, nx)]
        yy, xx = torch.meshgrid(c[1], c[2], indexing="ij")
        out = torch.empty(shape, device=dev)
        per = max(1, _CHUNK // (ny * nx))
        for z0 in range(0, nz, per):
            zs = c[0][z0:z0 + per]
            pts = torch.stack([zs[:, None, None].expand(-1, ny, nx), yy.expand(len(zs), -1, -1),
                               xx.expand(len(zs), -1, -1)], -1).reshape(-1, 3)
            out[z0:z0 + per] = (self(pts, t).reshape(len(zs), ny, nx) * scale + offset)
        return out


def module_ray_integral(model: nn.Module, points: torch.Tensor, distances: torch.Tensor, t,
                        max_distance_traveled: float) -> torch.Tensor:
    """y_pred [R] = sum over a ray's non-zero points of model(point, t) *
    distance / max_distance_traveled (base_trainer.py:523-554): points
    [R, S, 3] clamped to [0, 1] (projector.py:127), zero points dropped,
    model calls of at most 5 M points."""
    R, S, _ = points.shape
    flat = points.clamp_(0.0, 1.0).reshape(-1, 3)
    keep = torch.nonzero((flat != 0).any(1)).squeeze(1)
    sigma = torch.zeros(R * S, device=points.device, dtype=torch.float32)
    parts = [model(flat[keep[i:i + _CHUNK]], t).squeeze(1) for i in range(0, keep.numel(), _CHUNK)]
    if parts:
        sigma = sigma.index_put((keep,), torch.cat(parts))
    return sigma.view(R, S).sum(1) * distances / max_distance_traveled


class ModuleTrainer:
    """The reference's training step for a module the fused kernels do not
    cover, with the fused Trainer's interface (make_batch, step, split_step,
    train_projection, optimizer_moments) so that fit() drives either."""

    def __init__(self, model: nn.Module, geometry, points_per_batch: int, points_per_ray: int, loss: str = "l2",
                 lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0,
                 batch_per_proj: int = 1, random_offset_detector: float = 0.0, uniform_ray_spacing: bool = True,
                 device="cuda", data_parallel: bool = False, process_group=None, clip_grad_value: float | None = None):
        self.model = model
        self.geometry = geometry
        self.c_geometry = geometry.get_c_geometry()
        self.device = torch.device(device)
        self.points_per_batch = points_per_batch
        self.points_per_ray = points_per_ray
        self.loss = loss
        self.lr, self.betas, self.eps, self.weight_decay = lr, betas, eps, weight_decay
        self.batch_per_proj = batch_per_proj
        self.random_offset_detector = random_offset_detector
        self.uniform_ray_spacing = uniform_ray_spacing
        self.data_parallel, self.process_group = data_parallel, process_group
        self.clip_grad_value = clip_grad_value
        self.step_count = 0
        self.params = [p for p in model.parameters()]
        self.moments = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.params]

    @property
    def batch_size(self) -> int:
        return batching.rays_per_batch(self.points_per_batch, self.points_per_ray)

    def make_batch(self, perm: torch.Tensor, batch_num: int, angle: float, projection: torch.Tensor,
                   t: float = 0.0) -> RayBatch | None:
        window = batching.batch_window(perm.numel(), self.batch_size, batch_num)
        if window is None:
            return None
        start, size = window
        jitter, det_off = draw_ray_randoms(size, self.random_offset_detector, self.device)
        return RayBatch(perm=perm, start=start, num_rays=size, points_per_ray=self.points_per_ray, angle=angle,
                        max_ray_distance_per_point=self.geometry.max_distance_traveled / self.points_per_ray,
                        jitter=jitter, detector_offset=det_off, projection=projection, t=t,
                        uniform_ray_spacing=self.uniform_ray_spacing)

    def ray_integral(self, batch: RayBatch) -> torch.Tensor:
        points, distances = sample_with_draws(batch.perm, self.c_geometry, batch.angle, batch.points_per_ray,
                                              batch.num_rays, batch.start, batch.max_ray_distance_per_point,
                                              batch.uniform_ray_spacing, batch.jitter, batch.detector_offset)
        return module_ray_integral(self.model, points, distances, batch.t, self.geometry.max_distance_traveled)

    def step(self, batch: RayBatch) -> torch.Tensor:
        return self.split_step(batch)

    def split_step(self, batch: RayBatch, add_poisson: bool = False, s3im_patch: int = 0, tv_weight: float = 0.0,
                   tv_origin=None) -> torch.Tensor:
        if tv_weight > 0:
            raise NotImplementedError("the total-variation term applies to static models")
        y_pred = self.ray_integral(batch)
        y = batch.projection[batch.perm[batch.start:batch.start + batch.num_rays]]
        if add_poisson:   # base_trainer.py:555-556; the Poisson draw carries no gradient
            y_pred = (y_pred + torch.poisson(y_pred.detach() * 1e5) / 1e5) / 2
        loss = projection_loss(y_pred, y, self.loss)
        if s3im_patch:
            from .schedule import s3im_loss

            loss = loss + s3im_loss(y_pred, y, s3im_patch)
        grads = [g.contiguous() for g in torch.autograd.grad(loss, self.params)]
        self._update(grads)
        return loss.detach()

    def _update(self, grads) -> None:
        self.step_count += 1
        if self.data_parallel:
            reduce_gradients(grads, self.process_group)
        for p, g, (m, v) in zip(self.params, grads, self.moments):
            if self.clip_grad_value is not None:
                g.clamp_(-self.clip_grad_value, self.clip_grad_value)
            adam_step(p.data, g, m, v, self.step_count, self.lr, self.betas, self.eps, self.weight_decay)

    def train_projection(self, projection: torch.Tensor, angle: float, t: float = 0.0) -> torch.Tensor | None:
        P = projection.numel()
        perm = torch.randperm(P, dtype=torch.int64, device=self.device)
        loss = None
        for b in range(min(self.batch_per_proj, batching.batches_per_projection(P, self.batch_size))):
            batch = self.make_batch(perm, b, angle, projection, t)
            if batch is not None:
                loss = self.step(batch)
        return loss

    def optimizer_moments(self):
        return list(self.moments)

    @torch.no_grad()
    def load_optimizer_moments(self, moments) -> None:
        for (dm, dv), (m, v) in zip(self.moments, moments):
            dm.copy_(m)
            dv.copy_(v)

    def device_error(self) -> int:
        return 0
