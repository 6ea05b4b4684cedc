"""Fused training: one CUDA pipeline per batch of rays instead of the
reference's sample -> mask -> model -> sum -> loss -> backward sequence
(nect/trainers/base_trainer.py:517-653).

* ``train_step`` calls ``nectb_train_step`` once: it regenerates the samples of
  every ray (bit-identical to the sampler), encodes, runs the MLP, integrates
  along the ray, evaluates the L1/L2 loss and ADDS the gradients of the table
  and the MLP into fp32 buffers.
* ``FusedRayLoss`` wraps it as a torch.autograd.Function (the hand-written
  backward: gradients are computed in the same fused pass and returned scaled
  by the incoming gradient), so a standard torch optimizer works.
* ``Trainer`` reproduces the per-projection loop (randperm of the detector,
  ``batch_per_proj`` batches, Adam) with a fused Adam kernel that also
  refreshes the fp16 table on the mixed path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from .network import ModelPoints, _HashGridModel, model_points  # noqa: F401
from .sampling import batching
from .sampling.ct_sampling import draw_ray_randoms
from .sampling.geometry import Geometry

LOSS = {"l1": 1, "l2": 2}


def loss_kind(loss: str) -> str:
    """The reference's loss selection (nect/config.py:481-497): "l1" when the
    name contains l1 (so "L1+L2" is L1, its alternating branch being
    unreachable there), else "l2" when it contains l2; other names raise
    NotImplementedError."""
    name = loss.casefold()
    if "l1" in name:
        return "l1"
    if "l2" in name:
        return "l2"
    raise NotImplementedError(f"Loss {loss} is not supported")


@dataclass
class RayBatch:
    """One batch of rays of one projection (Projector.__call__ arguments)."""
    perm: torch.Tensor            # int64 [P] randperm of detector pixels
    start: int                    # starting_ray_index
    num_rays: int
    points_per_ray: int
    angle: float
    max_ray_distance_per_point: float
    jitter: torch.Tensor          # [R]
    detector_offset: torch.Tensor # [R, 2]
    projection: torch.Tensor      # fp32 [P] flattened projection (min-max scaled)
    t: float = 0.0
    uniform_ray_spacing: bool = True


class Workspace:
    """Caller-owned device workspace for nectb_train_step, grown on demand.

    With ``staging`` (default) it also holds the recommended staging buffer of
    the mixed path's two-pass backward (ray order, the encoding store and one
    round of staged gradients); without it the mixed backward runs as one
    fused pass.  ``staging_fraction`` < 1 takes that share of the
    recommendation: the library then keeps fewer rows in the encoding store
    (rays beyond it gather again), then none, then runs more rounds; results
    do not change."""

    def __init__(self, staging: bool = True, staging_fraction: float = 1.0):
        self.buf = None
        self.staging = staging
        self.staging_fraction = staging_fraction

    def get(self, model: _HashGridModel, c_geometry, num_rays: int, device,
            points_per_ray: int = 0, sub_angles: int = 1) -> tuple[int, int]:
        """(pointer, bytes) of a workspace for a batch of num_rays rays (a
        continuous-scan batch of sub_angles sub-angles when sub_angles > 1)."""
        args = (ctypes.byref(c_geometry.c_struct), ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc))
        if sub_angles > 1:
            need = _lib.lib.nectb_train_scan_workspace_bytes(*args, num_rays, sub_angles)
        else:
            need = _lib.lib.nectb_train_workspace_bytes(*args, num_rays)
        if self.staging and points_per_ray > 0:
            staging = (_lib.lib.nectb_train_scan_staging_bytes(*args, num_rays, points_per_ray, sub_angles)
                       if sub_angles > 1 else _lib.lib.nectb_train_staging_bytes(*args, num_rays, points_per_ray))
            need = ((need + 255) // 256) * 256 + int(self.staging_fraction * staging)
        if self.buf is None or self.buf.numel() < need or self.buf.device != torch.device(device):
            self.buf = torch.empty(need, dtype=torch.uint8, device=device)
        self.num_rays = num_rays
        self.sub_angles = sub_angles
        self.c_geometry = c_geometry
        return self.buf.data_ptr(), self.buf.numel()

    def error_word(self, c_geometry=None) -> int:
        """The device error word of the last step run in this workspace (0 = every
        tensor-core wait completed).  Synchronises the current stream."""
        cg = c_geometry if c_geometry is not None else self.c_geometry
        if getattr(self, "sub_angles", 1) > 1:
            addr = _lib.lib.nectb_train_scan_error_word(ctypes.byref(cg.c_struct), int(self.num_rays),
                                                        int(self.sub_angles), self.buf.data_ptr())
        else:
            addr = _lib.lib.nectb_train_error_word(ctypes.byref(cg.c_struct), int(self.num_rays), self.buf.data_ptr())
        if not addr:
            raise RuntimeError("nectb_train_error_word: " + _lib.lib.nectb_last_error().decode())
        off = addr - self.buf.data_ptr()
        return int(self.buf[off:off + 4].view(torch.int32).item())


def c_batch(batch: RayBatch, max_distance_traveled: float, loss: str, loss_scale: float = 1.0):
    b = _lib.NectbTrainBatch()
    b.random_ray_index = batch.perm.data_ptr()
    b.random_ray_index_len = batch.perm.numel()
    b.starting_ray_index = int(batch.start)
    b.num_rays = int(batch.num_rays)
    b.num_points_per_ray = int(batch.points_per_ray)
    b.angle_rad = float(batch.angle)
    b.t = float(batch.t)
    b.max_ray_distance_per_point = float(batch.max_ray_distance_per_point)
    b.uniform_ray_spacing = 1 if batch.uniform_ray_spacing else 0
    b.max_distance_traveled = float(max_distance_traveled)
    b.jitter = batch.jitter.data_ptr()
    b.detector_offset = batch.detector_offset.data_ptr()
    b.projection = batch.projection.data_ptr()
    b.loss_type = LOSS[loss_kind(loss)]
    b.loss_scale = float(loss_scale)
    return b


def train_step(model: _HashGridModel, c_geometry, batch: RayBatch, max_distance_traveled: float,
               table_grad: torch.Tensor, mlp_grad: torch.Tensor, workspace: Workspace, loss: str = "l2",
               loss_scale: float = 1.0):
    """Fused forward+backward; gradients are ADDED to table_grad / mlp_grad.

    Returns (loss [1] device tensor, y_pred [R])."""
    dev = batch.perm.device
    for name, t in (("perm", batch.perm), ("jitter", batch.jitter), ("detector_offset", batch.detector_offset),
                    ("projection", batch.projection)):
        _lib.require_cuda(t, name)
    y_pred = torch.empty(batch.num_rays, device=dev, dtype=torch.float32)
    loss_out = torch.empty(1, device=dev, dtype=torch.float32)
    ws_ptr, ws_size = workspace.get(model, c_geometry, batch.num_rays, dev, batch.points_per_ray)
    cb = c_batch(batch, max_distance_traveled, loss, loss_scale)
    rc = _lib.lib.nectb_train_step(ctypes.byref(c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                   ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(), model.mlp.data_ptr(),
                                   ctypes.byref(cb), table_grad.data_ptr(), mlp_grad.data_ptr(), y_pred.data_ptr(),
                                   loss_out.data_ptr(), ws_ptr, ws_size, _lib.stream_ptr(dev))
    _lib.check(rc, "nectb_train_step")
    return loss_out, y_pred


class RayIntegral(torch.autograd.Function):
    """y_pred[r] = (sum of sigma over ray r's samples) * distances / max_distance_traveled
    (base_trainer.py:552-554) as a function of (table, mlp): forward half
    nectb_train_forward, backward half nectb_train_backward with the
    incoming dL/dy_pred.  Any torch loss of y_pred may follow (L1/L2, Poisson
    noise, S3IM, sub-angle averages), as in the reference's composition
    (base_trainer.py:552-566).  The workspace passed in belongs to this
    forward until its backward has run."""

    @staticmethod
    def forward(ctx, table, mlp, model, c_geometry, batch, max_distance_traveled, workspace):
        dev = batch.perm.device
        for name, t in (("perm", batch.perm), ("jitter", batch.jitter), ("detector_offset", batch.detector_offset),
                        ("projection", batch.projection)):
            _lib.require_cuda(t, name)
        y_pred = torch.empty(batch.num_rays, device=dev, dtype=torch.float32)
        ws_ptr, ws_size = workspace.get(model, c_geometry, batch.num_rays, dev, batch.points_per_ray)
        cb = c_batch(batch, max_distance_traveled, "l2")
        rc = _lib.lib.nectb_train_forward(ctypes.byref(c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                          ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                          model.mlp.data_ptr(), ctypes.byref(cb), y_pred.data_ptr(), ws_ptr, ws_size,
                                          _lib.stream_ptr(dev))
        _lib.check(rc, "nectb_train_forward")
        # everything the backward half reads: the batch's tensors, the C batch and this workspace buffer
        ctx.model, ctx.c_geometry, ctx.batch, ctx.cb = model, c_geometry, batch, cb
        ctx.ws_buf, ctx.ws = workspace.buf, (ws_ptr, ws_size)
        return y_pred

    @staticmethod
    def backward(ctx, grad_y):
        model, dev = ctx.model, ctx.batch.perm.device
        g = grad_y.detach().to(torch.float32).contiguous()
        tg = torch.zeros_like(model.table)
        mg = torch.zeros_like(model.mlp)
        rc = _lib.lib.nectb_train_backward(ctypes.byref(ctx.c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                           ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                           model.mlp.data_ptr(), ctypes.byref(ctx.cb), g.data_ptr(), tg.data_ptr(),
                                           mg.data_ptr(), ctx.ws[0], ctx.ws[1], _lib.stream_ptr(dev))
        _lib.check(rc, "nectb_train_backward")
        return tg, mg, None, None, None, None, None


def ray_integral(model: _HashGridModel, c_geometry, batch: RayBatch, max_distance_traveled: float,
                 workspace: Workspace) -> torch.Tensor:
    """Differentiable y_pred [R] of one batch (see RayIntegral)."""
    return RayIntegral.apply(model.table, model.mlp, model, c_geometry, batch, max_distance_traveled, workspace)


class ScanIntegral(torch.autograd.Function):
    """The continuous-scan prediction y_pred[r] = mean over the sub angles of
    pixel r's line integral (continous_scanning_trainer.py:85-137) as a
    function of (table, mlp), all sub-angle rays in one launch of each fused
    kernel: forward nectb_train_scan_forward, backward
    nectb_train_scan_backward.  ``batch`` carries sub_angles * R jitter and
    detector-offset draws (sub-angle-major); its angle is ignored."""

    @staticmethod
    def forward(ctx, table, mlp, model, c_geometry, batch, sub_angles, max_distance_traveled, workspace):
        dev = batch.perm.device
        k = len(sub_angles)
        for name, t in (("perm", batch.perm), ("jitter", batch.jitter), ("detector_offset", batch.detector_offset),
                        ("projection", batch.projection)):
            _lib.require_cuda(t, name)
        if batch.jitter.numel() != k * batch.num_rays or batch.detector_offset.numel() != 2 * k * batch.num_rays:
            raise ValueError("a continuous-scan batch needs sub_angles * num_rays jitter and offset draws")
        angles = (ctypes.c_float * k)(*[float(a) for a in sub_angles])
        y_pred = torch.empty(batch.num_rays, device=dev, dtype=torch.float32)
        ws_ptr, ws_size = workspace.get(model, c_geometry, batch.num_rays, dev, batch.points_per_ray, k)
        cb = c_batch(batch, max_distance_traveled, "l2")
        rc = _lib.lib.nectb_train_scan_forward(ctypes.byref(c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                               ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                               model.mlp.data_ptr(), ctypes.byref(cb), angles, k, y_pred.data_ptr(),
                                               ws_ptr, ws_size, _lib.stream_ptr(dev))
        _lib.check(rc, "nectb_train_scan_forward")
        ctx.model, ctx.c_geometry, ctx.batch, ctx.cb, ctx.angles, ctx.k = model, c_geometry, batch, cb, angles, k
        ctx.ws_buf, ctx.ws = workspace.buf, (ws_ptr, ws_size)
        return y_pred

    @staticmethod
    def backward(ctx, grad_y):
        model, dev = ctx.model, ctx.batch.perm.device
        g = grad_y.detach().to(torch.float32).contiguous()
        tg = torch.zeros_like(model.table)
        mg = torch.zeros_like(model.mlp)
        rc = _lib.lib.nectb_train_scan_backward(ctypes.byref(ctx.c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                                ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                                model.mlp.data_ptr(), ctypes.byref(ctx.cb), ctx.angles, ctx.k,
                                                g.data_ptr(), tg.data_ptr(), mg.data_ptr(), ctx.ws[0], ctx.ws[1],
                                                _lib.stream_ptr(dev))
        _lib.check(rc, "nectb_train_scan_backward")
        return tg, mg, None, None, None, None, None, None


def scan_integral(model: _HashGridModel, c_geometry, batch: RayBatch, sub_angles, max_distance_traveled: float,
                  workspace: Workspace) -> torch.Tensor:
    """Differentiable continuous-scan y_pred [R] of one batch (see ScanIntegral)."""
    return ScanIntegral.apply(model.table, model.mlp, model, c_geometry, batch, list(sub_angles),
                              max_distance_traveled, workspace)


def scan_step(model: _HashGridModel, c_geometry, batch: RayBatch, sub_angles, max_distance_traveled: float,
              table_grad: torch.Tensor, mlp_grad: torch.Tensor, workspace: Workspace, loss: str = "l2",
              loss_scale: float = 1.0):
    """The fused continuous-scan step with the built-in L1/L2 loss
    (nectb_train_scan_step); gradients are ADDED.  Returns (loss [1], y_pred [R])."""
    dev = batch.perm.device
    k = len(sub_angles)
    angles = (ctypes.c_float * k)(*[float(a) for a in sub_angles])
    y_pred = torch.empty(batch.num_rays, device=dev, dtype=torch.float32)
    loss_out = torch.empty(1, device=dev, dtype=torch.float32)
    ws_ptr, ws_size = workspace.get(model, c_geometry, batch.num_rays, dev, batch.points_per_ray, k)
    cb = c_batch(batch, max_distance_traveled, loss, loss_scale)
    rc = _lib.lib.nectb_train_scan_step(ctypes.byref(c_geometry.c_struct), ctypes.byref(model.grid_desc),
                                        ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                        model.mlp.data_ptr(), ctypes.byref(cb), angles, k, table_grad.data_ptr(),
                                        mlp_grad.data_ptr(), y_pred.data_ptr(), loss_out.data_ptr(), ws_ptr, ws_size,
                                        _lib.stream_ptr(dev))
    _lib.check(rc, "nectb_train_scan_step")
    return loss_out, y_pred


def total_variation_3d(volume: torch.Tensor, weight: float = 1.0) -> torch.Tensor:
    """Sum of absolute neighbour differences along the three axes over the
    voxel count, times weight (nect/utils.py:64-80)."""
    di = (volume[1:] - volume[:-1]).abs().sum()
    dj = (volume[:, 1:] - volume[:, :-1]).abs().sum()
    dk = (volume[:, :, 1:] - volume[:, :, :-1]).abs().sum()
    return (di + dj + dk) / (volume.shape[0] * volume.shape[1] * volume.shape[2]) * weight


def tv_points(origin, n: int = 100, extent: float = 0.2, device="cuda") -> torch.Tensor:
    """The n^3 grid [origin, origin + extent] per axis, (z, y, x) order, as
    base_trainer.py:620-640 builds it for the total-variation term."""
    axes = [torch.linspace(float(o), float(o) + extent, n, device=device) for o in origin]
    z, y, x = torch.meshgrid(axes, indexing="ij")
    return torch.stack((z.flatten(), y.flatten(), x.flatten()), 1)


def projection_loss(y_pred: torch.Tensor, y: torch.Tensor, loss: str) -> torch.Tensor:
    """L1 or L2 (mean over rays), nect/config.py:481-497 (loss_kind)."""
    if loss_kind(loss) == "l1":
        return torch.nn.functional.l1_loss(y_pred, y)
    return torch.nn.functional.mse_loss(y_pred, y)


class FusedRayLoss(torch.autograd.Function):
    """loss = L(y_pred(table, mlp), y) with the hand-written fused backward."""

    @staticmethod
    def forward(ctx, table, mlp, model, c_geometry, batch, max_distance_traveled, loss, workspace):
        tg = torch.zeros_like(table)
        mg = torch.zeros_like(mlp)
        out, _ = train_step(model, c_geometry, batch, max_distance_traveled, tg, mg, workspace, loss)
        ctx.save_for_backward(tg, mg)
        return out[0]

    @staticmethod
    def backward(ctx, grad_out):
        tg, mg = ctx.saved_tensors
        return tg * grad_out, mg * grad_out, None, None, None, None, None, None


def adam_step(param: torch.Tensor, grad: torch.Tensor, m: torch.Tensor, v: torch.Tensor, step: int, lr: float,
              betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0, half: torch.Tensor | None = None,
              zero_grad: bool = True):
    n = param.numel()
    if grad.numel() != n or m.numel() != n or v.numel() != n or (half is not None and half.numel() != n):
        raise ValueError(f"adam_step: parameter, gradient and moments differ in size ({n}, {grad.numel()}, "
                         f"{m.numel()}, {v.numel()})")
    rc = _lib.lib.nectb_adam_step(param.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), param.numel(),
                                  float(lr), float(betas[0]), float(betas[1]), float(eps), float(weight_decay),
                                  int(step), half.data_ptr() if half is not None else None, 1 if zero_grad else 0,
                                  _lib.stream_ptr(param.device))
    _lib.check(rc, "nectb_adam_step")


def reduce_gradients(grads, group=None) -> None:
    """Average gradients over the ranks of ``group`` in place, as the
    reference's Fabric DDP does (base_trainer.py:106-112): one all-reduce per
    gradient tensor (the table gradient is one contiguous buffer; NCCL over
    NVLink/NVSwitch on GPUs), then division by the world size."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return
    world = dist.get_world_size(group)
    if world == 1:
        return
    for g in grads:
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
        g.div_(world)


class ShardedAdam:
    """Data-parallel Adam with the optimizer state sharded over the ranks.

    The reference averages gradients with one DDP all-reduce and runs the full
    Adam step on every rank (base_trainer.py:106-112).  Here each parameter
    buffer is cut into ``world`` contiguous shards of ``chunk`` elements (the
    last padded):

    1. the gradient buffer (padded, ``world * chunk``) is reduce-scattered, so
       rank r receives the summed shard r, which is divided by the world size;
    2. rank r runs Adam on shard r only, with moments held for that shard;
    3. the updated shards are all-gathered into every rank's parameters (and
       the fp16 table copy refreshed from them).

    The collectives move the bytes of one all-reduce; Adam's HBM traffic and
    the moment memory per rank fall by the world size.  Results equal the
    all-reduce step's: the sums are the same per element and Adam is
    elementwise.  ``adam`` is the update applied to each shard (the CUDA
    kernel behind ``adam_step`` unless a caller passes another)."""

    ALIGN = 8  # shard starts on 32-byte boundaries

    def __init__(self, params, group=None, adam=None):
        import torch.distributed as dist

        if not dist.is_available() or not dist.is_initialized():
            raise RuntimeError("ShardedAdam needs an initialised torch.distributed process group")
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.params = list(params)
        self.adam = adam or adam_step
        self.shards = []  # (n, chunk, lo, valid)
        self.grad_pad, self.grads, self.shard_grad, self.m, self.v, self.send, self.gathered = ([] for _ in range(7))
        for p in self.params:
            n = p.numel()
            chunk = -(-n // self.world)
            chunk = -(-chunk // self.ALIGN) * self.ALIGN
            lo = self.rank * chunk
            valid = max(0, min(n - lo, chunk))
            self.shards.append((n, chunk, lo, valid))
            gp = torch.zeros(self.world * chunk, dtype=p.dtype, device=p.device)
            self.grad_pad.append(gp)
            self.grads.append(gp[:n].view_as(p))
            self.shard_grad.append(torch.zeros(chunk, dtype=p.dtype, device=p.device))
            self.m.append(torch.zeros(chunk, dtype=p.dtype, device=p.device))
            self.v.append(torch.zeros(chunk, dtype=p.dtype, device=p.device))
            self.send.append(torch.zeros(chunk, dtype=p.dtype, device=p.device))
            # the all-gather lands in the parameter itself unless the buffer pads
            padded = self.world * chunk != n
            self.gathered.append(torch.empty(self.world * chunk, dtype=p.dtype, device=p.device) if padded else None)

    @torch.no_grad()
    def step(self, step: int, lr: float, betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0,
             halves=None, clip: float | None = None) -> None:
        """One update from the gradients accumulated in ``self.grads`` (zeroed
        afterwards).  ``halves[i]``, when given, is an fp16 copy of params[i]
        that is rewritten from the updated parameters; ``clip`` clamps the
        averaged gradients to [-clip, clip]."""
        import torch.distributed as dist

        halves = halves or [None] * len(self.params)
        for i, p in enumerate(self.params):
            n, chunk, lo, valid = self.shards[i]
            dist.reduce_scatter_tensor(self.shard_grad[i], self.grad_pad[i], op=dist.ReduceOp.SUM, group=self.group)
            self.shard_grad[i].div_(self.world)
            if clip is not None:
                self.shard_grad[i].clamp_(-clip, clip)
            self.grad_pad[i].zero_()
            flat = p.view(-1)
            if valid > 0:
                self.adam(flat[lo:lo + valid], self.shard_grad[i][:valid], self.m[i][:valid], self.v[i][:valid],
                          step, lr, betas, eps, weight_decay)
                self.send[i][:valid].copy_(flat[lo:lo + valid])
            if self.gathered[i] is None:
                dist.all_gather_into_tensor(flat, self.send[i], group=self.group)
            else:
                dist.all_gather_into_tensor(self.gathered[i], self.send[i], group=self.group)
                flat.copy_(self.gathered[i][:n])
            if halves[i] is not None:
                halves[i].view(-1).copy_(flat)

    @torch.no_grad()
    def full_moments(self, i: int):
        """(exp_avg, exp_avg_sq) of params[i] at full size on every rank (a
        collective: all ranks call it)."""
        import torch.distributed as dist

        n = self.shards[i][0]
        out = []
        for s in (self.m[i], self.v[i]):
            full = torch.empty(self.world * s.numel(), dtype=s.dtype, device=s.device)
            dist.all_gather_into_tensor(full, s.contiguous(), group=self.group)
            out.append(full[:n].view_as(self.params[i]))
        return tuple(out)

    @torch.no_grad()
    def load_moments(self, i: int, exp_avg: torch.Tensor, exp_avg_sq: torch.Tensor) -> None:
        """Take this rank's shard of full-size moments of params[i]."""
        n, chunk, lo, valid = self.shards[i]
        for dst, src in ((self.m[i], exp_avg), (self.v[i], exp_avg_sq)):
            dst.zero_()
            if valid > 0:
                dst[:valid].copy_(src.reshape(-1)[lo:lo + valid])


class Trainer:
    """Per-projection training loop on the fused kernels.

    Mirrors BaseTrainer.fit's inner structure (base_trainer.py:492-655): for each
    projection a device randperm of the detector pixels, up to ``batch_per_proj``
    batches of ``points_per_batch // points_per_ray`` rays, each followed by an
    Adam step (lr fixed unless a schedule is passed)."""

    def __init__(self, model: _HashGridModel, geometry: Geometry, points_per_batch: int, points_per_ray: int,
                 loss: str = "l2", lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8,
                 weight_decay: float = 0.0, batch_per_proj: int = 1, random_offset_detector: float = 0.0,
                 uniform_ray_spacing: bool = True, device="cuda", data_parallel: bool = False, process_group=None,
                 shard_optimizer: bool = False, clip_grad_value: float | None = None):
        self.model = model
        self.geometry = geometry
        self.c_geometry = geometry.get_c_geometry()
        self.device = torch.device(device)
        self.points_per_batch = points_per_batch
        self.points_per_ray = points_per_ray
        self.loss = loss
        self.lr = lr
        self.betas = betas
        self.eps = eps
        self.weight_decay = weight_decay
        self.batch_per_proj = batch_per_proj
        self.random_offset_detector = random_offset_detector
        self.uniform_ray_spacing = uniform_ray_spacing
        self.step_count = 0
        self.workspace = Workspace()
        # gradients clamped to [-c, c] after the averaging over ranks (base_trainer.py:651-652)
        self.clip_grad_value = clip_grad_value
        # data parallel: every rank trains on its own rays, gradients are averaged before Adam
        self.data_parallel = data_parallel
        self.process_group = process_group
        # shard_optimizer: Adam state and update split over the ranks (ShardedAdam); the
        # gradient buffers are views of its padded reduce-scatter buffers
        self.sharded = None
        if shard_optimizer:
            if not data_parallel:
                raise ValueError("shard_optimizer splits Adam over the data-parallel ranks: pass data_parallel=True")
            self.sharded = ShardedAdam([model.table, model.mlp], process_group)
            self.table_grad, self.mlp_grad = self.sharded.grads
            self.m_table = self.v_table = self.m_mlp = self.v_mlp = None
        else:
            self.table_grad = torch.zeros_like(model.table)
            self.mlp_grad = torch.zeros_like(model.mlp)
            self.m_table = torch.zeros_like(model.table)
            self.v_table = torch.zeros_like(model.table)
            self.m_mlp = torch.zeros_like(model.mlp)
            self.v_mlp = torch.zeros_like(model.mlp)

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

    def step(self, batch: RayBatch) -> torch.Tensor:
        loss, _ = train_step(self.model, self.c_geometry, batch, self.geometry.max_distance_traveled,
                             self.table_grad, self.mlp_grad, self.workspace, self.loss)
        self._update(self.table_grad, self.mlp_grad)
        return loss

    def _update(self, g_table: torch.Tensor, g_mlp: torch.Tensor) -> None:
        """Gradient averaging over the ranks (data parallel) and the Adam step;
        the gradients are zeroed."""
        self.step_count += 1
        if self.sharded is not None:
            if g_table is not self.table_grad:  # gradients from autograd
                self.table_grad.add_(g_table)
                self.mlp_grad.add_(g_mlp)
            self.sharded.step(self.step_count, self.lr, self.betas, self.eps, self.weight_decay,
                              halves=[self.model.table_half, None], clip=self.clip_grad_value)
            return
        if self.data_parallel:
            reduce_gradients([g_table, g_mlp], self.process_group)
        if self.clip_grad_value is not None:
            g_table.clamp_(-self.clip_grad_value, self.clip_grad_value)
            g_mlp.clamp_(-self.clip_grad_value, self.clip_grad_value)
        adam_step(self.model.table, g_table, self.m_table, self.v_table, self.step_count, self.lr, self.betas,
                  self.eps, self.weight_decay, half=self.model.table_half)
        adam_step(self.model.mlp, g_mlp, self.m_mlp, self.v_mlp, self.step_count, self.lr, self.betas, self.eps,
                  self.weight_decay)

    def optimizer_moments(self):
        """[(exp_avg, exp_avg_sq) of the table, the same of the MLP] at full
        size.  With the sharded optimizer this gathers them: every rank calls."""
        if self.sharded is not None:
            return [self.sharded.full_moments(0), self.sharded.full_moments(1)]
        return [(self.m_table, self.v_table), (self.m_mlp, self.v_mlp)]

    @torch.no_grad()
    def load_optimizer_moments(self, moments) -> None:
        """Inverse of optimizer_moments (full-size tensors, any device)."""
        if self.sharded is not None:
            for i, (m, v) in enumerate(moments):
                self.sharded.load_moments(i, m.to(self.model.table.device), v.to(self.model.table.device))
            return
        for (dm, dv), (m, v) in zip(self.optimizer_moments(), moments):
            dm.copy_(m)
            dv.copy_(v)

    def continuous_step(self, perm: torch.Tensor, batch_num: int, angle_start: float, angle_stop: float,
                        projection: torch.Tensor, t: float = 0.0, accumulation_steps: int = 4,
                        add_poisson: bool = False, fused: bool = True) -> torch.Tensor | None:
        """One continuous-rotation step (continous_scanning_trainer.py:85-140):
        the detector integrates while the object turns from angle_start to
        angle_stop, so y_pred is the mean of ``accumulation_steps`` forwards at
        the mid-angles of equal sub-intervals (same pixels and t, a fresh
        jitter draw per sub-angle, drawn in the reference's order), optionally
        with the reference's Poisson noise term; then the loss, the
        hand-written backward and the Adam update.  ``fused``: every
        sub-angle's rays in one launch of each kernel (ScanIntegral); else
        one forward per sub-angle, each on its own workspace."""
        import numpy as np

        edges = np.linspace(angle_start, angle_stop, accumulation_steps + 1)
        mids = [float((edges[j] + edges[j + 1]) / 2) for j in range(accumulation_steps)]
        if fused:
            window = batching.batch_window(perm.numel(), self.batch_size, batch_num)
            if window is None:
                return None
            start, size = window
            draws = [draw_ray_randoms(size, self.random_offset_detector, self.device)
                     for _ in range(accumulation_steps)]
            batch = RayBatch(perm=perm, start=start, num_rays=size, points_per_ray=self.points_per_ray,
                             angle=mids[0], max_ray_distance_per_point=self.geometry.max_distance_traveled /
                             self.points_per_ray, jitter=torch.cat([d[0] for d in draws]),
                             detector_offset=torch.cat([d[1] for d in draws]), projection=projection, t=t,
                             uniform_ray_spacing=self.uniform_ray_spacing)
            y_pred = scan_integral(self.model, self.c_geometry, batch, mids, self.geometry.max_distance_traveled,
                                   self.workspace)
            y = projection[perm[start:start + size]]
            return self._loss_and_update(y_pred, y, add_poisson)
        if not hasattr(self, "_scan_ws") or len(self._scan_ws) != accumulation_steps:
            # every sub-angle forward keeps its workspace until the backward:
            # together they take one step's recommended staging
            self._scan_ws = [Workspace(staging_fraction=1.0 / accumulation_steps) for _ in range(accumulation_steps)]
        y_pred, batch = None, None
        for j in range(accumulation_steps):
            batch = self.make_batch(perm, batch_num, mids[j], projection, t)
            if batch is None:
                return None
            yj = ray_integral(self.model, self.c_geometry, batch, self.geometry.max_distance_traveled,
                              self._scan_ws[j]) / accumulation_steps
            y_pred = yj if y_pred is None else y_pred + yj
        y = projection[perm[batch.start:batch.start + batch.num_rays]]
        return self._loss_and_update(y_pred, y, add_poisson)

    def split_step(self, batch: RayBatch, add_poisson: bool = False, s3im_patch: int = 0,
                   tv_weight: float = 0.0, tv_origin=None) -> torch.Tensor:
        """One step with the loss composed in torch on y_pred (base_trainer.py:552-566):
        the L1/L2 loss, optionally the Poisson noise term, the S3IM term over
        ``s3im_patch``-sized patches and the total-variation term of the model
        on a 100^3 grid of side 0.2 at ``tv_origin`` (base_trainer.py:615-649);
        forward and backward are the fused halves (RayIntegral, ModelPoints)."""
        y_pred = ray_integral(self.model, self.c_geometry, batch, self.geometry.max_distance_traveled,
                              self.workspace)
        y = batch.projection[batch.perm[batch.start:batch.start + batch.num_rays]]
        extra = None
        if tv_weight > 0:
            pts = tv_points(tv_origin, device=y_pred.device)
            extra = total_variation_3d(model_points(self.model, pts).view(100, 100, 100), tv_weight)
        return self._loss_and_update(y_pred, y, add_poisson, s3im_patch, extra)

    def _loss_and_update(self, y_pred, y, add_poisson=False, s3im_patch=0, extra=None):
        if add_poisson:   # base_trainer.py:555-556; the Poisson draw carries no gradient
            y_pred = (y_pred + torch.poisson(y_pred.detach() * 1e5) / 1e5) / 2
        loss = projection_loss(y_pred, y, self.loss)
        if s3im_patch:
            from .schedule import s3im_loss

            loss = loss + s3im_loss(y_pred, y, s3im_patch)
        if extra is not None:
            loss = loss + extra
        g_table, g_mlp = torch.autograd.grad(loss, [self.model.table, self.model.mlp])
        self._update(g_table, g_mlp)
        return loss.detach()

    def device_error(self) -> int:
        """Error word of the last step (non-zero if a tensor-core wait timed out)."""
        return self.workspace.error_word(self.c_geometry)

    def train_projection(self, projection: torch.Tensor, angle: float, t: float = 0.0) -> torch.Tensor | None:
        """All batches of one projection (flattened, min-max scaled, on device)."""
        P = projection.numel()
        perm = torch.randperm(P, dtype=torch.int64, device=self.device)
        n_batches = batching.batches_per_projection(P, self.batch_size)
        loss = None
        for b in range(min(self.batch_per_proj, n_batches)):
            batch = self.make_batch(perm, b, angle, projection, t)
            if batch is None:
                continue
            loss = self.step(batch)
        return loss
