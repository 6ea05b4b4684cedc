"""Per-projection training schedules and the S3IM loss.

The reference changes three things as training proceeds, once per projection:

* detector binning (base_trainer.py:235-270, 300-306): the projection is
  average-pooled by ``factor`` and the geometry binned, starting at
  ``downsampling_detector.start`` and halving every ``update_interval``
  projections down to ``end``; while binned, rays get a random detector
  offset of 0.5 pixel;
* points per ray (base_trainer.py:154-175, 200-205, 250-262): from ``start``
  up to ``end`` (auto: 1.5 x the largest detector size), one more (linear) or
  twice as many per ``update_interval`` projections (auto: the ramp ends after
  90 % of the epochs);
* the learning rate (config.py:437-479, base_trainer.py:283-288): an
  exponential or linear warm-up (LambdaLR) interleaved with a cosine or
  exponential decay on the same optimizer.  The exact sequence the
  reference's torch schedulers produce is obtained here by running the same
  torch scheduler objects, in the same order, on a dummy optimizer.

``Schedule.steps()`` yields the settings of each projection in turn.
``s3im_loss`` is the reference's S3IM term (config.py:526-548): SSIM over
random patches of the batch's rays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass
class ProjectionSettings:
    projection: int
    detector_binning: int
    points_per_ray: int
    lr: float
    random_offset_detector: float


class Schedule:
    def __init__(self, n_detector, n_projections: int, epochs: int | str = "auto", base_lr: float = 1e-3,
                 downsampling_start: int = 2, downsampling_end: int = 1, downsampling_update_interval: int = 1000,
                 points_start: int = 100, points_end: int | str = "auto", points_update_interval: int | str = "auto",
                 points_linear: bool = True, warmup_steps: int = 500, warmup_lr0: float = 1e-3,
                 warmup_otype: str = "exponential", lr_otype: str = "cosine", lrf: float | str = "auto",
                 n_gpus: int = 1):
        nmax = max(n_detector)
        if isinstance(epochs, str):   # base_trainer.py:81-85
            e = math.ceil(49 / n_projections * nmax)
            parts = epochs.split("x")
            epochs = math.ceil(e * float(parts[0])) if len(parts) == 2 else e
        self.epochs = int(epochs)
        self.n_projections = n_projections
        if points_end == "auto":
            points_end = math.ceil(nmax * 1.5)
        elif isinstance(points_end, str):
            points_end = math.ceil(nmax * float(points_end.split("x")[0]))
        if isinstance(points_update_interval, str):
            factor = 0.9 if points_update_interval == "auto" else float(points_update_interval.split("x")[0])
            total_updates = n_projections * self.epochs * factor / n_gpus
            points_update_interval = math.ceil(total_updates / max(points_end - points_start, 1))
        self.ds = (downsampling_start, downsampling_end, downsampling_update_interval)
        self.pts = (points_start, int(points_end), int(points_update_interval), points_linear)
        self.warmup = (warmup_steps, warmup_lr0, warmup_otype)
        if lrf == "auto":
            lrf = max(1e-2, min(0.5, 1 / (self.epochs * 0.1)))
        self.lr = (base_lr, lr_otype, float(lrf))
        self.n_gpus = n_gpus

    @property
    def total_projections(self) -> int:
        return self.epochs * self.n_projections

    def _schedulers(self):
        base_lr, otype, lrf = self.lr
        steps, lr0, wtype = self.warmup
        opt = torch.optim.SGD([torch.zeros(1, requires_grad=True)], lr=base_lr)
        fexp = (1 / lr0) ** (1 / steps)
        flin = (1 - lr0) / steps
        if wtype == "linear":
            def warm(p):
                return p * flin if p < steps else 1
        else:
            def warm(p):
                return 1 / (fexp ** (steps - p)) if p < steps else 1
        warmup = torch.optim.lr_scheduler.LambdaLR(opt, lr_lambda=warm)
        torch.optim.lr_scheduler.LambdaLR(opt, lr_lambda=lambda x: x / 500)   # constructed, never stepped
        if otype.casefold() == "exponential":
            decay = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=lrf ** (1 / (self.epochs * self.n_projections)))
        else:
            decay = torch.optim.lr_scheduler.CosineAnnealingLR(
                opt, T_max=self.epochs * self.n_projections // self.n_gpus, eta_min=base_lr * lrf)
        return opt, warmup, decay

    def steps(self, start: int = 0):
        """Settings of projections start, start+1, ... total_projections-1."""
        ds_start, ds_end, ds_int = self.ds
        p_start, p_end, p_int, linear = self.pts
        opt, warmup, decay = self._schedulers()
        factor = max(1, ds_start // 2 ** (start // ds_int))           # base_trainer.py:200-205
        pts = (min(p_end, p_start + start // p_int) if linear
               else min(p_end, p_start * 2 ** (start // p_int)))
        for p in range(start):                                       # bring the lr to `start`
            opt.step()   # no gradients: keeps the reference's optimizer-then-scheduler order
            decay.step()
            if p + 1 <= self.warmup[0]:
                warmup.step()
        for p in range(start, self.total_projections):
            if p != 0 and p % ds_int == 0 and factor > ds_end:       # set_projection, base_trainer.py:244-262
                factor //= 2
            if p != 0 and p % p_int == 0 and pts < p_end:
                pts = pts + 1 if linear else pts * 2
            yield ProjectionSettings(p, factor, min(pts, p_end), opt.param_groups[0]["lr"],
                                     0.5 if factor > 1 else 0.0)
            opt.step()
            decay.step()                                             # on_angle_end, base_trainer.py:283-288
            if p + 1 <= self.warmup[0]:
                warmup.step()


def bin_projection(projection: torch.Tensor, factor: int) -> torch.Tensor:
    """[rows, cols] -> average-pooled [rows // f, cols // f] (base_trainer.py:300-306)."""
    if factor == 1:
        return projection
    return torch.nn.functional.avg_pool2d(projection[None], kernel_size=factor, stride=factor)[0]


def ssim2d(x: torch.Tensor, y: torch.Tensor, data_range: float = 1.0, win: int = 5, stride: int = 5,
           sigma: float = 1.5) -> torch.Tensor:
    """Mean SSIM (Wang et al. 2004) of [N,1,H,W] images with a Gaussian
    window of size ``win`` evaluated every ``stride`` pixels; the reference
    uses torch_extra's SSIM(data_range=1, win_size=5, stride=5), which is not
    installed here."""
    g = torch.exp(-((torch.arange(win, device=x.device, dtype=x.dtype) - win // 2) ** 2) / (2 * sigma ** 2))
    g = g / g.sum()
    w = (g[:, None] * g[None, :])[None, None]

    def f(v):
        return torch.nn.functional.conv2d(v, w, stride=stride)

    mx, my = f(x), f(y)
    sxx, syy, sxy = f(x * x) - mx * mx, f(y * y) - my * my, f(x * y) - mx * my
    c1, c2 = (0.01 * data_range) ** 2, (0.03 * data_range) ** 2
    return (((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))).mean()


def s3im_loss(pred: torch.Tensor, target: torch.Tensor, patch_size: int) -> torch.Tensor:
    """S3IM (config.py:526-548): five times, shuffle the batch's rays, take
    patch_size^2 of them as one image and add (1 - SSIM) / 5; times 3."""
    loss = pred.new_zeros(())
    if patch_size < 5:
        return loss
    pred, target = pred.float(), target.float()
    for _ in range(5):
        idx = torch.randperm(target.size(0), device=target.device)
        a = pred[idx][: patch_size ** 2].reshape(-1, 1, patch_size, patch_size)
        b = target[idx][: patch_size ** 2].reshape(-1, 1, patch_size, patch_size)
        loss = loss + (1 - ssim2d(a, b)) / 5
    return loss * 3


def s3im_patch_size(total_detector_pixels: int, batch_size: int) -> int:
    """base_trainer.py:559-562."""
    return min(math.floor(math.sqrt(total_detector_pixels)), math.floor(math.sqrt(batch_size)))
