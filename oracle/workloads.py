"""The benchmark workloads and one training step of the reference path on CPU.

TEST AND BASELINE INFRASTRUCTURE ONLY: bench.py's CPU arms (``--impl
reference`` and the ``cpu_baseline`` object) time ``CpuTrainer.step``; the
product path never imports this module, and this module imports nothing of
the product (``nect_b200``), so the CPU arm runs none of the product's code.

Workloads (static parallel 128^2, static cone 512^2, 4D cone 512^2, large 4D
cylindrical cone 2048^2) restate the reference's geometry rules:
``sVoxel = nVoxel * dVoxel``, ``distance_origin_to_detector = DSD - DSO``,
cylinder radius ``max(sVoxel[1], sVoxel[2]) / 2`` and height ``sVoxel[0]``
(nect/sampling/geometry.py:119-132, 322-407), ``max_distance_traveled``
(:156-174), and the hash grid's ``per_level_scale`` (nect/config.py:99-112).

``CpuTrainer.step`` is the reference's inner loop (nect/trainers/
base_trainer.py:517-568, 650-654) on the host cores: the C sampler
(oracle/sampling.c, the restatement of nect/sampling/ct_sampling.cu), clamp,
the all-zero mask, a PyTorch-CPU fp32 hash grid and MLP (oracle/hashgrid.py),
the line integral, the L2 loss, autograd and torch.optim.Adam.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import hashgrid as ohg
from . import sampling as osamp

KINDS = {("cone", "voxel"): 0, ("cone", "cylindrical"): 1, ("parallel", "voxel"): 2, ("parallel", "cylindrical"): 3}


@dataclass
class Workload:
    name: str
    mode: str                    # "cone" or "parallel"
    reconstruction_mode: str     # "voxel" or "cylindrical"
    nDetector: tuple
    dDetector: tuple
    nVoxel: tuple
    dVoxel: tuple
    DSO: float | None
    DSD: float | None
    n_dims: int
    n_features: int
    log2_T: int
    base: float
    finest: float | None         # finest resolution; None: max_resolution_factor 2 x max(nDetector)
    base_t: float | None
    hidden_layers: int
    S: int
    rays: int
    n_angles: int
    turns: float

    @property
    def sVoxel(self):
        return tuple(n * d for n, d in zip(self.nVoxel, self.dVoxel))

    @property
    def pixels(self) -> int:
        return self.nDetector[0] * self.nDetector[1]

    @property
    def per_level_scale(self) -> float:
        finest = self.finest if self.finest is not None else 2.0 * max(self.nDetector)
        return (finest / self.base) ** (1.0 / 15)

    @property
    def max_distance_traveled(self) -> float:
        sv, dv = self.sVoxel, self.dVoxel
        length = ((sv[1] - dv[1]) ** 2 + (sv[2] - dv[2]) ** 2) ** 0.5
        if self.mode == "cone":
            theta = math.atan(((sv[0] - dv[0]) / 2) / (self.DSO + length / 2))
            return length / math.cos(theta)
        if self.reconstruction_mode == "voxel":
            return length
        return max(sv[1], sv[2])

    def c_struct(self) -> osamp.Geometry:
        g = osamp.Geometry()
        g.kind = KINDS[(self.mode, self.reconstruction_mode)]
        for i in range(2):
            g.nDetector[i] = int(self.nDetector[i])
            g.dDetector[i] = float(self.dDetector[i])
        sv = self.sVoxel
        if self.reconstruction_mode == "voxel":   # the cylindrical structs carry no voxel grid
            for i in range(3):
                g.sVoxel[i] = float(sv[i])
                g.dVoxel[i] = float(self.dVoxel[i])
        if self.mode == "cone":
            g.distance_source_to_origin = float(self.DSO)
            g.distance_origin_to_detector = float(self.DSD - self.DSO)
        if self.reconstruction_mode == "cylindrical":
            g.object_radius = float(max(sv[1], sv[2]) / 2)
            g.object_height = float(sv[0])
        return g


def _w(**kw) -> Workload:
    return Workload(**kw)


WORKLOADS = {
    "c1_static_parallel": _w(name="c1_static_parallel", mode="parallel", reconstruction_mode="voxel",
                             nDetector=(128, 128), dDetector=(1 / 128, 1 / 128), nVoxel=(128,) * 3,
                             dVoxel=(1 / 128,) * 3, DSO=None, DSD=None, n_dims=3, n_features=2, log2_T=19, base=16,
                             finest=1024, base_t=None, hidden_layers=2, S=256, rays=65536, n_angles=180, turns=0.5),
    "c2_static_cone": _w(name="c2_static_cone", mode="cone", reconstruction_mode="voxel", nDetector=(512, 512),
                         dDetector=(1.0, 1.0), nVoxel=(256,) * 3, dVoxel=(1.0,) * 3, DSO=500.0, DSD=1000.0, n_dims=3,
                         n_features=2, log2_T=20, base=16, finest=None, base_t=None, hidden_layers=2, S=512,
                         rays=1 << 18, n_angles=720, turns=1),
    "c3_dynamic_cone": _w(name="c3_dynamic_cone", mode="cone", reconstruction_mode="voxel", nDetector=(512, 512),
                          dDetector=(1.0, 1.0), nVoxel=(256,) * 3, dVoxel=(1.0,) * 3, DSO=500.0, DSD=1000.0,
                          n_dims=4, n_features=2, log2_T=21, base=16, finest=None, base_t=4, hidden_layers=2, S=512,
                          rays=1 << 18, n_angles=3600, turns=10),
    "c5_large_cone": _w(name="c5_large_cone", mode="cone", reconstruction_mode="cylindrical",
                        nDetector=(2048, 2048), dDetector=(1.0, 1.0), nVoxel=(1024,) * 3, dVoxel=(1.0,) * 3,
                        DSO=2000.0, DSD=4000.0, n_dims=4, n_features=4, log2_T=22, base=16, finest=4096, base_t=4,
                        hidden_layers=3, S=1024, rays=1 << 20, n_angles=7200, turns=20),
}


def view_angles(w: Workload, n: int):
    """n of the workload's views: (angles, normalised timesteps)."""
    all_angles = np.linspace(0, 2 * math.pi * w.turns, w.n_angles, endpoint=False)
    idx = np.linspace(0, w.n_angles - 1, n).astype(int)
    return [float(a) for a in all_angles[idx]], [float(i / max(w.n_angles - 1, 1)) for i in idx]


class CpuTrainer:
    """The reference's training step on the host cores, fp32 (see module doc).

    Parameters are initialised as the product initialises them (table
    U(-1e-4, 1e-4), Glorot-uniform weights) from a seeded generator."""

    def __init__(self, w: Workload, lr: float = 1e-3, seed: int = 1337):
        self.w = w
        self.levels, total = ohg.layout(w.n_dims, 16, w.log2_T, float(w.base), w.per_level_scale,
                                        float(w.base_t or w.base))
        g = torch.Generator().manual_seed(seed)
        self.n_in = 16 * w.n_features
        self.table = ((torch.rand(total, w.n_features, generator=g) * 2 - 1) * 1e-4).requires_grad_(True)
        shapes = [(64, self.n_in)] + [(64, 64)] * (w.hidden_layers - 1) + [(1, 64)]
        self.mlp = torch.cat([(torch.rand(o * i, generator=g) * 2 - 1) * math.sqrt(6 / (o + i))
                              for o, i in shapes]).requires_grad_(True)
        self.opt = torch.optim.Adam([self.table, self.mlp], lr=lr)
        self.geom = w.c_struct()
        self.rng = np.random.default_rng(seed)

    def step(self, projection: torch.Tensor, angle: float, t: float, rays: int) -> float:
        """One batch of ``rays`` rays of one projection (a random pixel
        permutation, jittered samples), forward, backward and Adam."""
        w = self.w
        S = w.S
        perm = torch.randperm(w.pixels).numpy()
        jitter = (self.rng.random(rays, dtype=np.float32) - 0.5).astype(np.float32)
        det_off = np.zeros((rays, 2), np.float32)
        maxd = w.max_distance_traveled / S
        pts, dist, _ = osamp.oracle_sample(self.geom, perm, 0, rays, S, angle, maxd, True, jitter, det_off)
        self.opt.zero_grad()
        y_pred = ohg.line_integrals(pts, dist, self.table, self.mlp, self.levels, w.log2_T, self.n_in, 64,
                                    w.hidden_layers, w.max_distance_traveled, t=t if w.n_dims == 4 else None)
        y = projection[torch.from_numpy(perm[:rays])]
        loss = torch.nn.functional.mse_loss(y_pred, y)
        loss.backward()
        self.opt.step()
        return float(loss.detach())
