"""FP64 central finite differences of the training loss.  TEST INFRASTRUCTURE ONLY.

The loss is the reference's training objective for one batch
(nect/trainers/base_trainer.py:517-568): sample, clamp, drop all-zero points,
sigma = MLP(encode(x)), y_pred = sum(sigma) * distances / max_distance_traveled,
L2 or L1 against the measured values.  It is evaluated in float64 on the
sampling oracle's points.

To make 1,000 parameters affordable the encodings, corner indices and weights
of every sample are cached once.  Perturbing one table value changes only the
samples whose corners hit that entry: their encoding moves by h times the
summed corner weights, their sigma is recomputed, and so is the loss.  That is
exact, not an approximation.  Perturbing an MLP weight recomputes the network
on the cached encodings.
"""
from __future__ import annotations

import numpy as np
import torch

from . import hashgrid as ohg


class BatchLoss:
    def __init__(self, points: np.ndarray, distances: np.ndarray, measured: np.ndarray, table: torch.Tensor,
                 mlp_flat: torch.Tensor, levels, log2_T: int, n_input: int, width: int, n_hidden: int,
                 max_distance_traveled: float, loss: str = "l2", act: str = "relu", out_act: str = "softplus",
                 t: float | None = None):
        R, S, _ = points.shape
        pts = torch.from_numpy(points).clamp(0, 1)
        keep = ~torch.all(pts.view(-1, 3) == 0, dim=-1)
        x = pts.view(-1, 3)[keep]
        if t is not None:
            x = torch.cat([x, torch.full((x.shape[0], 1), float(t), dtype=torch.float32)], 1)
        self.ray = torch.arange(R).repeat_interleave(S)[keep]          # ray of each kept sample
        self.table = table.detach().double().clone()
        self.mlp_flat = mlp_flat.detach().double().clone()
        self.levels, self.log2_T = levels, log2_T
        self.n_input, self.width, self.n_hidden = n_input, width, n_hidden
        self.act, self.out_act, self.loss_kind = act, out_act, loss.lower()
        self.F = self.table.shape[1]
        self.idx, self.w = [], []
        for lv in levels:
            i, w = ohg.corner_indices(x, lv, log2_T)
            self.idx.append(i + lv.offset)                              # global entry per corner
            self.w.append(w.double())
        self.enc = torch.cat([(self.table[i] * w.unsqueeze(-1)).sum(1) for i, w in zip(self.idx, self.w)], 1)
        self.scale = torch.from_numpy(distances).double() / max_distance_traveled
        self.y = torch.from_numpy(measured).double()
        self.R = R
        self.sigma = self._sigma(self.enc, self.mlp_flat)
        self.level_of = np.concatenate([[l] * lv.entries for l, lv in enumerate(levels)])

    def _sigma(self, enc: torch.Tensor, flat: torch.Tensor) -> torch.Tensor:
        Ws = ohg.split_mlp_params(flat, self.n_input, self.width, self.n_hidden)
        return ohg.mlp(enc, Ws, self.act, self.out_act).squeeze(-1)

    def _loss(self, sigma: torch.Tensor) -> float:
        y_pred = torch.zeros(self.R, dtype=torch.float64).index_add_(0, self.ray, sigma) * self.scale
        d = y_pred - self.y
        return float((d * d).mean() if self.loss_kind == "l2" else d.abs().mean())

    def loss(self) -> float:
        return self._loss(self.sigma)

    def touched_entries(self) -> np.ndarray:
        """Global table entries hit by at least one sample's corners."""
        return np.unique(torch.cat([i.flatten() for i in self.idx]).numpy())

    def table_fd(self, entry: int, feature: int, h: float) -> float:
        """(L(theta + h e) - L(theta - h e)) / 2h for table value [entry, feature]."""
        l = int(self.level_of[entry])
        hit = (self.idx[l] == entry)
        wsum = (self.w[l] * hit).sum(1)                                 # summed weight per sample
        rows = torch.nonzero(wsum != 0).flatten()
        if rows.numel() == 0:
            return 0.0
        col = l * self.F + feature
        out = []
        for sgn in (1.0, -1.0):
            enc = self.enc[rows].clone()
            enc[:, col] += sgn * h * wsum[rows]
            sig = self.sigma.clone()
            sig[rows] = self._sigma(enc, self.mlp_flat)
            out.append(self._loss(sig))
        return (out[0] - out[1]) / (2 * h)

    def mlp_fd(self, i: int, h: float) -> float:
        out = []
        for sgn in (1.0, -1.0):
            flat = self.mlp_flat.clone()
            flat[i] += sgn * h
            out.append(self._loss(self._sigma(self.enc, flat)))
        return (out[0] - out[1]) / (2 * h)

    def autograd(self):
        """Analytic gradients (autograd through the same fp64 graph)."""
        tab = self.table.clone().requires_grad_(True)
        flat = self.mlp_flat.clone().requires_grad_(True)
        enc = torch.cat([(tab[i] * w.unsqueeze(-1)).sum(1) for i, w in zip(self.idx, self.w)], 1)
        sig = self._sigma(enc, flat)
        y_pred = torch.zeros(self.R, dtype=torch.float64).index_add(0, self.ray, sig) * self.scale
        d = y_pred - self.y
        L = (d * d).mean() if self.loss_kind == "l2" else d.abs().mean()
        L.backward()
        return tab.grad.detach(), flat.grad.detach()


def seeded_parameters(bl: BatchLoss, n_table: int, n_mlp: int, seed: int = 0):
    """n_table (entry, feature) pairs among the touched entries and n_mlp MLP
    weight indices, drawn with numpy's default_rng(seed)."""
    rng = np.random.default_rng(seed)
    touched = bl.touched_entries()
    ent = rng.choice(touched, size=min(n_table, touched.size), replace=False)
    feat = rng.integers(0, bl.F, ent.size)
    mlp_idx = rng.choice(bl.mlp_flat.numel(), size=n_mlp, replace=False)
    return list(zip(ent.tolist(), feat.tolist())), mlp_idx.tolist()
