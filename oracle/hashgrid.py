"""CPU oracle for the hash-grid encoding, the MLP and one fused training step.

TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's CPU
baseline).  The product path never imports this module.

Encoding: the multiresolution hash encoding of Mueller, Evans, Schied and
Keller, "Instant Neural Graphics Primitives with a Multiresolution Hash
Encoding", ACM TOG 41(4), 2022 (section 3), which the reference obtains from
tiny-cuda-nn (nect/network/networks.py:52-57, 478-481).  tiny-cuda-nn is not
vendored in the reference and its version is not pinned (the reference README
installs git HEAD), so this oracle restates the PUBLISHED method and the build
defines the details the paper leaves open.  Parity of the encoding and MLP with
tiny-cuda-nn itself is therefore UNPINNED; hash indices are compared bit for
bit with the build's kernels, values within stated tolerances.

Build-defined details (shared with nect_b200/csrc/hashgrid.cuh):
  * level l resolution N_l = floor(N_min * b^l) per spatial axis, and
    floor(N_min_t * b^l) along t for 4D grids (paper eq. 2-3);
  * x in [0,1] is scaled by N_l in fp32; the cell is floor(x*N_l) clamped to
    N_l - 1; the (N_l+1)^d vertices are stored densely when they fit in T
    entries (rounded up to a multiple of 8), otherwise hashed;
  * hash = XOR_i (v_i * pi_i) mod T with pi = (1, 2654435761, 805459861) from
    the paper and a fourth prime 2246822519 chosen by this build for t;
  * axis order is the input order (z, y, x[, t]); axis 0 gets pi = 1 / stride 1;
  * features interpolate d-linearly; entries are F contiguous values.
MLP: tiny-cuda-nn FullyFusedMLP semantics as configured by MLPNetConfig
(nect/config.py:115-135): no biases, hidden activation, output activation.
Training step: the reference's inner loop restated without Fabric
(nect/trainers/base_trainer.py:517-568 + :650): sample, clamp, drop all-zero
points, model, y_pred = sum * distances / max_distance_traveled, L1/L2 loss.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

PRIMES = (1, 2654435761, 805459861, 2246822519)


@dataclass
class Level:
    res: tuple          # per-axis resolution (d entries)
    offset: int         # first entry of the level
    entries: int        # entries of the level
    hashed: bool


def layout(n_dims: int, n_levels: int, log2_T: int, base: float, scale: float, base_t: float | None = None):
    T = 1 << log2_T
    levels, off = [], 0
    for l in range(n_levels):
        r = int(math.floor(base * math.pow(scale, l)))
        res = [r, r, r]
        if n_dims == 4:
            res.append(int(math.floor((base_t if base_t else base) * math.pow(scale, l))))
        verts = 1
        for v in res:
            verts *= v + 1
        if verts <= T:
            entries, hashed = ((verts + 7) // 8) * 8, False
        else:
            entries, hashed = T, True
        levels.append(Level(tuple(res), off, entries, hashed))
        off += entries
    return levels, off


def corner_indices(x: torch.Tensor, lv: Level, log2_T: int):
    """x [N,d] fp32 in [0,1] -> (idx [N, 2^d] int64 within the level, w [N, 2^d] fp32 weights).

    Index arithmetic is exact integer work: the build's kernels must agree bit
    for bit."""
    d = x.shape[1]
    res = torch.tensor(lv.res, dtype=torch.float32)
    p = x.to(torch.float32) * res
    c = torch.floor(p)
    c = torch.minimum(c, res - 1).clamp(min=0)
    w = p - c
    c = c.to(torch.int64)
    idx, wts = [], []
    for corner in range(1 << d):
        bits = [(corner >> k) & 1 for k in range(d)]
        v = [c[:, k] + bits[k] for k in range(d)]
        if lv.hashed:
            h = torch.zeros_like(v[0])
            for k in range(d):
                h = h ^ ((v[k] * PRIMES[k]) & 0xFFFFFFFF)
            i = h & ((1 << log2_T) - 1)
        else:
            i = torch.zeros_like(v[0])
            stride = 1
            for k in range(d):
                i = i + v[k] * stride
                stride *= lv.res[k] + 1
        wt = torch.ones(x.shape[0], dtype=torch.float32)
        for k in range(d):
            wt = wt * (w[:, k] if bits[k] else (1 - w[:, k]))
        idx.append(i)
        wts.append(wt)
    return torch.stack(idx, 1), torch.stack(wts, 1)


def encode(x: torch.Tensor, table: torch.Tensor, levels, log2_T: int) -> torch.Tensor:
    """table [total, F] (any float dtype, may require grad) -> [N, L*F] in table's dtype."""
    outs = []
    for lv in levels:
        idx, w = corner_indices(x, lv, log2_T)
        feats = table[lv.offset + idx]                       # [N, 2^d, F]
        outs.append((feats * w.to(table.dtype).unsqueeze(-1)).sum(1))
    return torch.cat(outs, 1)


def activation(z: torch.Tensor, kind: str) -> torch.Tensor:
    kind = (kind or "none").lower()
    if kind == "none":
        return z
    if kind == "relu":
        return torch.relu(z)
    if kind == "leakyrelu":
        return torch.nn.functional.leaky_relu(z, 0.01)
    if kind == "softplus":
        return torch.nn.functional.softplus(z)
    if kind == "sigmoid":
        return torch.sigmoid(z)
    raise ValueError(kind)


def mlp(h: torch.Tensor, weights: list[torch.Tensor], act: str = "relu", out_act: str = "softplus"):
    """weights: [W0 [64,in], ..., W_out [1,64]] (PyTorch Linear layout, no bias)."""
    for W in weights[:-1]:
        h = activation(h @ W.t(), act)
    return activation(h @ weights[-1].t(), out_act)


def split_mlp_params(flat: torch.Tensor, n_input: int, width: int, n_hidden: int):
    shapes = [(width, n_input)] + [(width, width)] * (n_hidden - 1) + [(1, width)]
    out, o = [], 0
    for s in shapes:
        n = s[0] * s[1]
        out.append(flat[o:o + n].view(*s))
        o += n
    return out


def line_integrals(points: np.ndarray, distances: np.ndarray, tab: torch.Tensor, wf: torch.Tensor, levels,
                   log2_T: int, n_input: int, width: int, n_hidden: int, max_distance_traveled: float,
                   act: str = "relu", out_act: str = "softplus", t: float | None = None):
    """y_pred [R] of one batch of sampled rays, differentiable in (tab, wf):
    clamp (projector.py:127), drop all-zero points (base_trainer.py:523),
    sigma = MLP(encode(x)), y_pred = sum * distances / max_distance_traveled
    (base_trainer.py:552-554)."""
    R, S, _ = points.shape
    pts = torch.from_numpy(points).clamp(0, 1)
    keep = ~torch.all(pts.view(-1, 3) == 0, dim=-1)
    x = pts.view(-1, 3)[keep]
    if t is not None:
        x = torch.cat([x, torch.full((x.shape[0], 1), float(t), dtype=torch.float32)], 1)
    Ws = split_mlp_params(wf, n_input, width, n_hidden)
    sig = mlp(encode(x, tab, levels, log2_T), Ws, act, out_act).squeeze(-1)
    full = torch.zeros(R * S, dtype=tab.dtype).masked_scatter(keep, sig)
    scale = torch.from_numpy(distances).to(tab.dtype) / max_distance_traveled
    return full.view(R, S).sum(1) * scale


def _loss(y_pred, y, loss):
    if loss.lower() == "l2":
        return torch.nn.functional.mse_loss(y_pred, y)
    return torch.nn.functional.l1_loss(y_pred, y)


def train_step(points: np.ndarray, counts: np.ndarray, distances: np.ndarray, measured: np.ndarray,
               table: torch.Tensor, mlp_flat: torch.Tensor, levels, log2_T: int, n_input: int, width: int,
               n_hidden: int, max_distance_traveled: float, loss: str = "l2", act: str = "relu",
               out_act: str = "softplus", t: float | None = None, dtype=torch.float64):
    """Forward + backward of one batch (points from the sampling oracle).

    Returns (y_pred [R], loss scalar, grad_table, grad_mlp) as float64 tensors."""
    tab = table.detach().to(dtype).requires_grad_(True)
    wf = mlp_flat.detach().to(dtype).requires_grad_(True)
    y_pred = line_integrals(points, distances, tab, wf, levels, log2_T, n_input, width, n_hidden,
                            max_distance_traveled, act, out_act, t)
    L = _loss(y_pred, torch.from_numpy(measured).to(dtype), loss)
    L.backward()
    return y_pred.detach(), L.detach(), tab.grad.detach(), wf.grad.detach()


def averaged_step(samples: list, measured: np.ndarray, table: torch.Tensor, mlp_flat: torch.Tensor, levels,
                  log2_T: int, n_input: int, width: int, n_hidden: int, max_distance_traveled: float,
                  loss: str = "l2", act: str = "relu", out_act: str = "softplus", t: float | None = None,
                  dtype=torch.float64):
    """Continuous-rotation step (nect/trainers/continous_scanning_trainer.py:85-140):
    y_pred is the mean of the line integrals of the same pixels at several
    sub-angles; samples = [(points, distances), ...] one entry per sub-angle.

    Returns (y_pred [R], loss scalar, grad_table, grad_mlp) as float64 tensors."""
    tab = table.detach().to(dtype).requires_grad_(True)
    wf = mlp_flat.detach().to(dtype).requires_grad_(True)
    y_pred = sum(line_integrals(p, d, tab, wf, levels, log2_T, n_input, width, n_hidden, max_distance_traveled,
                                act, out_act, t) for p, d in samples) / len(samples)
    L = _loss(y_pred, torch.from_numpy(measured).to(dtype), loss)
    L.backward()
    return y_pred.detach(), L.detach(), tab.grad.detach(), wf.grad.detach()
