"""The identity behind QuadCubes' composite encoder (nect_b200/csrc/quadcubes.cu),
checked on the CPU against the oracle's 3D encoding in fp64.

For a 3D grid over (a, b, t) and one t, level l's trilinear interpolation at
(a, b, t) equals the bilinear interpolation over (a, b) of the plane

    P[k] = w0 * table[e0(k)] + w1 * table[e1(k)],

with t's lower vertex c and weights w0 = 1 - f, w1 = f taken as the oracle
takes them, and k and e0/e1 in one of three forms:
  - dense 3D level: k = a + b (r+1), e_v = k + (c+v) (r+1)^2;
  - hashed level whose (r+1)^2 vertices fit in T: k as above,
    e_v = (a ^ b pi_1 ^ (c+v) pi_2) mod T;
  - otherwise k = (a ^ b pi_1) mod T, e_v = k ^ ((c+v) pi_2 mod T), the hash
    being an XOR of per-axis terms.
The backward is the same identity transposed: the points' bilinear
contributions reduced into a plane-shaped gradient G, then spread as
grad[e_v(k)] += w_v G[k], equal the 3D scatter of the trilinear weights.
Tolerance 1e-6 of the largest entry: the oracle forms each corner's weight as
an fp32 product (wa wb wt), the plane as (wa wb) times an fp64 blend."""
import math

import numpy as np
import torch

from oracle import hashgrid as ohg

L, LOG2_T, F = 6, 11, 4
BASE, SCALE = 4.0, 1.65
T = 1 << LOG2_T
MASK = T - 1
P1, P2 = ohg.PRIMES[1], ohg.PRIMES[2]


def t_vertex(t: float, r: int):
    p = np.float32(t) * np.float32(r)
    c = int(min(max(math.floor(p), 0), r - 1))
    f = np.float32(p - np.float32(c))
    return c, float(np.float32(1) - f), float(f)


def plane_sources(lv, k: np.ndarray, c: int):
    """The two 3D entries (within the level) of plane entries k."""
    r = lv.res[0]
    v2 = (r + 1) ** 2
    if v2 > T:   # plane keyed by the hash
        return [k ^ (((c + v) * P2) & MASK) for v in (0, 1)]
    a, b = k % (r + 1), k // (r + 1)
    if lv.hashed:
        return [(a ^ ((b * P1) & 0xFFFFFFFF) ^ (((c + v) * P2) & 0xFFFFFFFF)) & MASK for v in (0, 1)]
    return [k + (c + v) * v2 for v in (0, 1)]


def plane_size(lv):
    return min((lv.res[0] + 1) ** 2, T)


def plane_corners(lv, ab: torch.Tensor):
    """Plane entry indices [N, 4] and bilinear weights [N, 4] (fp32 products)."""
    r = lv.res[0]
    res = torch.tensor([r, r], dtype=torch.float32)
    p = ab.to(torch.float32) * res
    cell = torch.minimum(torch.floor(p), res - 1).clamp(min=0)
    w = p - cell
    cell = cell.to(torch.int64)
    idx, wts = [], []
    for q in range(4):
        va, vb = cell[:, 0] + (q & 1), cell[:, 1] + (q >> 1)
        if (r + 1) ** 2 > T:
            i = (va ^ ((vb * P1) & 0xFFFFFFFF)) & MASK
        else:
            i = va + vb * (r + 1)
        wa = w[:, 0] if q & 1 else 1 - w[:, 0]
        wb = w[:, 1] if q >> 1 else 1 - w[:, 1]
        idx.append(i)
        wts.append(wa * wb)
    return torch.stack(idx, 1), torch.stack(wts, 1)


def setup():
    levels, total = ohg.layout(3, L, LOG2_T, BASE, SCALE)
    forms = {("dense" if not lv.hashed else ("plane" if (lv.res[0] + 1) ** 2 <= T else "hashed")) for lv in levels}
    assert forms == {"dense", "plane", "hashed"}, forms
    gen = torch.Generator().manual_seed(21)
    table = (torch.rand(total, F, generator=gen, dtype=torch.float64) - 0.5)
    ab = torch.rand(3000, 2, generator=gen)
    ab[:6] = torch.tensor([[0, 0], [1, 1], [1, 0], [0.5, 0.5], [1e-7, 0.999999], [0.25, 1.0]])
    return levels, table, ab


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_plane_encoding_equals_the_trilinear_grid():
    levels, table, ab = setup()
    for t in (0.0, 0.43, 0.999, 1.0):
        x3 = torch.cat([ab, torch.full((ab.shape[0], 1), t)], 1)
        ref = ohg.encode(x3, table, levels, LOG2_T)
        got = []
        for lv in levels:
            c, w0, w1 = t_vertex(t, lv.res[0])
            k = np.arange(plane_size(lv))
            e0, e1 = plane_sources(lv, k, c)
            assert e0.max() < lv.entries and e1.max() < lv.entries and e0.min() >= 0
            plane = w0 * table[lv.offset + torch.from_numpy(e0)] + w1 * table[lv.offset + torch.from_numpy(e1)]
            idx, w = plane_corners(lv, ab)
            got.append((plane[idx] * w.double().unsqueeze(-1)).sum(1))
        assert rel(torch.cat(got, 1), ref) < 1e-6, t


def test_plane_gradient_spread_equals_the_trilinear_scatter():
    levels, table, ab = setup()
    gen = torch.Generator().manual_seed(22)
    dout = torch.randn(ab.shape[0], L * F, generator=gen, dtype=torch.float64)
    t = 0.61
    x3 = torch.cat([ab, torch.full((ab.shape[0], 1), t)], 1)
    tab = table.clone().requires_grad_(True)
    (ohg.encode(x3, tab, levels, LOG2_T) * dout).sum().backward()
    grad = torch.zeros_like(table)
    for l, lv in enumerate(levels):
        idx, w = plane_corners(lv, ab)
        G = torch.zeros(plane_size(lv), F, dtype=torch.float64)
        d = dout[:, l * F:(l + 1) * F]
        for q in range(4):
            G.index_add_(0, idx[:, q], w[:, q].double().unsqueeze(-1) * d)
        c, w0, w1 = t_vertex(t, lv.res[0])
        e0, e1 = plane_sources(lv, np.arange(plane_size(lv)), c)
        grad.index_add_(0, lv.offset + torch.from_numpy(e0), w0 * G)
        grad.index_add_(0, lv.offset + torch.from_numpy(e1), w1 * G)
    assert rel(grad, tab.grad) < 1e-6
