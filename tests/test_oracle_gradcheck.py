"""The oracle's analytic gradients against FP64 central finite differences
(CPU).  The GPU kernels' gradients are checked against the same finite
differences in test_gradcheck_gpu.py; this file checks the checker."""
import math

import numpy as np
import torch

from oracle import gradcheck as ogc
from oracle import hashgrid as ohg
from oracle import sampling as osamp


def parallel_cube(n=16):
    return osamp.to_struct(dict(kind=2, nDetector=(n, n), dDetector=(1 / n, 1 / n), offOrigin=(0, 0, 0),
                                offDetector=(0, 0), rotDetector=(0, 0, 0), COR=0.0, distance_source_to_origin=0.0,
                                distance_origin_to_detector=0.0, sVoxel=(1.0, 1.0, 1.0),
                                dVoxel=(1 / n, 1 / n, 1 / n), object_radius=0.0, object_height=0.0,
                                remove_factor_top=0.0, remove_factor_bottom=0.0))


def make_batch_loss(n_dims, loss):
    g = parallel_cube()
    rng = np.random.default_rng(5)
    R, S = 64, 24
    perm = rng.permutation(256).astype(np.int64)
    maxd = math.sqrt(2) * (1 - 1 / 16) / S
    pts, dist, _ = osamp.oracle_sample(g, perm, 0, R, S, 0.6, maxd, True,
                                       (rng.random(R, dtype=np.float32) - 0.5).astype(np.float32),
                                       np.zeros((R, 2), np.float32))
    levels, total = ohg.layout(n_dims, 16, 10, 2.0, 1.3, 2.0 if n_dims == 4 else None)
    table = torch.from_numpy(rng.uniform(-0.5, 0.5, (total, 2)))
    n_in = 32
    mlp = torch.cat([torch.from_numpy(rng.uniform(-1, 1, o * i) * math.sqrt(6 / (o + i)))
                     for o, i in [(64, n_in), (64, 64), (1, 64)]])
    measured = rng.random(R)
    return ogc.BatchLoss(pts, dist, measured, table, mlp, levels, 10, n_in, 64, 2, math.sqrt(2) * (1 - 1 / 16),
                         loss=loss, t=0.4 if n_dims == 4 else None)


def test_oracle_autograd_matches_finite_differences():
    for n_dims, loss in ((3, "l2"), (4, "l2")):
        bl = make_batch_loss(n_dims, loss)
        gt, gm = bl.autograd()
        tab, mlp_idx = ogc.seeded_parameters(bl, 150, 50, seed=1)
        h = 1e-6
        fd_t = np.array([bl.table_fd(e, f, h) for e, f in tab])
        ad_t = np.array([float(gt[e, f]) for e, f in tab])
        fd_m = np.array([bl.mlp_fd(i, h) for i in mlp_idx])
        ad_m = np.array([float(gm[i]) for i in mlp_idx])
        scale_t = np.abs(fd_t).max()
        scale_m = np.abs(fd_m).max()
        assert scale_t > 0 and scale_m > 0
        assert np.abs(fd_t - ad_t).max() <= 1e-6 * scale_t, np.abs(fd_t - ad_t).max() / scale_t
        assert np.abs(fd_m - ad_m).max() <= 1e-6 * scale_m, np.abs(fd_m - ad_m).max() / scale_m
