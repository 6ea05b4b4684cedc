"""End-to-end reconstructions on the GPU kernels (small parallel-beam
ellipsoid phantoms): what the trained network gains over reconstruction
without a learned model, and training with the reference's per-projection
schedules, S3IM and Poisson terms."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def problem(n=64, views=180, arc=math.pi):
    from nect_b200 import phantoms
    from nect_b200.sampling import Geometry

    geo = Geometry(nDetector=[n, n], dDetector=[1 / n, 1 / n], mode="parallel", nVoxel=[n] * 3, dVoxel=[1 / n] * 3)
    ph = phantoms.ellipsoid_phantom(20, 0)
    angles = np.linspace(0, arc, views, endpoint=False)
    projs = torch.stack([phantoms.ellipsoid_projection(ph, geo, float(a), "cuda") for a in angles])
    return geo, angles, projs, phantoms.ellipsoid_volume(ph, n, "cuda")


def model_cfg(n, precision="mixed"):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig

    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=17, base_resolution=8,
                            finest_resolution=4 * n)
    return ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), precision)


def test_trained_network_beats_back_projection_on_sparse_views(cuda_device):
    """With 24 views the filtered back-projection (the classical method,
    nect/fdk.py) streaks; the trained network interpolates between views."""
    from nect_b200.reconstruct import fbp_parallel, fit, psnr

    geo, angles, projs, truth = problem(64, views=24)
    fbp = fbp_parallel(projs, geo, angles)
    rec = fit(geo, projs, angles, model_cfg=model_cfg(64), niter=1500, lr=2e-3, points_per_ray=128, seed=0,
              evaluate=lambda r: {"psnr": psnr(r.volume(), truth)}, eval_every=1500)
    untrained, trained = rec.history[0][2]["psnr"], rec.history[-1][2]["psnr"]
    assert trained > untrained + 10
    assert trained > psnr(fbp, truth) + 1.0, (trained, psnr(fbp, truth))


def test_fit_with_schedules_s3im_and_poisson(cuda_device):
    from nect_b200.reconstruct import fit, psnr
    from nect_b200.schedule import Schedule

    geo, angles, projs, truth = problem(64, views=60)
    sch = Schedule(n_detector=geo.nDetector, n_projections=60, epochs=5, base_lr=2e-3, downsampling_start=4,
                   downsampling_update_interval=60, points_start=48, points_end=128, warmup_steps=30)
    seen = []
    rec = fit(geo, projs, angles, model_cfg=model_cfg(64), niter=10_000, points_per_ray=128, seed=1, schedule=sch, s3im=True,
              add_poisson=True, evaluate=lambda r: {"psnr": psnr(r.volume(), truth)}, eval_every=100)
    assert rec.trainer.step_count == sch.total_projections == 300
    assert geo.detector_binning == 1 and rec.trainer.c_geometry.nDetector[0] == 64
    first, last = rec.history[0][2]["psnr"], rec.history[-1][2]["psnr"]
    assert math.isfinite(last) and last > first + 8, (first, last)
