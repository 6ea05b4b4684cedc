"""CPU tests of the batch windows the Projector and the trainer share
(nect/sampling/projector.py:87-112 semantics), the default model
configurations reconstruct() builds, and the porous phantom's packing."""
import math

import numpy as np
import pytest


@pytest.mark.parametrize("pixels,rays,expect", [
    (100, 30, [(0, 30), (30, 30), (60, 30), None, None]),   # a partial last batch is skipped
    (90, 30, [(0, 30), (30, 30), (60, 30), None]),
    (20, 30, [(0, 20), None]),                               # a projection smaller than one batch
    (30, 30, [(0, 30), None]),
])
def test_batch_windows(pixels, rays, expect):
    from nect_b200.sampling import batching

    got = [batching.batch_window(pixels, rays, k) for k in range(len(expect))]
    assert got == expect
    assert batching.batches_per_projection(pixels, rays) == math.ceil(pixels / rays)
    assert batching.rays_per_batch(rays * 7 + 3, 7) == rays


def test_default_models_of_reconstruct():
    """Static scans train the reference's default static model
    (nect/cfg/static/hash_grid.yaml), dynamic scans its default dynamic model
    (nect/cfg/dynamic/quadcubes.yaml); the fused single-4D-grid model stays
    available."""
    from nect_b200.reconstruct import default_model_config, fused_dynamic_config, plan_reconstruction
    from nect_b200.sampling import Geometry

    geo = Geometry(nDetector=[256, 256], dDetector=[1.0, 1.0], mode="cone", DSD=800.0, DSO=400.0,
                   nVoxel=[128] * 3, dVoxel=[1.0] * 3)
    st = default_model_config(geo, "static", "mixed")
    assert (st.model, st.encoder.n_levels, st.encoder.n_features_per_level, st.encoder.base_resolution,
            st.encoder.log2_hashmap_size) == ("hash_grid", 19, 4, 8, 21)
    assert (st.net.n_hidden_layers, st.net.n_neurons, st.net.activation, st.net.output_activation) == (
        6, 64, "LeakyReLU", "ReLU")
    assert abs(st.encoder.per_level_scale - (2 * 256 / 8) ** (1 / 18)) < 1e-12
    dy = default_model_config(geo, "dynamic", "mixed", log2_hashmap_size=23)
    assert (dy.model, dy.encoder.n_levels, dy.encoder.n_features_per_level, dy.encoder.log2_hashmap_size,
            dy.encoder.base_resolution) == ("quadcubes", 23, 4, 23, 16)
    assert (dy.net.n_hidden_layers, dy.net.n_neurons, dy.net.activation, dy.net.output_activation,
            dy.net.include_identity) == (4, 128, "LeakyReLU", "None", True)
    assert abs(dy.encoder.per_level_scale - (2 * 256 / 16) ** (1 / 22)) < 1e-12
    fu = fused_dynamic_config(geo, "mixed")
    assert (fu.model, fu.encoder.n_levels, fu.encoder.n_features_per_level, fu.net.n_hidden_layers) == (
        "hash_grid_4d", 16, 2, 2)
    plan = plan_reconstruction(geo, "static", 100, quality="poor")
    assert plan.model_cfg.encoder.n_levels == 19 and plan.model_cfg.encoder.log2_hashmap_size == 19


def test_porous_phantom_reaches_the_packing_target():
    """Collective rearrangement fills the cylinder to the target fraction with
    spheres that neither overlap nor leave the cylinder, radii within
    [r_min, r_max] up to the final 0.01-voxel shrink."""
    from nect_b200.phantoms import porous_phantom

    # the benchmark phantom's proportions at half the size: 128^3, radii U[1.5, 6]
    ph = porous_phantom(128, seed=3, r_min=1.5, r_max=6.0, target=0.6)
    assert ph.packing > 0.599, ph.packing
    c, r = ph.centers, ph.radii
    assert r.min() >= 1.5 - 0.011 and r.max() <= 6.0
    d = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(d, np.inf)
    assert (d - (r[:, None] + r[None, :])).min() >= -1e-9
    rho = np.sqrt(c[:, 0] ** 2 + c[:, 1] ** 2)
    assert (rho + r <= ph.radius + 1e-9).all() and (np.abs(c[:, 2]) + r <= ph.half_height + 1e-9).all()
