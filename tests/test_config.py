"""The configuration interface the reference's users write (CPU):
HashEncoderConfig.per_level_scale (nect/config.py:99-112) for both resolution
types and sample_outside, its error when the size is missing, and the tcnn
schema dicts of get_encoder_config / get_network_config
(nect/config.py:86-94, 125-132), and the loss selection by name
(nect/config.py:481-497)."""
import pytest


def test_per_level_scale_rules():
    from nect_b200.config import HashEncoderConfig

    enc = HashEncoderConfig(n_levels=16, base_resolution=16, max_resolution_factor=2.0, nDetector=[256, 300])
    assert enc.per_level_scale == pytest.approx((2.0 * 300 / 16) ** (1 / 15), rel=1e-15)
    enc = HashEncoderConfig(n_levels=12, base_resolution=8, max_resolution_factor=1.5, nVoxel=[100, 120, 110],
                            sample_outside=3, max_resolution_type="nVoxel")
    assert enc.per_level_scale == pytest.approx((1.5 * 126 / 8) ** (1 / 11), rel=1e-15)   # 120 + 2 * 3
    with pytest.raises(ValueError, match="nDetector"):
        _ = HashEncoderConfig(nVoxel=[64] * 3).per_level_scale
    with pytest.raises(ValueError, match="nVoxel"):
        _ = HashEncoderConfig(nDetector=[64, 64], max_resolution_type="nVoxel").per_level_scale


def test_tcnn_schema_dicts():
    from nect_b200.config import HashEncoderConfig, MLPNetConfig

    enc = HashEncoderConfig(n_levels=19, n_features_per_level=4, log2_hashmap_size=21, base_resolution=8,
                            nDetector=[512, 512])
    assert enc.get_encoder_config() == {"otype": "HashGrid", "n_levels": 19, "n_features_per_level": 4,
                                        "log2_hashmap_size": 21, "base_resolution": 8,
                                        "per_level_scale": enc.per_level_scale}
    net = MLPNetConfig(n_hidden_layers=3, activation="ReLU", output_activation="Softplus")
    cfg = net.get_network_config()
    assert set(cfg) == {"otype", "n_hidden_layers", "n_neurons", "activation", "output_activation"}
    assert (cfg["n_hidden_layers"], cfg["n_neurons"], cfg["activation"]) == (3, 64, "ReLU")


def test_loss_selection_follows_the_reference():
    import torch

    from nect_b200.trainer import loss_kind, projection_loss

    assert [loss_kind(n) for n in ("L1", "l2", "L1+L2", "myl2")] == ["l1", "l2", "l1", "l2"]
    with pytest.raises(NotImplementedError):
        loss_kind("huber")
    a, b = torch.tensor([0.0, 1.0, 3.0]), torch.tensor([1.0, 1.0, 1.0])
    assert float(projection_loss(a, b, "L1")) == pytest.approx(1.0)
    assert float(projection_loss(a, b, "l2")) == pytest.approx(5.0 / 3)
