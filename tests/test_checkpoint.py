"""Checkpoints in the reference's directory layout and keys (CPU): save,
prune, load into a fresh model built from config.yaml, resume the Adam state,
and load that state into a stock torch.optim.Adam."""
import torch
import yaml


def make(precision):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    geo = Geometry(nDetector=[32, 32], dDetector=[1.0, 1.0], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[16] * 3,
                   dVoxel=[1.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=10, base_resolution=4,
                            finest_resolution=64, base_resolution_t=2)
    model = get_model(ModelConfig("hash_grid_4d", enc, MLPNetConfig(n_hidden_layers=2), precision), device="cpu")
    g = torch.Generator().manual_seed(3)
    with torch.no_grad():
        model.table.copy_(torch.rand(model.table.shape, generator=g))
        model.mlp.copy_(torch.rand(model.mlp.shape, generator=g))
        model.refresh_half()
    tr = Trainer(model, geo, points_per_batch=64 * 32, points_per_ray=32, lr=2e-3, device="cpu")
    for t in (tr.m_table, tr.v_table, tr.m_mlp, tr.v_mlp):
        t.copy_(torch.rand(t.shape, generator=g))
    tr.step_count = 7
    return geo, model, tr


def test_save_prune_load_resume(tmp_path):
    from nect_b200 import checkpoint

    for precision in ("plain_fp32", "mixed"):
        geo, model, tr = make(precision)
        run = tmp_path / precision
        path = checkpoint.save(run, model, tr, geo, epoch=2, angle=5)
        assert path == run / "model" / "checkpoints" / "last.ckpt"
        data = torch.load(path, map_location="cpu", weights_only=False)
        assert set(data) == {"model", "optim", "epoch", "angle", "lr_scheduler"}
        assert set(data["model"]) == {"table", "mlp"}
        cfg = yaml.safe_load(open(run / "model" / "config.yaml"))
        assert cfg["model"] == "hash_grid_4d" and cfg["geometry"] == "SAME_FOLDER"
        assert yaml.safe_load(open(run / "model" / "geometry.yaml"))["nDetector"] == [32, 32]

        pruned = torch.load(checkpoint.prune(run), map_location="cpu", weights_only=False)
        assert set(pruned) == {"model"}
        m2 = checkpoint.model_from_dir(run / "pruned", device="cpu")
        assert torch.equal(m2.table, model.table) and torch.equal(m2.mlp, model.mlp)
        if precision == "mixed":
            assert torch.equal(m2.table_half, model.table.detach().half())

        _, m3, tr3 = make(precision)
        with torch.no_grad():
            m3.table.zero_()
            tr3.m_table.zero_()
        tr3.step_count = 0
        pos = checkpoint.resume(path, m3, tr3)
        assert pos == {"epoch": 2, "angle": 5}
        assert torch.equal(m3.table, model.table)
        assert torch.equal(tr3.m_table, tr.m_table) and torch.equal(tr3.v_mlp, tr.v_mlp)
        assert tr3.step_count == 7

        opt = torch.optim.Adam([m3.table, m3.mlp], lr=2e-3)
        opt.load_state_dict(data["optim"])
        assert torch.equal(opt.state[m3.table]["exp_avg"], tr.m_table)
        assert torch.equal(opt.state[m3.mlp]["exp_avg_sq"], tr.v_mlp)
