"""Adam sharded over data-parallel ranks (trainer.ShardedAdam) on three gloo
ranks on CPU: the parameters, moments and fp16 table copy equal those of the
gradient all-reduce followed by the full Adam step, with buffers that pad, a
rank that holds no element of a small buffer and a buffer gathered in place;
then the Trainer's update with the sharded optimizer, the checkpoint of its
gathered moments (rank 0 writes) and resume into every rank's shard.  The per-shard update here is
torch.optim.Adam's rule written in torch (the CUDA Adam kernel is the default
and needs a GPU); both arms use it, so the test checks the sharding."""
import math
import os

import torch
import torch.multiprocessing as mp

LR, WD = 1e-2, 0.01


def cpu_adam(param, grad, m, v, step, lr, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, half=None,
             zero_grad=True):
    b1, b2 = betas
    g = grad + weight_decay * param if weight_decay else grad.clone()
    m.lerp_(g, 1 - b1)
    v.mul_(b2).addcmul_(g, g, value=1 - b2)
    denom = (v.sqrt() / math.sqrt(1 - b2 ** step)).add_(eps)
    param.addcdiv_(m, denom, value=-lr / (1 - b1 ** step))
    if half is not None:
        half.copy_(param)
    if zero_grad:
        grad.zero_()


def rel(a, b):
    a, b = a.detach().double(), b.detach().double()
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


def make_trainer():
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    geo = Geometry(nDetector=[32, 32], dDetector=[1.0, 1.0], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[16] * 3,
                   dVoxel=[1.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=10, base_resolution=4,
                            finest_resolution=64)
    model = get_model(ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "mixed"), device="cpu")
    g = torch.Generator().manual_seed(3)
    with torch.no_grad():
        model.table.copy_(torch.rand(model.table.shape, generator=g))
        model.mlp.copy_(torch.rand(model.mlp.shape, generator=g))
        model.refresh_half()
    tr = Trainer(model, geo, points_per_batch=64 * 32, points_per_ray=32, lr=LR, weight_decay=WD, device="cpu",
                 data_parallel=True, shard_optimizer=True)
    tr.sharded.adam = cpu_adam
    return geo, model, tr


def _rank(rank, world, port, run_dir, out):
    import torch.distributed as dist

    from nect_b200 import checkpoint
    from nect_b200.trainer import ShardedAdam, reduce_gradients

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    res = {}
    try:
        # ShardedAdam against all-reduce + full Adam
        g = torch.Generator().manual_seed(0)
        params = [torch.rand(1003, 2, generator=g), torch.rand(10, generator=g), torch.rand(6, 8, generator=g)]
        ref = [p.clone() for p in params]
        ref_m, ref_v = [torch.zeros_like(p) for p in ref], [torch.zeros_like(p) for p in ref]
        half = params[0].half()
        sa = ShardedAdam(params, adam=cpu_adam)
        res["valid"] = [s[3] for s in sa.shards]
        gr = torch.Generator().manual_seed(100 + rank)
        for step in range(1, 4):
            grads = [torch.randn(p.shape, generator=gr) for p in ref]
            avg = [x.clone() for x in grads]
            reduce_gradients(avg)
            for i in range(3):
                cpu_adam(ref[i], avg[i], ref_m[i], ref_v[i], step, LR, weight_decay=WD)
                sa.grads[i].add_(grads[i])
            sa.step(step, LR, weight_decay=WD, halves=[half, None, None])
        res["param"] = max(rel(params[i], ref[i]) for i in range(3))
        res["padded"] = [g is not None for g in sa.gathered]
        res["half"] = bool(torch.equal(half, params[0].half()))
        mom = [sa.full_moments(i) for i in range(3)]
        res["moments"] = max(max(rel(mom[i][0], ref_m[i]), rel(mom[i][1], ref_v[i])) for i in range(3))
        res["grads_zeroed"] = all(float(gp.abs().max()) == 0.0 for gp in sa.grad_pad)

        # Trainer update (gradients from autograd), checkpoint, resume
        _, model, tr = make_trainer()
        t_ref, m_ref = model.table.detach().clone(), model.mlp.detach().clone()
        rm = [torch.zeros_like(t_ref), torch.zeros_like(m_ref)]
        rv = [torch.zeros_like(t_ref), torch.zeros_like(m_ref)]
        gt = torch.Generator().manual_seed(200 + rank)
        for step in range(1, 3):
            g_table, g_mlp = torch.randn(t_ref.shape, generator=gt), torch.randn(m_ref.shape, generator=gt)
            avg = [g_table.clone(), g_mlp.clone()]
            reduce_gradients(avg)
            cpu_adam(t_ref, avg[0], rm[0], rv[0], step, LR, weight_decay=WD)
            cpu_adam(m_ref, avg[1], rm[1], rv[1], step, LR, weight_decay=WD)
            tr._update(g_table, g_mlp)
        res["trainer"] = max(rel(model.table, t_ref), rel(model.mlp, m_ref))
        res["trainer_half"] = bool(torch.equal(model.table_half, model.table.detach().half()))
        path = checkpoint.save(run_dir, model, tr, epoch=1, angle=2)
        dist.barrier()
        data = torch.load(path, map_location="cpu", weights_only=False)
        st = data["optim"]["state"]
        res["ckpt"] = max(rel(st[0]["exp_avg"], rm[0]), rel(st[0]["exp_avg_sq"], rv[0]),
                          rel(st[1]["exp_avg"], rm[1]), rel(st[1]["exp_avg_sq"], rv[1]))
        _, m2, tr2 = make_trainer()
        checkpoint.resume(path, m2, tr2)
        n, chunk, lo, valid = tr2.sharded.shards[0]
        res["resume"] = bool(torch.equal(tr2.sharded.m[0][:valid], rm[0].reshape(-1)[lo:lo + valid])) and \
            tr2.step_count == 2 and bool(torch.equal(m2.table, model.table))
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_sharded_adam_matches_all_reduce_adam(tmp_path):
    world = 3
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29000 + os.getpid() % 1000
        procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path / "run"), out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        assert [out[r]["valid"][1] for r in range(world)] == [8, 2, 0]  # 10 elements, shards of 8
        assert out[0]["padded"] == [True, True, False]  # 48 elements in 3 shards of 16 gather in place
        for r in range(world):
            res = out[r]
            assert res["param"] < 1e-6 and res["moments"] < 1e-6, res
            assert res["half"] and res["grads_zeroed"], res
            assert res["trainer"] < 1e-6 and res["trainer_half"], res
            assert res["ckpt"] < 1e-6 and res["resume"], res


def test_shard_optimizer_needs_data_parallel():
    import pytest

    from nect_b200.trainer import Trainer

    with pytest.raises(ValueError, match="data_parallel"):
        Trainer.__init__(Trainer.__new__(Trainer), model=_DummyModel(), geometry=_DummyGeometry(),
                         points_per_batch=64, points_per_ray=32, device="cpu", shard_optimizer=True)


class _DummyGeometry:
    def get_c_geometry(self):
        return None


class _DummyModel:
    table = torch.zeros(4)
    mlp = torch.zeros(4)


def test_gradient_value_clipping_both_optimizer_paths(monkeypatch):
    """clip_grad_value clamps the averaged gradients before Adam
    (base_trainer.py:651-652), in the plain update and in the sharded one."""
    import torch.distributed as dist

    from nect_b200 import trainer as tmod
    from nect_b200.trainer import ShardedAdam

    g = torch.Generator().manual_seed(4)
    # plain path: Trainer._update with the module's Adam replaced by the torch rule
    monkeypatch.setattr(tmod, "adam_step", torch.no_grad()(cpu_adam))   # the kernel writes through pointers
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
    from nect_b200.sampling import Geometry

    geo = Geometry(nDetector=[32, 32], dDetector=[1.0, 1.0], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[16] * 3,
                   dVoxel=[1.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=10, base_resolution=4,
                            finest_resolution=64)
    model = get_model(ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "plain_fp32"), device="cpu")
    tr = tmod.Trainer(model, geo, points_per_batch=64 * 32, points_per_ray=32, lr=LR, device="cpu",
                      clip_grad_value=0.05)
    t0, m0 = model.table.detach().clone(), model.mlp.detach().clone()
    gt, gm = torch.randn(t0.shape, generator=g), torch.randn(m0.shape, generator=g)
    ref_t, ref_m = t0.clone(), m0.clone()
    cpu_adam(ref_t, gt.clamp(-0.05, 0.05), torch.zeros_like(t0), torch.zeros_like(t0), 1, LR)
    cpu_adam(ref_m, gm.clamp(-0.05, 0.05), torch.zeros_like(m0), torch.zeros_like(m0), 1, LR)
    tr._update(gt.clone(), gm.clone())
    assert rel(model.table, ref_t) < 1e-6 and rel(model.mlp, ref_m) < 1e-6

    # sharded path on a one-rank group
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(28000 + os.getpid() % 1000)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        p = torch.rand(100, generator=g)
        ref = p.clone()
        grad = torch.randn(100, generator=g)
        sa = ShardedAdam([p], adam=cpu_adam)
        sa.grads[0].add_(grad)
        sa.step(1, LR, clip=0.1)
        cpu_adam(ref, grad.clamp(-0.1, 0.1), torch.zeros(100), torch.zeros(100), 1, LR)
        assert rel(p, ref) < 1e-6
    finally:
        dist.destroy_process_group()
