"""Per-projection schedules (CPU): detector binning, points-per-ray ramp and
the learning rate sequence, and the S3IM loss."""
import math

import torch


def test_schedule_follows_the_reference_rules():
    from nect_b200.schedule import Schedule

    sch = Schedule(n_detector=(128, 128), n_projections=50, epochs=10, base_lr=1e-3, downsampling_start=4,
                   downsampling_end=1, downsampling_update_interval=100, points_start=100, points_end="auto",
                   points_update_interval="auto", warmup_steps=50, warmup_lr0=1e-3, lrf=0.05)
    st = list(sch.steps())
    assert len(st) == sch.total_projections == 500
    # binning 4 -> 2 -> 1 at projections 100 and 200
    assert [s.detector_binning for s in st[:100]] == [4] * 100
    assert st[100].detector_binning == 2 and st[199].detector_binning == 2 and st[200].detector_binning == 1
    assert all(s.random_offset_detector == (0.5 if s.detector_binning > 1 else 0.0) for s in st)
    # points per ray: linear ramp from 100 to ceil(1.5 * 128) = 192, every ceil(50*10*0.9/92) projections
    step = math.ceil(50 * 10 * 0.9 / 92)
    assert st[0].points_per_ray == 100 and st[step].points_per_ray == 101 and st[-1].points_per_ray == 192
    assert all(b.points_per_ray - a.points_per_ray in (0, 1) for a, b in zip(st, st[1:]))
    # learning rate: exponential warm-up up to the base rate, then cosine decay towards lrf * base
    lrs = [s.lr for s in st]
    assert all(b >= a for a, b in zip(lrs[1:50], lrs[2:51]))
    assert abs(lrs[50] - 1e-3) < 1e-4
    assert lrs[-1] < 0.1 * 1e-3 and lrs[-1] >= 0.05 * 1e-3 * 0.99


def test_schedule_resumes_mid_run():
    from nect_b200.schedule import Schedule

    sch = Schedule(n_detector=(64, 64), n_projections=20, epochs=5, warmup_steps=10, downsampling_update_interval=30)
    full = list(sch.steps())
    tail = list(sch.steps(start=37))
    assert [(s.detector_binning, s.points_per_ray) for s in tail] == \
           [(s.detector_binning, s.points_per_ray) for s in full[37:]]
    assert all(abs(a.lr - b.lr) <= 1e-12 for a, b in zip(tail, full[37:]))


def test_s3im_is_zero_for_identical_rays_and_grows_with_noise():
    from nect_b200.schedule import s3im_loss, s3im_patch_size

    torch.manual_seed(0)
    y = torch.rand(4096)
    assert s3im_patch_size(128 * 128, 4096) == 64
    assert float(s3im_loss(y, y, 64)) < 1e-6
    assert float(s3im_loss(y + 0.3 * torch.rand(4096), y, 64)) > 0.05
    assert float(s3im_loss(y, y, 4)) == 0.0


def _old_loop_order(n_proj, seed, niter):
    """The projection order of fit's loop as first written (inline)."""
    import numpy as np

    order = np.random.default_rng(seed).permutation(n_proj)
    out = []
    for step in range(1, niter + 1):
        out.append(int(order[(step - 1) % n_proj]))
        if (step - 1) % n_proj == n_proj - 1:
            order = np.random.default_rng(seed + step).permutation(n_proj)
    return out


def test_step_plan_keeps_the_order_and_resumes_exactly():
    from nect_b200.reconstruct import step_plan
    from nect_b200.schedule import Schedule

    n_proj, seed, niter = 7, 3, 40
    full = list(step_plan(n_proj, seed, niter))
    assert [k for _, k, _ in full] == _old_loop_order(n_proj, seed, niter)
    assert [s for s, _, _ in full] == list(range(1, niter + 1))
    for start in (1, 6, 7, 8, 20, 21, 39):
        assert list(step_plan(n_proj, seed, niter, start=start)) == full[start:]

    sch = Schedule([64, 64], n_projections=n_proj, epochs=6, base_lr=2e-3, downsampling_start=8,
                   downsampling_update_interval=9, points_start=40, points_end=96, points_update_interval=4,
                   warmup_steps=10)
    full = list(step_plan(n_proj, seed, sch.total_projections, sch))
    for start in (5, 14, 30):   # between the binning (9) and points-per-ray (4) updates
        tail = list(step_plan(n_proj, seed, sch.total_projections, sch, start=start))
        assert [(s, k) for s, k, _ in tail] == [(s, k) for s, k, _ in full[start:]]
        for (_, _, a), (_, _, b) in zip(tail, full[start:]):
            assert (a.detector_binning, a.points_per_ray) == (b.detector_binning, b.points_per_ray)
            assert abs(a.lr - b.lr) <= 1e-12 * abs(b.lr)
    # Resumed on an update boundary the reference applies that update twice:
    # its resume derives binning and points per ray from projection // interval
    # (base_trainer.py:198-205), then set_projection updates again at the same
    # projection (base_trainer.py:244-262).  Schedule.steps(start) keeps that.
    (_, _, a), (_, _, b) = next(iter(step_plan(n_proj, seed, sch.total_projections, sch, start=18))), full[18]
    assert (a.detector_binning, a.points_per_ray) == (b.detector_binning // 2, b.points_per_ray)   # 18 % 9 == 0
    (_, _, a), (_, _, b) = next(iter(step_plan(n_proj, seed, sch.total_projections, sch, start=36))), full[36]
    assert (a.detector_binning, a.points_per_ray) == (b.detector_binning, b.points_per_ray + 1)    # 36 % 4 == 0
