"""Benchmark of the fused NeCT training step on B200.

One step = one batch of rays of one projection through the whole hot path:
device randperm of the detector pixels, per-ray jitter draw, fused
sample -> encode -> MLP -> line integral -> loss -> backward (nectb_train_step),
and the Adam update of the table and the MLP (fused Adam kernel).

Default workload (N=1): the 4D dynamic cone beam, 512x512 detector (one batch
= all 262,144 pixels of a projection, each projection at its own t), 256^3
porous medium with a rising brine front and shrinking grains, 512 jittered
samples per ray, 4D hash grid of 16 levels x 2 features, 2^21 entries per
level, temporal base resolution 4, 2x64 MLP, mixed precision.  The plain fp32
path is timed on the same workload in the same process (``plain_fp32`` and
``mixed_over_plain`` in the line), and so is the mixed step with the other
backward (encodings recomputed instead of read back from the store, or the
reverse; ``other_backward``).  Inputs are seeded synthetic projections
made before the timed region.  Timing: W warm-up steps, then K steps
bracketed by a barrier and cuda synchronize, CUDA events on the launching
stream, max over ranks.  Per-step state (tables, gradients, Adam moments)
exceeds the 126 MB L2, so consecutive steps do not hit a warm L2.

Rooflines: the encoding's corner gathers and the gradient scatter's
reductions are served by the L2 (the table and one scatter pass's gradient
slice are L2-sized), so their roofs are measured here, before the timed
region, by the library's probes: random gathers of the table's entry size
from a buffer of the fp16 table's size, and random fp32 reductions of the
gradient's entry size into a buffer of one scatter pass's slice.  Achieved =
algorithmic bytes per launch (per valid sample: L * 2^d * F * 2 bytes for the
forward, L * 2^d * F * 4 bytes for the scatter) / the kernel's mean CUDA-event
launch time.  The tensor-core backward is reported against the measured bf16
peak (MLP flops per sample: the forward recompute and the two backward
products).

--impl reference times the reference path's CPU restatement (oracle/
workloads.py: the C sampler, PyTorch-CPU fp32 hash grid, MLP, autograd and
torch.optim.Adam) on the host cores, on a bounded sample of each step's rays;
it imports nothing of the product package.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "train rays/s fwd+bwd"

# what each workload is, in words, and its batch: the `config` both arms print
WORKLOAD_TEXT = {
    "c1_static_parallel": "static parallel beam 128x128 detector, 128^3 volume, S=256, hash 16x2 fp32 2^19, MLP 2x64",
    "c2_static_cone": "static cone beam 512x512 detector (DSO 500, DSD 1000), 256^3 volume, S=512, hash 16x2 2^20, "
                      "MLP 2x64",
    "c3_dynamic_cone": "4D cone beam 512x512 detector (DSO 500, DSD 1000), 256^3 volume, 3,600 views over 10 turns "
                       "each at its own t, S=512, 4D hash 16x2 2^21 temporal base 4, MLP 2x64",
    "c5_large_cone": "large 4D cylindrical cone beam 2048x2048 detector (DSO 2000, DSD 4000), 1024^3 volume, 7,200 "
                     "views over 20 turns, S<=1024, 4D hash 16x4 2^22 finest 4096, MLP 3x64",
}
WORKLOAD_RAYS = {"c1_static_parallel": 65536, "c2_static_cone": 1 << 18, "c3_dynamic_cone": 1 << 18,
                 "c5_large_cone": 1 << 20}
WORKLOAD_S = {"c1_static_parallel": 256, "c2_static_cone": 512, "c3_dynamic_cone": 512, "c5_large_cone": 1024}


def bench_config(name: str, rays: int) -> dict:
    return {"workload": f"{name}: {WORKLOAD_TEXT[name]}", "rays_per_step": rays, "samples_per_ray": WORKLOAD_S[name],
            "l2": "per-step state (tables, gradients, Adam moments) exceeds the 126 MB L2"}


# ----------------------------------------------------------------- workloads
def workload_spec(name: str, precision: str):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig

    if name == "c2_static_cone":
        geo = dict(nDetector=[512, 512], dDetector=[1.0, 1.0], mode="cone", DSD=1000.0, DSO=500.0,
                   nVoxel=[256, 256, 256], dVoxel=[1.0, 1.0, 1.0])
        enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=20, base_resolution=16,
                                max_resolution_factor=2.0, nDetector=[512, 512], nVoxel=[256] * 3)
        return dict(geo=geo, model=ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), precision),
                    S=512, rays=1 << 18, n_angles=720, turns=1, phantom="porous", n_dims=3)
    if name == "c1_static_parallel":
        geo = dict(nDetector=[128, 128], dDetector=[1 / 128, 1 / 128], mode="parallel", nVoxel=[128] * 3,
                   dVoxel=[1 / 128] * 3)
        enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=19, base_resolution=16,
                                finest_resolution=1024)
        return dict(geo=geo, model=ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), precision),
                    S=256, rays=65536, n_angles=180, turns=0.5, phantom="ellipsoids", n_dims=3)
    if name == "c3_dynamic_cone":
        geo = dict(nDetector=[512, 512], dDetector=[1.0, 1.0], mode="cone", DSD=1000.0, DSO=500.0,
                   nVoxel=[256, 256, 256], dVoxel=[1.0, 1.0, 1.0])
        enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=21, base_resolution=16,
                                max_resolution_factor=2.0, nDetector=[512, 512], base_resolution_t=4)
        return dict(geo=geo, model=ModelConfig("hash_grid_4d", enc, MLPNetConfig(n_hidden_layers=2), precision),
                    S=512, rays=1 << 18, n_angles=3600, turns=10, phantom="dynamic", n_dims=4)
    if name == "c5_large_cone":
        # 2048^2 detector, object 1024 voxels across at magnification 2, cylindrical clipping
        geo = dict(nDetector=[2048, 2048], dDetector=[1.0, 1.0], mode="cone", DSD=4000.0, DSO=2000.0,
                   nVoxel=[1024, 1024, 1024], dVoxel=[1.0, 1.0, 1.0], reconstruction_mode="cylindrical")
        enc = HashEncoderConfig(n_levels=16, n_features_per_level=4, log2_hashmap_size=22, base_resolution=16,
                                finest_resolution=4096, base_resolution_t=4)
        return dict(geo=geo, model=ModelConfig("hash_grid_4d", enc, MLPNetConfig(n_hidden_layers=3), precision),
                    S=1024, rays=1 << 20, n_angles=7200, turns=20, phantom="ellipsoids", n_dims=4)
    raise ValueError(name)


def make_projections(spec, geometry, n_proj: int, device, seed: int = 0):
    from nect_b200 import phantoms

    angles_all = np.linspace(0, 2 * math.pi * spec["turns"], spec["n_angles"], endpoint=False)
    idx = np.linspace(0, spec["n_angles"] - 1, n_proj).astype(int)
    angles = angles_all[idx]
    ts = idx / max(spec["n_angles"] - 1, 1)
    if spec["phantom"] == "ellipsoids":
        ph = phantoms.ellipsoid_phantom(20, seed, size=geometry.sVoxel[0])   # the large 4D workload: 1024 voxels
        projs = torch.stack([phantoms.ellipsoid_projection(ph, geometry, float(a), device) for a in angles])
    elif spec["phantom"] == "dynamic":
        # each projection at its own t; Poisson noise at 1e4 incident photons
        ph = phantoms.dynamic_porous(geometry.nVoxel[0], seed=seed, attempts=8000)
        projs = torch.stack([phantoms.dynamic_porous_projection(ph, geometry, float(a), float(t), device)
                             for a, t in zip(angles, ts)])
        projs = phantoms.poisson_projections(projs, geometry.nVoxel[0], seed=seed)
    else:
        ph = phantoms.porous_phantom(geometry.nVoxel[0], seed=seed, attempts=8000)
        projs = torch.stack([phantoms.porous_projection(ph, geometry, float(a), device) for a in angles])
    projs, _, _ = phantoms.minmax_scale(projs)
    return projs.reshape(n_proj, -1).contiguous(), [float(a) for a in angles], [float(t) for t in ts]


# ------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        under_load = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(under_load)) if under_load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU baseline


# ------------------------------------------------------------ CPU baseline
def run_cpu_port(name: str, steps: int, warmup: int, rays: int, seed: int = 0):
    """The reference path's CPU restatement (oracle/workloads.CpuTrainer) on a
    bounded sample of ``rays`` rays per step; all host threads.  Returns
    (rays/s, threads, seconds per step).  Projections are seeded uniform
    values in [0, 1) (the min-max scaled range): the CPU time does not depend
    on them."""
    from oracle import workloads as owl

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    w = owl.WORKLOADS[name]
    tr = owl.CpuTrainer(w)
    g = torch.Generator().manual_seed(seed)
    projs = torch.rand(2, w.pixels, generator=g)
    angles, ts = owl.view_angles(w, 2)
    for k in range(warmup):
        tr.step(projs[k % 2], angles[k % 2], ts[k % 2], rays)
    t0 = time.perf_counter()
    for k in range(steps):
        tr.step(projs[k % 2], angles[k % 2], ts[k % 2], rays)
    dt = time.perf_counter() - t0
    return rays * steps / dt, threads, dt / steps


def run_reference(args):
    """--impl reference: the CPU arm alone (rank 0), product package untouched."""
    name = args.workload
    rays = args.cpu_rays
    val, threads, per = run_cpu_port(name, args.steps, args.warmup, rays)
    R = args.rays or WORKLOAD_RAYS[name]
    sample = (f"{rays} of the {R} rays x {WORKLOAD_S[name]} samples of each step's batch, {args.steps} steps "
              f"after {args.warmup} warm-up (C sampler + PyTorch-CPU fp32 hash grid/MLP/autograd/torch.optim.Adam)")
    print(json.dumps({
        "metric": METRIC, "value": val, "unit": "rays/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded projection values)",
        "config": bench_config(name, R), "precision": "plain_fp32 on the host cores",
        "cpu_baseline": {"value": val, "unit": "rays/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ----------------------------------------------------------------- GPU arm
PROFILE_SLOTS = ["ray_prep", "forward", "backward", "adam", "sample", "model_forward", "scatter", "ray_order",
                 "time_slice"]


def collect_profile():
    from nect_b200 import _lib
    import ctypes

    n = (ctypes.c_int32 * len(PROFILE_SLOTS))()
    ms = (ctypes.c_double * len(PROFILE_SLOTS))()
    _lib.lib.nectb_profile_collect(ctypes.addressof(n), ctypes.addressof(ms))
    return {PROFILE_SLOTS[i]: (int(n[i]), float(ms[i])) for i in range(len(PROFILE_SLOTS)) if n[i]}


def valid_samples(trainer, batches) -> int:
    """Sum of per-ray sample counts of the timed batches (the sampler's counts,
    identical by construction to what the fused kernels regenerate)."""
    from nect_b200.sampling import ct_sampling

    total = 0
    for b in batches:
        _, _, counts = ct_sampling.sample_with_draws(b.perm, trainer.c_geometry, b.angle, b.points_per_ray,
                                                     b.num_rays, b.start, b.max_ray_distance_per_point, True,
                                                     b.jitter, b.detector_offset, want_points=False,
                                                     want_counts=True)
        total += int(counts.sum().item())
    return total


def probe_roofs(table_entries: int, entry_bytes: int, slice_entries: int, grad_entry_bytes: int, device) -> dict:
    """Measured roofs (GB/s of the bytes each access moves) of the memory
    system under the kernels' access kinds, on buffers the size of the fp16
    table (gathers) and of one scatter pass's fp32 gradient slice
    (reductions): random entries of the table's entry size, random whole
    32-byte sectors, random whole lines (a warp's 32 consecutive entries), and
    for reductions random entries, random 16-byte pairs and random lines of
    16-byte reductions.  Library probes (nectb_probe_gather/_reduce), CUDA
    events on the launching stream, best of 3 after a warm-up."""
    from nect_b200 import _lib

    stream = torch.cuda.current_stream(device)
    sink = torch.zeros(1, dtype=torch.int32, device=device)
    table_bytes = table_entries * entry_bytes
    slice_bytes = slice_entries * grad_entry_bytes
    runs = {   # name: (kind, buffer bytes, access bytes, mode)
        "gather_entry": ("gather", table_bytes, entry_bytes, 0),
        "gather_sector": ("gather", table_bytes, 32, 0),
        "gather_line": ("gather", table_bytes, entry_bytes, 1),
        "reduce_entry": ("reduce", slice_bytes, grad_entry_bytes, 0),
        "reduce_pair": ("reduce", slice_bytes, 16, 0),
        "reduce_line": ("reduce", slice_bytes, 16, 1),
    }
    out = {}
    n_ops = 1 << 28
    ops = _lib.lib.nectb_probe_ops(n_ops)
    for name, (kind, nbytes, eb, mode) in runs.items():
        n_ent = nbytes // eb
        buf = torch.zeros(n_ent * eb // 4, device=device)
        best = None
        for rep in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if kind == "gather":
                rc = _lib.lib.nectb_probe_gather(buf.data_ptr(), n_ent, eb, mode, n_ops, sink.data_ptr(),
                                                 _lib.stream_ptr(device))
            else:
                rc = _lib.lib.nectb_probe_reduce(buf.data_ptr(), n_ent, eb, mode, n_ops, _lib.stream_ptr(device))
            e1.record(stream)
            _lib.check(rc, f"nectb_probe_{kind}")
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            if rep and (best is None or ms < best):
                best = ms
        out[name] = {"gbs": ops * eb / (best / 1e3) / 1e9, "access_bytes": eb, "buffer_mb": n_ent * eb / 1e6,
                     "pattern": "random lines of 32 consecutive entries per warp" if mode else "random entry per lane",
                     "ops": int(ops), "ms": best}
        del buf
    return out


def time_steps(trainer, make_step_batch, steps: int, first: int, world: int, clocks=None, nvtx: str | None = None):
    """K training steps between a barrier + synchronize on both sides, timed
    with CUDA events on the launching stream (max over ranks)."""
    batches = []
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)   # ncu --nvtx --nvtx-include "timed/" lists only these launches
    ev0.record(stream)
    for k in range(steps):
        b = make_step_batch(first + k)
        batches.append(b)
        trainer.step(b)
    ev1.record(stream)
    if nvtx:
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        import torch.distributed as dist

        t_ = torch.tensor([ms], device="cuda")
        dist.all_reduce(t_, op=dist.ReduceOp.MAX)
        ms = float(t_.item())
    return ms, batches


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c3_dynamic_cone",
                    choices=["c3_dynamic_cone", "c2_static_cone", "c1_static_parallel", "c5_large_cone"])
    ap.add_argument("--precision", default=os.environ.get("NECTB_PRECISION", "mixed"),
                    choices=["mixed", "plain_fp32"])
    ap.add_argument("--cpu-rays", type=int, default=2048)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain fp32 arm")
    ap.add_argument("--plain-steps", type=int, default=0,
                    help="timed steps of the plain fp32 arm (0: --steps, 2 on the large 4D workload)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-other-backward", action="store_true",
                    help="skip timing the other backward (recompute vs encoding store) on the same trainer")
    ap.add_argument("--rays", type=int, default=0, help="override rays per step (profiling of smaller cases)")
    ap.add_argument("--encoding-store", default="auto", choices=["auto", "on", "off"],
                    help="off: the mixed backward recomputes the encodings instead of reading the rows the forward "
                         "stored (encoding_store 0); auto: off on the large 4D workload, on elsewhere")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner (launch shapes and scheduling tuned on this workload before the "
                         "warm-up, outside the timed region); the library defaults are used")
    ap.add_argument("--tuning", default="",
                    help="launch-shape settings KEY=VALUE[,KEY=VALUE] (NectbTuning fields) applied after the "
                         "autotuner, e.g. forward_blocks_per_sm=4")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from nect_b200 import _lib, autotune
    from nect_b200.config import get_model
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    spec = workload_spec(args.workload, args.precision)
    geometry = Geometry(**spec["geo"])
    S, R = spec["S"], (args.rays or spec["rays"])
    model_cfg = spec["model"]
    recompute = args.encoding_store == "off" or (args.encoding_store == "auto" and args.workload == "c5_large_cone")
    autotune.set_tuning({"encoding_store": 0 if recompute else 1})

    torch.manual_seed(1234 + rank)
    n_proj = 8
    projs, angles, ts = make_projections(spec, geometry, n_proj, dev, seed=rank)
    P = projs.shape[1]

    def make_trainer(cfg):
        model = get_model(cfg, device=dev)
        # N > 1: data parallel as the reference's DDP: each rank trains on its own projections (weak scaling) and
        # the table and MLP gradients are averaged over NCCL before every Adam step
        tr = Trainer(model, geometry, points_per_batch=R * S, points_per_ray=S, loss="l2", lr=1e-3, device=dev,
                     data_parallel=world > 1)

        def make_step_batch(k):
            perm = torch.randperm(P, dtype=torch.int64, device=dev)
            return tr.make_batch(perm, 0, angles[k % n_proj], projs[k % n_proj], ts[k % n_proj])

        return model, tr, make_step_batch

    model, trainer, make_step_batch = make_trainer(model_cfg)
    tuning = None
    if not args.no_autotune and args.precision == "mixed":   # the tunables belong to the mixed path
        # every rank tunes on its own GPU without the gradient all-reduce (the
        # search may take different numbers of steps on different ranks, and a
        # collective needs all of them), then all ranks take rank 0's choice
        trainer.data_parallel = False
        tuning = autotune.tune(trainer, make_step_batch, steps=3, warmup=2)
        trainer.data_parallel = world > 1
        if world > 1:
            import torch.distributed as dist

            chosen = [tuning]
            dist.broadcast_object_list(chosen, src=0)
            tuning = chosen[0]
            autotune.set_tuning(tuning)
    if args.tuning:
        cur = autotune.get_tuning()
        for kv in args.tuning.split(","):
            key, val = (x.strip() for x in kv.split("="))
            cur[key] = int(float(val)) if isinstance(cur[key], int) else float(val)
        autotune.set_tuning(cur)
    for k in range(args.warmup):
        trainer.step(make_step_batch(k))
    torch.cuda.synchronize()

    # ---- roofs of the gathers and reductions, measured on this GPU (outside the timed region)
    enc = model_cfg.encoder
    F = enc.n_features_per_level
    feat_bytes = 2 if args.precision == "mixed" else 4
    cur = autotune.get_tuning()
    slice_entries = max(64, min(model.table.shape[0], int(cur["scatter_group_bytes"]) // (F * 4)))
    roofs = probe_roofs(model.table.shape[0], F * feat_bytes, slice_entries, F * 4, dev)

    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    time.sleep(0.3)
    _lib.lib.nectb_profile_enable(1)
    ms, batches = time_steps(trainer, make_step_batch, args.steps, args.warmup, world, nvtx="timed")
    _lib.lib.nectb_profile_enable(0)
    clock_info = clocks.stop()
    prof = collect_profile()
    rays_per_step = batches[0].num_rays
    value = world * rays_per_step * args.steps / (ms / 1e3)

    # ---- rooflines (algorithmic bytes or flops per launch / mean launch time)
    n_valid = valid_samples(trainer, batches)
    per_step_samples = n_valid / args.steps
    corners = 1 << spec["n_dims"]
    L = enc.n_levels
    gather = L * corners * F * feat_bytes       # corner gathers of one sample
    scatter = L * corners * F * 4               # fp32 gradient reductions of one sample
    H = model_cfg.net.n_hidden_layers
    n_in = L * F
    mlp_fwd = 2 * (n_in * 64 + (H - 1) * 64 * 64 + 64)
    kernel_ms = {k: v[1] / max(v[0], 1) for k, v in prof.items()}
    launches_per_step = {k: v[0] / args.steps for k, v in prof.items()}
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    tensor_peak = float(peaks.get("bf16_tflops_sustained", 1400.0))
    peak_src = "of measured" if peaks else "of fallback"
    traffic_step = {}   # DRAM bytes per step and kernel kind (an ncu capture of a small case, scaled per sample)
    tfile = ROOT / "profiles" / "dram_bytes_per_sample.txt"
    if tfile.exists():
        for line in tfile.read_text().splitlines():
            f = line.split()
            if len(f) == 4 and not line.startswith("#") and f[:2] == [args.workload, args.precision]:
                traffic_step[f[2]] = float(f[3]) * per_step_samples

    l2_step = {}   # L2 bytes per step and kernel kind (lts__t_bytes.sum of an ncu capture, scaled per sample)
    lfile = ROOT / "profiles" / "l2_bytes_per_sample.txt"
    if lfile.exists():
        for line in lfile.read_text().splitlines():
            f = line.split()
            if len(f) == 4 and not line.startswith("#") and f[:2] == [args.workload, args.precision]:
                l2_step[f[2]] = float(f[3]) * per_step_samples

    # the 4D mixed step gathers and reduces on the time slice: 8 spatial corners per level, half of the
    # 16 the 4D interpolation counts (the time blend runs once per table entry and step instead)
    sliced = spec["n_dims"] == 4 and args.precision == "mixed" and bool(autotune.get_tuning()["time_slice"])
    executed = {"forward": gather // 2 if sliced else gather, "scatter": scatter // 2 if sliced else scatter}

    def roof(kind, per_sample, peak_name, bound, unit, scale, peak=None, peak_src=None):
        if kind not in kernel_ms:
            return None
        per_launch = per_step_samples * per_sample / launches_per_step[kind]
        secs = kernel_ms[kind] / 1e3
        achieved = per_launch / secs / scale
        if peak is None:
            peak, peak_src = roofs[peak_name]["gbs"], f"measured in this run: {peak_name} probe ({roofs[peak_name]['pattern']}, {roofs[peak_name]['access_bytes']} B, {roofs[peak_name]['buffer_mb']:.0f} MB buffer)"
        tr = traffic_step.get(kind)
        out = {"bound": bound, "kernel": kind, "achieved": achieved, "peak": peak, "unit": unit,
               "frac": achieved / peak, "peak_source": peak_src,
               "traffic": tr / launches_per_step[kind] if tr is not None else None,
               "algorithmic_per_launch": per_launch, "launch_ms": kernel_ms[kind],
               "launches_per_step": launches_per_step[kind]}
        if kind in executed:   # the bytes the kernel's own algorithm moves (time slice: 8 corners)
            ex = per_step_samples * executed[kind] / launches_per_step[kind]
            out["executed_per_launch"] = ex
            out["executed_frac"] = ex / secs / scale / peak
        if tr is not None:
            out["dram_gbs"] = tr / launches_per_step[kind] / secs / 1e9
            out["dram_frac_of_hbm"] = out["dram_gbs"] / hbm
        if kind in l2_step and bound == "l2":
            out["l2_gbs"] = l2_step[kind] / launches_per_step[kind] / secs / 1e9
            out["l2_frac"] = out["l2_gbs"] / peak
        return out

    rooflines = {
        "forward": roof("forward", gather, "gather_line", "l2", "GB/s", 1e9),
        "scatter": roof("scatter", scatter, "reduce_line", "l2", "GB/s", 1e9),
        "backward": roof("backward", 3 * mlp_fwd, None, "tensor", "TFLOP/s", 1e12, tensor_peak,
                         f"{peak_src} bf16 dense, sustained"),
    }
    if args.precision == "plain_fp32":
        rooflines["backward"] = None   # the plain backward is SIMT, no tensor-core roof
    rooflines = {k: v for k, v in rooflines.items() if v}
    # the dominant kernel of the step (most time)
    dominant = max((k for k in rooflines), key=lambda k: prof[k][1])
    roofline = dict(rooflines[dominant])

    # ---- end to end through the public API, host buffers (pinned projection in, loss out)
    e2e = None
    if not args.no_e2e:
        host = projs.cpu().pin_memory()
        dproj = torch.empty_like(projs[0])
        loss_host = torch.empty(1, pin_memory=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            dproj.copy_(host[k % n_proj], non_blocking=True)
            loss = trainer.train_projection(dproj, angles[k % n_proj], ts[k % n_proj])
            loss_host.copy_(loss, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            t_ = torch.tensor([ems], device=dev)
            dist.all_reduce(t_, op=dist.ReduceOp.MAX)
            ems = float(t_.item())
        e2e = {"value": world * rays_per_step * args.steps / (ems / 1e3), "unit": "rays/s",
               "h2d_bytes_per_step": int(P * 4), "d2h_bytes_per_step": 4}

    # ---- the other backward (encodings recomputed, or read from the store) on the same trainer
    other = None
    if args.precision == "mixed" and not args.no_other_backward and args.workload != "c5_large_cone":
        autotune.set_tuning({"encoding_store": 1 if recompute else 0})
        for k in range(2):
            trainer.step(make_step_batch(k))
        oms, _ = time_steps(trainer, make_step_batch, args.steps, 2, world)
        other = {"backward": "encoding store" if recompute else "recompute (encodings gathered again)",
                 "value": world * rays_per_step * args.steps / (oms / 1e3), "unit": "rays/s",
                 "ms_per_step": oms / args.steps}
        autotune.set_tuning({"encoding_store": 0 if recompute else 1})

    # ---- the plain fp32 path on the same workload, same process
    plain = None
    if args.precision == "mixed" and not args.no_plain:
        del trainer, model
        torch.cuda.empty_cache()
        pcfg = workload_spec(args.workload, "plain_fp32")["model"]
        _, ptr, pbatch = make_trainer(pcfg)
        psteps = args.plain_steps or (2 if args.workload == "c5_large_cone" else args.steps)
        pwarm = min(args.warmup, 3 if args.workload != "c5_large_cone" else 1)
        for k in range(pwarm):
            ptr.step(pbatch(k))
        pms, _ = time_steps(ptr, pbatch, psteps, pwarm, world)
        pval = world * rays_per_step * psteps / (pms / 1e3)
        plain = {"value": pval, "unit": "rays/s", "ms_per_step": pms / psteps, "steps": psteps, "warmup": pwarm}
        del ptr
        torch.cuda.empty_cache()

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu:
        val, threads, per = run_cpu_port(args.workload, args.cpu_steps, 1, args.cpu_rays)
        cpu_baseline = {"value": val, "unit": "rays/s", "cores": threads, "kind": "port",
                        "sample": f"{args.cpu_rays} of the {rays_per_step} rays x {S} samples of each step's batch, "
                                  f"{args.cpu_steps} steps (C sampler + PyTorch-CPU fp32 hash grid/MLP/autograd/"
                                  f"torch.optim.Adam)"}

    # the ray-order slot times its three launches (count, scan, compaction) as one
    gpu_launches = sum(v[0] * (3 if k == "ray_order" else 1) for k, v in prof.items())
    out = {
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16/bf16" if args.precision == "mixed" else "f32",
        "data": "synthetic (seeded phantom, exact or ray-marched projections)",
        "config": bench_config(args.workload, rays_per_step),
        "precision": args.precision,
        "samples_per_step": per_step_samples, "samples_per_s": world * n_valid / (ms / 1e3),
        "parallelism": f"dp{world} (gradient all-reduce per step)" if world > 1 else "single",
        "backward": "recompute (encodings gathered again)" if recompute else "encoding store",
        "tuning": tuning if tuning is not None else autotune.get_tuning(),
        "roofline": roofline,
        "rooflines": rooflines,
        "probes": roofs,
        "other_backward": other,
        "plain_fp32": plain,
        "mixed_over_plain": (value / plain["value"]) if plain else None,
        "cpu_baseline": cpu_baseline,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "clocks": clock_info,
    }
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_psnr(args):
    """Time-to-PSNR of the mixed path against the plain fp32 path at equal
    iterations on the static parallel-beam workload (128^3 phantom of 20
    ellipsoids, 180 exact projections over [0, pi) on 128^2 pixels, S = 256,
    one full projection (16,384 rays) per step, L2 loss, Adam lr 1e-3).
    PSNR (-10 log10 MSE) and 3D SSIM of the exported volume against the
    phantom; the untrained network and filtered back-projection (no learned
    model) are reported beside them."""
    from nect_b200 import phantoms
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig
    from nect_b200.reconstruct import fbp_parallel, fit, psnr, ssim3d
    from nect_b200.sampling import Geometry

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    geo = Geometry(nDetector=[128, 128], dDetector=[1 / 128, 1 / 128], mode="parallel", nVoxel=[128] * 3,
                   dVoxel=[1 / 128] * 3)
    ph = phantoms.ellipsoid_phantom(20, 0)
    angles = np.linspace(0, math.pi, 180, endpoint=False)
    projs = torch.stack([phantoms.ellipsoid_projection(ph, geo, float(a), dev) for a in angles])
    truth = phantoms.ellipsoid_volume(ph, 128, dev)
    fbp = fbp_parallel(projs, geo, angles)
    out = {"metric": "time-to-PSNR, mixed vs plain fp32 at equal iterations", "unit": "s",
           "higher_is_better": False, "n_gpus": 1, "steps": args.psnr_steps,
           "config": {"workload": "c1_static_parallel: 128^3 ellipsoid phantom, 180 views over [0,pi), 128^2 "
                                  "detector, S=256, 16,384 rays/step, hash 16x2 2^19 base 16 finest 1024, MLP 2x64, "
                                  "L2, Adam 1e-3", "data": "synthetic (seeded phantom, exact chord-length projections)"},
           "fbp": {"psnr": psnr(fbp, truth), "ssim": ssim3d(fbp, truth)}}
    runs = {}
    for precision in ("plain_fp32", "mixed"):
        enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=19, base_resolution=16,
                                finest_resolution=1024)
        cfg = ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), precision)

        def evaluate(rec):
            v = rec.volume()
            return {"psnr": psnr(v, truth), "ssim": ssim3d(v, truth)}

        rec = fit(geo, projs, angles, model_cfg=cfg, niter=args.psnr_steps, lr=1e-3, rays_per_batch=65536,
                  points_per_ray=256, loss="l2", seed=0, device=dev, evaluate=evaluate, eval_every=args.eval_every)
        runs[precision] = {"history": [(st, round(sec, 4), m["psnr"], m["ssim"]) for st, sec, m in rec.history],
                           "final_psnr": rec.history[-1][2]["psnr"], "final_ssim": rec.history[-1][2]["ssim"],
                           "untrained_psnr": rec.history[0][2]["psnr"], "train_seconds": rec.train_seconds}
    target = runs["plain_fp32"]["final_psnr"] - 0.1
    for precision, r in runs.items():
        hit = next(((st, sec) for st, sec, p_, _ in r["history"] if p_ >= target), None)
        r["time_to_target_s"] = hit[1] if hit else None
        r["steps_to_target"] = hit[0] if hit else None
    out["target_psnr"] = target
    out["runs"] = runs
    out["psnr_gap_db"] = runs["mixed"]["final_psnr"] - runs["plain_fp32"]["final_psnr"]
    out["value"] = runs["mixed"]["time_to_target_s"]
    out["plain_value"] = runs["plain_fp32"]["time_to_target_s"]
    print(json.dumps(out))


def run_serving(args):
    """Query serving of the 4D dynamic cone-beam model (16 x 2 fp16 features,
    2^21 entries per level, 2 x 64 MLP): a seeded Poisson request stream, and
    the same request classes answered one at a time by the plain fp32 model.
    Weights are seeded random values of the trained model's architecture
    (serving cost does not depend on the values)."""
    from nect_b200.config import get_model
    from nect_b200.sampling import Geometry
    from nect_b200.serving import (QueryServer, Request, query_points, reproject, reproject_workspace_bytes,
                                   slice_items, time_slice, time_slice_bytes, volume_items)

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    spec = workload_spec("c3_dynamic_cone", "mixed")
    geometry = Geometry(**spec["geo"])
    S = spec["S"]
    model = get_model(spec["model"], device=dev)
    rng = np.random.default_rng(0)
    n_req = int(args.serve_rate * args.serve_seconds)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n_req))
    reqs = []
    for k in range(n_req):
        u = rng.random()
        t = float(rng.random())
        if args.serve_mix == "no_reproject" and 0.6 <= u < 0.9:
            u = 0.0
        if u < 0.6:
            size = int(rng.choice([256, 384, 512, 768, 1024]))
            if rng.random() < 0.5:
                axis = int(rng.integers(3))
                uu, vv = [(0.0, 0.0, 1.0), (0.0, 1.0, 0.0)], None
                basis = np.eye(3)
                others = [b for b in range(3) if b != axis]
                uu, vv = tuple(basis[others[1]]), tuple(basis[others[0]])
            else:
                q = rng.normal(size=(2, 3))
                uu = q[0] / np.linalg.norm(q[0])
                vv = q[1] - (q[1] @ uu) * uu
                vv = tuple(vv / np.linalg.norm(vv))
                uu = tuple(uu)
            reqs.append(dict(kind="slice", size=size, t=t, centre=tuple(0.3 + 0.4 * rng.random(3)), u=uu, v=vv))
        elif u < 0.9:
            reqs.append(dict(kind="reproject", t=t, angle=float(rng.random() * 2 * math.pi)))
        else:
            reqs.append(dict(kind="volume", size=256, t=t))
    # the mixed model alone, one request at a time (GPU time of each class as the server launches it):
    # the load the request stream offers is sum over classes of rate x share x time
    alone = {}
    srv_slow_blocks = args.slow_blocks or 3 * torch.cuda.get_device_properties(dev).multi_processor_count
    P = geometry.nDetector[0] * geometry.nDetector[1]
    out_s, out_r, out_v = (torch.empty(512, 512, device=dev), torch.empty(P, device=dev),
                           torch.empty(256, 256, 256, device=dev))
    items_s, items_v = slice_items(out_s, out_s.shape, 0.5), volume_items(out_v, out_v.shape, 0.5)
    ws_r = torch.empty(reproject_workspace_bytes(model, geometry, args.piece_pixels), dtype=torch.uint8, device=dev)
    slc = torch.empty(max(time_slice_bytes(model), 1), dtype=torch.uint8, device=dev)
    for kind, n in (("slice", 10), ("reproject", 4), ("volume", 2)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for k in range(n + 1):
            torch.cuda.synchronize()
            e0.record()
            if kind == "slice":
                query_points(model, items_s)
            elif kind == "reproject":
                for b in range(0, P, args.piece_pixels):
                    reproject(model, geometry, 0.3 * k, 0.5, S, out=out_r, workspace=ws_r,
                              pixels=(b, min(args.piece_pixels, P - b)), warpgroups=args.slow_warpgroups)
            elif time_slice_bytes(model):   # as the server: the time slice at t, then the items on it
                time_slice(model, 0.5, out=slc)
                query_points(model, items_v, max_blocks=srv_slow_blocks, slice=slc)
            else:
                query_points(model, items_v, max_blocks=srv_slow_blocks)
            e1.record()
            torch.cuda.synchronize()
            if k:
                ms.append(e0.elapsed_time(e1))
        alone[kind] = {"n": n, "mean_ms": float(np.mean(ms))}
    mean_slice_points = float(np.mean(np.array([256, 384, 512, 768, 1024]) ** 2))
    share = {"slice": 0.6, "reproject": 0.3, "volume": 0.1}
    per_req_ms = {"slice": alone["slice"]["mean_ms"] * mean_slice_points / 512 ** 2,
                  "reproject": alone["reproject"]["mean_ms"], "volume": alone["volume"]["mean_ms"]}
    offered = args.serve_rate * sum(share[k] * per_req_ms[k] for k in share) / 1e3
    srv = QueryServer(model, geometry, memory_budget=40 << 30, points_per_ray=S, piece_pixels=args.piece_pixels,
                      slow_warpgroups=args.slow_warpgroups, slow_blocks=args.slow_blocks)
    warm = [srv.submit(Request(**d)) for d in reqs[:6]]
    for r in warm:
        r.event.wait(120)
    srv.completed.clear()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    submitted = []
    for d, ta in zip(reqs, arrivals):
        delay = t0 + ta - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        submitted.append(srv.submit(Request(**d)))
    for r in submitted:
        r.event.wait(600)
    makespan = max(r.done for r in submitted) - t0
    srv.close()
    stats = srv.latency_stats()
    s512 = np.array([r.latency_ms() for r in submitted if r.kind == "slice" and r.size == 512])
    w512 = np.array([r.wait_ms() for r in submitted if r.kind == "slice" and r.size == 512])
    voxels = sum(int(np.prod(r.out_shape(geometry))) for r in submitted)

    # one request at a time, plain fp32 model of the same architecture
    plain_cfg = workload_spec("c3_dynamic_cone", "plain_fp32")["model"]
    pm = get_model(plain_cfg, device=dev)
    base = {}
    for kind, n in (("slice", 10), ("reproject", 4), ("volume", 2)):
        lat = []
        for k in range(n + 1):
            torch.cuda.synchronize()
            a = time.perf_counter()
            if kind == "slice":
                out = torch.empty(512, 512, device=dev)
                query_points(pm, slice_items(out, out.shape, 0.5))
            elif kind == "reproject":
                out = reproject(pm, geometry, 0.3 * k, 0.5, S)
            else:
                out = torch.empty(256, 256, 256, device=dev)
                query_points(pm, volume_items(out, out.shape, 0.5))
            host = out.cpu()
            torch.cuda.synchronize()
            if k:
                lat.append((time.perf_counter() - a) * 1e3)
        base[kind] = {"n": n, "p50_ms": float(np.percentile(lat, 50))}
    print(json.dumps({
        "metric": "query latency p50/p99 (serving, 4D model)", "unit": "ms", "higher_is_better": False,
        "value": float(np.percentile(s512, 99)) if s512.size else None, "value_is": "p99 of 512^2 slices",
        "n_gpus": 1, "requests": n_req, "rate_per_s": args.serve_rate, "seconds": args.serve_seconds,
        "makespan_s": makespan, "voxels_per_s": voxels / makespan, "classes": stats,
        "slice512": {"n": int(s512.size), "p50_ms": float(np.percentile(s512, 50)) if s512.size else None,
                     "p99_ms": float(np.percentile(s512, 99)) if s512.size else None,
                     "wait_p99_ms": float(np.percentile(w512, 99)) if w512.size else None},
        "one_at_a_time_plain_fp32": base,
        "one_at_a_time_mixed_gpu_ms": alone,
        "offered_gpu_load": offered, "offered_gpu_load_is": "GPU-seconds per second the request stream asks for "
                                                            "(rate x class share x the class's GPU time alone); "
                                                            "above 1 no schedule keeps up",
        "server": {"piece_pixels": args.piece_pixels, "slow_warpgroups": args.slow_warpgroups,
                   "slow_blocks": args.slow_blocks},
        "config": {"workload": "4D cone 512x512, 2^21 x 16 x 2 fp16, MLP 2x64 (bf16 tensor cores); requests: "
                               "60% slices 256^2-1024^2 axis/oblique, 30% re-projections 512^2 (S=512), "
                               "10% volumes 256^3, random t; 40 GB admission budget",
                   "data": "synthetic (seeded random weights of the trained architecture)"},
    }))


def run_psnr4d(args):
    """Reconstruction quality of the 4D cone workload, mixed against plain fp32
    at equal iterations: the dynamic porous phantom (brine front, shrinking
    grains), ``--views`` projections spread over the 10 turns, each at its own
    t, Poisson noise at 1e4 incident photons, one full 512^2 projection per
    step (262,144 rays, S = 512), L2, Adam 1e-3.  PSNR (-10 log10 MSE) of the
    exported 256^3 volume against the phantom, averaged over t = 0.2, 0.5,
    0.8, with the training seconds at each evaluation (the exported volume
    without the export's offset of the projections' minimum)."""
    from nect_b200 import phantoms
    from nect_b200.reconstruct import fit, psnr
    from nect_b200.sampling import Geometry

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    spec = workload_spec("c3_dynamic_cone", "mixed")
    geometry = Geometry(**spec["geo"])
    n = geometry.nVoxel[0]
    all_angles = np.linspace(0, 2 * math.pi * spec["turns"], spec["n_angles"], endpoint=False)
    idx = np.linspace(0, spec["n_angles"] - 1, args.views).astype(int)
    angles, ts = all_angles[idx], idx / (spec["n_angles"] - 1)
    ph = phantoms.dynamic_porous(n, seed=0)
    projs = torch.stack([phantoms.dynamic_porous_projection(ph, geometry, float(a), float(t), dev)
                         for a, t in zip(angles, ts)])
    projs = phantoms.poisson_projections(projs, n, seed=0)
    t_eval = (0.2, 0.5, 0.8)
    truths = {t: phantoms.dynamic_porous_volume(ph, n, t, dev) for t in t_eval}

    # Every ray of this geometry crosses the object, so the data set's minimum (the line integral of the
    # shortest chord) is well above 0, and the export adds it to every voxel (sigma * (max - min) /
    # max_distance_traveled + min, nect/static_export.py:139-140).  The PSNR is taken on the attenuation
    # sigma * (max - min) / max_distance_traveled, the export without that offset.
    def evaluate(rec):
        return {"psnr": float(np.mean([psnr(rec.volume(t) - rec.minimum, truths[t]) for t in t_eval]))}

    out = {"metric": "4D reconstruction PSNR, mixed vs plain fp32 at equal iterations", "unit": "dB",
           "higher_is_better": True, "n_gpus": 1, "steps": args.psnr_steps, "views": args.views,
           "config": bench_config("c3_dynamic_cone", spec["rays"]),
           "data": "synthetic (seeded dynamic porous phantom, ray-marched front, Poisson noise)"}
    runs = {}
    for precision in ("plain_fp32", "mixed"):
        cfg = workload_spec("c3_dynamic_cone", precision)["model"]
        rec = fit(geometry, projs, list(angles), timesteps=list(ts), model_cfg=cfg, niter=args.psnr_steps, lr=1e-3,
                  rays_per_batch=spec["rays"], points_per_ray=spec["S"], loss="l2", seed=0, device=dev,
                  evaluate=evaluate, eval_every=args.eval_every)
        runs[precision] = {"history": [(st, round(sec, 3), m["psnr"]) for st, sec, m in rec.history],
                           "final_psnr": rec.history[-1][2]["psnr"], "train_seconds": rec.train_seconds}
        del rec
        torch.cuda.empty_cache()
    target = runs["plain_fp32"]["final_psnr"] - 0.1
    for r in runs.values():
        hit = next(((st, sec) for st, sec, p_ in r["history"] if p_ >= target), None)
        r["time_to_target_s"] = hit[1] if hit else None
    out["runs"] = runs
    out["projection_min"] = float(projs.min())
    out["target_psnr"] = target
    out["psnr_gap_db"] = runs["mixed"]["final_psnr"] - runs["plain_fp32"]["final_psnr"]
    out["value"] = runs["mixed"]["final_psnr"]
    out["train_seconds_ratio"] = runs["plain_fp32"]["train_seconds"] / runs["mixed"]["train_seconds"]
    print(json.dumps(out))


def run_quadcubes(args):
    """Training throughput of the reference's default dynamic model, QuadCubes
    (nect/cfg/dynamic/quadcubes.yaml: four 3D grids of 23 levels x 4 features,
    2^23 entries, the raw inputs appended, 4 x 128 LeakyReLU MLP) on the 4D cone
    workload's geometry and projections, through the module loop
    (quadcubes.ModuleTrainer: the library's sampler and encoder kernels, the MLP
    on cuBLAS, the library's Adam), at the reference's 5 M points per batch; the
    fused single-4D-grid model's line is the default bench."""
    from nect_b200.config import get_model
    from nect_b200.quadcubes import ModuleTrainer
    from nect_b200.reconstruct import default_model_config
    from nect_b200.sampling import Geometry

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    spec = workload_spec("c3_dynamic_cone", "mixed")
    geometry = Geometry(**spec["geo"])
    S = spec["S"]
    cfg = default_model_config(geometry, "dynamic", args.precision, log2_hashmap_size=23)
    model = get_model(cfg, device=dev)
    projs, angles, ts = make_projections(spec, geometry, 8, dev)
    tr = ModuleTrainer(model, geometry, points_per_batch=5_000_000, points_per_ray=S, loss="l2", lr=2e-4, device=dev)
    P = projs.shape[1]

    def batch(k):
        perm = torch.randperm(P, dtype=torch.int64, device=dev)
        return tr.make_batch(perm, 0, angles[k % len(angles)], projs[k % len(angles)], ts[k % len(angles)])

    # the module loop's tensors change size with each batch's count of
    # non-zero points: the caching allocator grows for the first few steps
    warmup = max(args.warmup, 8)
    for k in range(warmup):
        tr.step(batch(k))
    ms, _ = time_steps(tr, batch, args.steps, warmup, 1, nvtx="timed")
    rays = tr.batch_size
    params = sum(p.numel() for p in model.parameters())
    print(json.dumps({
        "metric": "train rays/s fwd+bwd, the reference's default dynamic model (QuadCubes) through the module loop",
        "value": rays * args.steps / (ms / 1e3), "unit": "rays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "precision": args.precision,
        "rays_per_step": rays, "samples_per_ray": S, "parameters": params,
        "config": {"workload": "c3_dynamic_cone geometry and projections; QuadCubes 4 x (23 levels x 4 features, "
                               "2^23), identity inputs, MLP 4 x 128 LeakyReLU, 5 M points per batch"},
        "data": "synthetic (seeded dynamic porous phantom)"}))


def run_scan(args):
    """Continuous-scan training steps (nect/trainers/continous_scanning_trainer.py:
    85-140) on the 4D cone workload: each step's prediction averages k
    sub-angles of the same 262,144 pixels.  The fused step (every sub-angle's
    rays in one launch of each kernel) is timed beside the per-sub-angle
    version (one forward and backward per sub-angle), same draws, CUDA events
    on the training stream after warm-up."""
    from nect_b200.config import get_model
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    spec = workload_spec("c3_dynamic_cone", "mixed")
    geometry = Geometry(**spec["geo"])
    S, R, k = spec["S"], spec["rays"], args.sub_angles
    torch.manual_seed(0)
    projs, angles, ts = make_projections(spec, geometry, 4, dev)
    step_angle = 2 * math.pi * spec["turns"] / spec["n_angles"]
    out = {"metric": "continuous-scan train rays/s fwd+bwd (pixels per step x steps / time)", "unit": "rays/s",
           "higher_is_better": True, "n_gpus": 1, "sub_angles": k, "steps": args.steps,
           "config": bench_config("c3_dynamic_cone", R), "data": "synthetic"}
    for fused in (True, False):
        model = get_model(spec["model"], device=dev)
        tr = Trainer(model, geometry, points_per_batch=R * S, points_per_ray=S, loss="l2", lr=1e-3, device=dev)
        P = projs.shape[1]

        def step(i):
            perm = torch.randperm(P, dtype=torch.int64, device=dev)
            a0 = angles[i % 4]
            return tr.continuous_step(perm, 0, a0, a0 + step_angle, projs[i % 4], ts[i % 4], accumulation_steps=k,
                                      fused=fused)

        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            step(args.warmup + i)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out["fused" if fused else "per_sub_angle"] = {"ms_per_step": ms, "value": R / (ms / 1e3)}
        del tr, model
        torch.cuda.empty_cache()
    out["value"] = out["fused"]["value"]
    out["fused_over_per_sub_angle"] = out["per_sub_angle"]["ms_per_step"] / out["fused"]["ms_per_step"]
    print(json.dumps(out))


if __name__ == "__main__":
    if "--quadcubes" in sys.argv:
        ap = argparse.ArgumentParser()
        ap.add_argument("--quadcubes", action="store_true")
        ap.add_argument("--steps", type=int, default=10)
        ap.add_argument("--warmup", type=int, default=3)
        ap.add_argument("--precision", default="mixed", choices=["mixed", "plain_fp32"])
        run_quadcubes(ap.parse_args())
    elif "--scan" in sys.argv:
        ap = argparse.ArgumentParser()
        ap.add_argument("--scan", action="store_true")
        ap.add_argument("--sub-angles", type=int, default=4)
        ap.add_argument("--steps", type=int, default=10)
        ap.add_argument("--warmup", type=int, default=3)
        run_scan(ap.parse_args())
    elif "--psnr4d" in sys.argv:
        ap = argparse.ArgumentParser()
        ap.add_argument("--psnr4d", action="store_true")
        ap.add_argument("--psnr-steps", type=int, default=240)
        ap.add_argument("--views", type=int, default=60)
        ap.add_argument("--eval-every", type=int, default=60)
        run_psnr4d(ap.parse_args())
    elif "--psnr" in sys.argv:
        ap = argparse.ArgumentParser()
        ap.add_argument("--psnr", action="store_true")
        ap.add_argument("--psnr-steps", type=int, default=2000)
        ap.add_argument("--eval-every", type=int, default=100)
        run_psnr(ap.parse_args())
    elif "--serving" in sys.argv:
        ap = argparse.ArgumentParser()
        ap.add_argument("--serving", action="store_true")
        ap.add_argument("--serve-rate", type=float, default=200.0)
        ap.add_argument("--serve-seconds", type=float, default=5.0)
        ap.add_argument("--serve-mix", default="full", choices=["full", "no_reproject"])
        ap.add_argument("--piece-pixels", type=int, default=16384)
        ap.add_argument("--slow-warpgroups", type=int, default=4)
        ap.add_argument("--slow-blocks", type=int, default=None)
        run_serving(ap.parse_args())
    else:
        main()
