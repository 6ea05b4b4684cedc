"""Launch shapes and scheduling of the mixed training path, tuned per workload.

The library's tunables (NectbTuning, include/nectb.h): blocks per SM of the
forward, of the tensor-core backward and of the gradient scatter, the rounds
of the two-pass backward, the gradient slice one scatter pass covers and the
run-merging thresholds.  None changes results beyond fp32 reassociation.
``tune`` runs coordinate descent over them on real training steps of the
caller's workload (CUDA-event timing on the training stream), keeps the
fastest setting in the library and returns it; the model and optimizer state
are restored afterwards.  Results can be cached in a JSON file keyed by the
workload (model layout, batch shape, detector and GPU).
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

import torch

from . import _lib

FIELDS = ("forward_blocks_per_sm", "backward_blocks_per_sm", "scatter_blocks_per_sm", "staged_rounds",
          "scatter_group_bytes", "run_threshold_3d", "run_threshold_4d", "time_slice", "encoding_store")

# candidates per tunable, tried one tunable at a time
SPACE = {
    "forward_blocks_per_sm": (4, 5, 6),
    "backward_blocks_per_sm": (2, 3),
    "scatter_blocks_per_sm": (0, 2, 3),
    "staged_rounds": (4, 8, 16),
    "scatter_group_bytes": (24 << 20, 48 << 20, 96 << 20),
    "run_threshold_3d": (0.5, 0.75, 1.0),
    "run_threshold_4d": (0.75, 1.5, 3.0),
}


def get_tuning() -> dict:
    t = _lib.NectbTuning()
    _lib.check(_lib.lib.nectb_get_tuning(ctypes.byref(t)), "nectb_get_tuning")
    return {f: getattr(t, f) for f in FIELDS}


def set_tuning(values: dict) -> None:
    cur = get_tuning()
    cur.update(values)
    t = _lib.NectbTuning(**{f: cur[f] for f in FIELDS})
    _lib.check(_lib.lib.nectb_set_tuning(ctypes.byref(t)), "nectb_set_tuning")


def workload_key(trainer, num_rays: int) -> str:
    m = trainer.model
    g, p = m.grid_desc, m.mlp_desc
    dev = torch.cuda.get_device_name(trainer.device)
    return (f"{dev}|d{g.n_dims} L{g.n_levels} F{g.n_features} T2^{g.log2_hashmap_size} b{g.base_resolution:g} "
            f"s{g.per_level_scale:.6f}|H{p.n_hidden_layers} W{p.width} {m.precision}|R{num_rays} "
            f"S{trainer.points_per_ray}|det{tuple(trainer.geometry.nDetector)} {trainer.geometry.mode}")


def _time_steps(trainer, make_batch, steps: int, warmup: int) -> float:
    from .trainer import Workspace

    trainer.workspace = Workspace()   # the staging size follows staged_rounds
    for k in range(warmup):
        trainer.step(make_batch(k))
    stream = torch.cuda.current_stream(trainer.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batches = [make_batch(warmup + k) for k in range(steps)]
    e0.record(stream)
    for b in batches:
        trainer.step(b)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def _best_of(trainer, make_batch, steps: int, warmup: int, reps: int) -> float:
    return min(_time_steps(trainer, make_batch, steps, warmup) for _ in range(reps))


def tune(trainer, make_batch, steps: int = 3, warmup: int = 2, space: dict | None = None,
         cache: str | Path | None = None, reps: int = 2, margin: float = 0.01) -> dict:
    """Pick the fastest tuning for this trainer's workload.  ``make_batch(k)``
    returns the k-th RayBatch of a representative stream (it is called for
    warm-up and timed steps of every candidate).  Each candidate is timed as
    the best of ``reps`` runs and replaces the incumbent only when faster by
    more than ``margin``; the result is checked once more against the tuning
    the search started from, so timing noise cannot leave a slower choice."""
    if getattr(trainer, "sharded", None) is not None:
        raise ValueError("tune a trainer without the sharded optimizer: its steps are collectives, and the "
                         "search takes a different number of steps on each rank")
    space = space or SPACE
    probe = make_batch(0)
    key = workload_key(trainer, probe.num_rays)
    if cache is not None and Path(cache).exists():
        stored = json.loads(Path(cache).read_text())
        if key in stored:
            set_tuning(stored[key]["tuning"])
            return stored[key]["tuning"]
    model = trainer.model
    saved = [t.detach().clone() for t in (model.table, model.mlp, trainer.m_table, trainer.v_table, trainer.m_mlp,
                                          trainer.v_mlp)]
    saved_step = trainer.step_count
    start = get_tuning()
    best = dict(start)
    try:
        set_tuning(best)
        best_ms = _best_of(trainer, make_batch, steps, warmup, reps)
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                cand = dict(best, **{name: v})
                set_tuning(cand)
                ms = _best_of(trainer, make_batch, steps, warmup, reps)
                if ms < best_ms * (1.0 - margin):
                    best, best_ms = cand, ms
        if best != start:   # confirm against the starting point with fresh timings
            set_tuning(start)
            start_ms = _best_of(trainer, make_batch, steps, warmup, reps)
            set_tuning(best)
            best_ms = _best_of(trainer, make_batch, steps, warmup, reps)
            if start_ms <= best_ms * (1.0 + margin / 2):
                best, best_ms = start, start_ms
        set_tuning(best)
    finally:
        with torch.no_grad():
            for dst, src in zip((model.table, model.mlp, trainer.m_table, trainer.v_table, trainer.m_mlp,
                                 trainer.v_mlp), saved):
                dst.copy_(src)
            model.refresh_half()
        trainer.step_count = saved_step
        trainer.table_grad.zero_()
        trainer.mlp_grad.zero_()
    if cache is not None:
        path = Path(cache)
        stored = json.loads(path.read_text()) if path.exists() else {}
        stored[key] = {"tuning": best, "ms_per_step": best_ms}
        path.write_text(json.dumps(stored, indent=1))
    return best
