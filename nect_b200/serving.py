"""Queries against a trained model and a continuous-batching query server.

The reference answers queries offline, one request at a time, one model call
per slice (create_volume, nect/trainers/base_trainer.py:402-450;
export_volume, nect/static_export.py:15-144; export_volumes/_at_timesteps and
export_video, nect/dynamic_export.py:145-544).  Here:

* ``slice_items`` / ``volume_items`` describe the points of a request as
  compact work items (origin + step vectors, a numpy table in the layout of
  NectbQueryItem); ``query_points`` evaluates any set of items of any requests
  in ONE persistent launch (nectb_query_points), generating coordinates on the
  fly and writing de-normalised values (``/max_distance_traveled * (max - min)
  + min``, as the reference exports them).
* ``reproject`` computes a detector view at (angle, t) with the training
  sampler (nectb_query_reproject).
* ``QueryServer`` keeps the model on the device and serves a stream of mixed
  requests (continuous batching): requests are admitted into preallocated
  device/pinned slots (the memory budget is split into slots per request class
  at start-up, so serving never allocates), slice requests are packed several
  per launch on high-priority streams, volume exports (cut into z-slice items)
  and re-projections run on low-priority streams with their persistent grids
  capped at one block per SM so slice blocks always find free SMs; point
  launches are replayed from CUDA graphs captured per chunk-count bucket.  A
  request completes when its last launch finished and its result reached
  pinned host memory; latency is arrival-to-result.
"""
from __future__ import annotations

import ctypes
import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .network import _HashGridModel

CHUNK = 128

ITEM_DTYPE = np.dtype({
    "names": ["origin", "du", "dv", "nu", "nv", "t", "out_scale", "out_offset", "out", "out_stride", "chunk_begin"],
    "formats": [("<f4", 3), ("<f4", 3), ("<f4", 3), "<i4", "<i4", "<f4", "<f4", "<f4", "<u8", "<i8", "<i8"],
    "offsets": [0, 12, 24, 36, 40, 44, 48, 52, 56, 64, 72],
    "itemsize": 80,
})  # NectbQueryItem (include/nectb.h)


def denormalisation(max_distance_traveled: float, minimum: float = 0.0, maximum: float = 1.0):
    """(scale, offset) of sigma/max_distance_traveled*(max-min)+min (static_export.py:139-140)."""
    return (maximum - minimum) / max_distance_traveled, minimum


def centres(n: int) -> np.ndarray:
    """Voxel centres linspace(0.5/n, 1-0.5/n, n) as create_volume uses (base_trainer.py:411-432)."""
    return (np.arange(n) + 0.5) / n


def item_chunks(items: np.ndarray) -> np.ndarray:
    return (items["nu"].astype(np.int64) * items["nv"] + CHUNK - 1) // CHUNK


def volume_items(out: torch.Tensor | int, shape: tuple, t: float, scale: float = 1.0,
                 offset: float = 0.0) -> np.ndarray:
    """Volume [nz, ny, nx] at voxel centres, one item per z-slice; out is the
    output tensor or its device address."""
    nz, ny, nx = shape
    base = out.data_ptr() if isinstance(out, torch.Tensor) else int(out)
    it = np.zeros(nz, ITEM_DTYPE)
    it["origin"][:, 0] = (np.arange(nz) + 0.5) / nz
    it["origin"][:, 1] = 0.5 / ny
    it["origin"][:, 2] = 0.5 / nx
    it["du"][:, 2] = 1.0 / nx
    it["dv"][:, 1] = 1.0 / ny
    it["nu"], it["nv"], it["t"] = nx, ny, t
    it["out_scale"], it["out_offset"] = scale, offset
    it["out"] = base + 4 * np.arange(nz, dtype=np.uint64) * np.uint64(ny * nx)
    it["out_stride"] = nx
    return it


def slice_items(out: torch.Tensor | int, shape: tuple, t: float, centre=(0.5, 0.5, 0.5), u=(0.0, 0.0, 1.0),
                v=(0.0, 1.0, 0.0), scale: float = 1.0, offset: float = 0.0, rows_per_item: int = 64) -> np.ndarray:
    """nv x nu plane through ``centre`` spanned by unit vectors u (columns) and v
    (rows), sampled at cell centres of a unit square (axis-aligned slices
    reproduce create_volume's grid; oblique ones rotate it)."""
    nv_, nu_ = shape
    base = out.data_ptr() if isinstance(out, torch.Tensor) else int(out)
    c = np.asarray(centre, np.float64)
    u = np.asarray(u, np.float64) / np.linalg.norm(u)
    v = np.asarray(v, np.float64) / np.linalg.norm(v)
    r0 = np.arange(0, nv_, rows_per_item)
    it = np.zeros(r0.size, ITEM_DTYPE)
    it["origin"] = c + ((0.5 / nu_) - 0.5) * u + ((r0[:, None] + 0.5) / nv_ - 0.5) * v
    it["du"], it["dv"] = u / nu_, v / nv_
    it["nu"], it["nv"], it["t"] = nu_, np.minimum(rows_per_item, nv_ - r0), t
    it["out_scale"], it["out_offset"] = scale, offset
    it["out"] = base + 4 * r0.astype(np.uint64) * np.uint64(nu_)
    it["out_stride"] = nu_
    return it


def _call_points(model: _HashGridModel, items_dev: int, n_items: int, total_chunks: int, counter_dev: int,
                 stream: int, max_blocks: int = 0):
    rc = _lib.lib.nectb_query_points(ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc),
                                     model.grid_table.data_ptr(), model.mlp.data_ptr(), items_dev, n_items,
                                     total_chunks, counter_dev, max_blocks, stream)
    _lib.check(rc, "nectb_query_points")


def time_slice_bytes(model: _HashGridModel) -> int:
    """Bytes of a time slice of the model (0: a model without one, i.e. not
    4D with an fp16 table)."""
    return int(_lib.lib.nectb_time_slice_bytes(ctypes.byref(model.grid_desc)))


def time_slice(model: _HashGridModel, t: float, out: torch.Tensor | None = None,
               stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """The model's fp16 table blended at t into a 3D slice (nectb_time_slice):
    queries at that t gather 8 corners per level on it instead of 16."""
    n = time_slice_bytes(model)
    if n == 0:
        raise ValueError("the model has no time slice (4D with an fp16 table only)")
    if out is None:
        out = torch.empty(n, dtype=torch.uint8, device=model.table.device)
    stream = stream or torch.cuda.current_stream()
    rc = _lib.lib.nectb_time_slice(ctypes.byref(model.grid_desc), model.grid_table.data_ptr(), float(t),
                                   out.data_ptr(), out.numel() * out.element_size(), stream.cuda_stream)
    _lib.check(rc, "nectb_time_slice")
    return out


def _call_points_slice(model: _HashGridModel, slice_ptr: int, items_dev: int, n_items: int, total_chunks: int,
                       counter_dev: int, stream: int, max_blocks: int = 0):
    rc = _lib.lib.nectb_query_points_slice(ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc), slice_ptr,
                                           model.mlp.data_ptr(), items_dev, n_items, total_chunks, counter_dev,
                                           max_blocks, stream)
    _lib.check(rc, "nectb_query_points_slice")


def query_points(model: _HashGridModel, items: np.ndarray, stream: torch.cuda.Stream | None = None,
                 max_blocks: int = 0, slice: torch.Tensor | None = None):
    """Evaluate the items (any requests) in one launch (outputs written in place);
    max_blocks > 0 caps the persistent grid.  With ``slice`` (time_slice at
    some t) every item is evaluated on it, at its t."""
    if items.size == 0:
        return
    stream = stream or torch.cuda.current_stream()
    items = items.copy()
    ch = item_chunks(items)
    items["chunk_begin"] = np.concatenate([[0], np.cumsum(ch)[:-1]])
    dev = model.table.device
    buf = torch.empty(items.nbytes + 16, dtype=torch.uint8, device=dev)
    with torch.cuda.stream(stream):
        buf[items.nbytes:].zero_()   # work cursor and error word
        buf[:items.nbytes].copy_(torch.from_numpy(items.view(np.uint8)), non_blocking=False)
        if slice is None:
            _call_points(model, buf.data_ptr(), items.size, int(ch.sum()), buf.data_ptr() + items.nbytes,
                         stream.cuda_stream, max_blocks)
        else:
            _call_points_slice(model, slice.data_ptr(), buf.data_ptr(), items.size, int(ch.sum()),
                               buf.data_ptr() + items.nbytes, stream.cuda_stream, max_blocks)


def reproject_workspace_bytes(model: _HashGridModel, geometry, pixels: int | None = None) -> int:
    """Workspace of a re-projection of ``pixels`` detector pixels (default the
    whole view) by pieces: the sampler's workspace plus, for a 4D mixed model,
    room for the time slice."""
    cg = geometry.get_c_geometry()
    n = pixels or geometry.nDetector[0] * geometry.nDetector[1]
    return int(_lib.lib.nectb_train_workspace_bytes(ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc),
                                                    ctypes.byref(model.mlp_desc), n)
               + _lib.lib.nectb_query_reproject_slice_bytes(ctypes.byref(model.grid_desc),
                                                            ctypes.byref(model.mlp_desc), n))


def reproject(model: _HashGridModel, geometry, angle: float, t: float = 0.0, points_per_ray: int | None = None,
              out: torch.Tensor | None = None, workspace: torch.Tensor | None = None,
              stream: torch.cuda.Stream | None = None, max_blocks: int = 0, pixels: tuple[int, int] | None = None,
              warpgroups: int = 0) -> torch.Tensor:
    """Detector view [nDetector] at (angle, t): sum of sigma * distance / max_distance_traveled per ray.

    pixels=(begin, count) computes only those detector pixels (row-major) of
    ``out``; warpgroups (1-4) sets the mixed forward's warpgroups per SM, and
    such a call runs a 4D mixed model on a time slice at t when the
    workspace has room for it (reproject_workspace_bytes)."""
    cg = geometry.get_c_geometry()
    S = points_per_ray or int(math.ceil(1.5 * max(geometry.nDetector)))
    P = geometry.nDetector[0] * geometry.nDetector[1]
    dev = model.table.device
    if out is None:
        out = torch.empty(P, device=dev)
    stream = stream or torch.cuda.current_stream()
    if pixels is None and not warpgroups:
        need = _lib.lib.nectb_train_workspace_bytes(ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc),
                                                    ctypes.byref(model.mlp_desc), P)
        if workspace is None or workspace.numel() < need:
            workspace = torch.empty(need, dtype=torch.uint8, device=dev)
        rc = _lib.lib.nectb_query_reproject(ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc),
                                            ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                            model.mlp.data_ptr(), float(angle), float(t), S,
                                            geometry.max_distance_traveled / S, geometry.max_distance_traveled,
                                            out.data_ptr(), workspace.data_ptr(), workspace.numel(), int(max_blocks),
                                            stream.cuda_stream)
        _lib.check(rc, "nectb_query_reproject")
    else:
        begin, count = pixels or (0, P)
        if workspace is None:
            workspace = torch.empty(reproject_workspace_bytes(model, geometry, count), dtype=torch.uint8, device=dev)
        rc = _lib.lib.nectb_query_reproject_range(
            ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc),
            model.grid_table.data_ptr(), model.mlp.data_ptr(), float(angle), float(t), S,
            geometry.max_distance_traveled / S, geometry.max_distance_traveled, out.data_ptr(), int(begin), int(count),
            workspace.data_ptr(), workspace.numel(), int(max_blocks), int(warpgroups), stream.cuda_stream)
        _lib.check(rc, "nectb_query_reproject_range")
    return out.view(geometry.nDetector[0], geometry.nDetector[1])


# ---------------------------------------------------------------- server ----
@dataclass
class Request:
    kind: str                      # "slice" | "reproject" | "volume"
    t: float = 0.0
    size: int = 512                # slice n (n x n) / volume n (n^3)
    angle: float = 0.0             # reproject
    centre: tuple = (0.5, 0.5, 0.5)
    u: tuple = (0.0, 0.0, 1.0)
    v: tuple = (0.0, 1.0, 0.0)
    # filled by the server
    arrival: float = 0.0
    launched: float = 0.0          # host time its last launch was issued
    done: float = 0.0
    result: np.ndarray | None = None
    event: threading.Event = field(default_factory=threading.Event)

    def out_shape(self, geometry) -> tuple:
        if self.kind == "slice":
            return (self.size, self.size)
        if self.kind == "volume":
            return (self.size, self.size, self.size)
        return tuple(geometry.nDetector)

    def latency_ms(self) -> float:
        return (self.done - self.arrival) * 1e3

    def wait_ms(self) -> float:
        """Arrival to the issue of its last launch (queueing on the host)."""
        return (self.launched - self.arrival) * 1e3


BUCKETS = (64, 256, 1024, 4096, 16384)   # chunks per launch (128 points each)
MAX_ITEMS = 512


class _Pool:
    """Fixed device + pinned host slots of one request class."""

    def __init__(self, n: int, floats: int, dev, ws_bytes: int = 0):
        self.dev_buf = torch.empty(n, floats, device=dev)
        self.host_buf = torch.empty(n, floats).pin_memory()
        self.ws = torch.empty(n, max(ws_bytes, 1), dtype=torch.uint8, device=dev) if ws_bytes else None
        self.free = list(range(n))


class _Lane:
    """One stream with graph-captured point launches (one graph per bucket).

    priority: CUDA stream priority (lower is higher priority); max_blocks caps
    the persistent grid (0 = two blocks per SM)."""

    def __init__(self, dev, priority: int = 0, max_blocks: int = 0):
        self.stream = torch.cuda.Stream(device=dev, priority=priority)
        self.max_blocks = max_blocks
        self.items_dev = torch.zeros(MAX_ITEMS * ITEM_DTYPE.itemsize + 64, dtype=torch.uint8, device=dev)
        self.items_host = torch.empty(MAX_ITEMS * ITEM_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        self.table = self.items_host.numpy().view(ITEM_DTYPE)
        self.dummy = torch.empty(CHUNK * BUCKETS[-1], device=dev)   # sink for padding chunks
        self.graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self.last: torch.cuda.Event | None = None

    def counter_ptr(self) -> int:
        return self.items_dev.data_ptr() + MAX_ITEMS * ITEM_DTYPE.itemsize

    def idle(self) -> bool:
        return self.last is None or self.last.query()

    def error_word(self) -> int:
        """Sticky error word of this lane's launches (non-zero if a tensor-core
        wait timed out).  Synchronises the lane."""
        off = MAX_ITEMS * ITEM_DTYPE.itemsize + 4
        self.stream.synchronize()
        return int(self.items_dev[off:off + 4].view(torch.int32).item())

    def capture(self, model):
        for b in BUCKETS:
            self._write(np.zeros(0, ITEM_DTYPE), b)
            with torch.cuda.stream(self.stream):   # warm-up launch sets kernel attributes
                self.items_dev[:self.items_host.numel()].copy_(self.items_host, non_blocking=True)
                _call_points(model, self.items_dev.data_ptr(), MAX_ITEMS, b, self.counter_ptr(),
                             self.stream.cuda_stream, self.max_blocks)
            self.stream.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=self.stream, capture_error_mode="relaxed"):
                _call_points(model, self.items_dev.data_ptr(), MAX_ITEMS, b, self.counter_ptr(),
                             torch.cuda.current_stream().cuda_stream, self.max_blocks)
            self.graphs[b] = g

    def _write(self, items: np.ndarray, bucket: int):
        """items, one padding item over the bucket's unused chunks (to a sink),
        then empty items."""
        n = items.size
        tab = self.table
        ch = item_chunks(items)
        tab[:n] = items
        begins = np.concatenate([[0], np.cumsum(ch)]).astype(np.int64)
        tab["chunk_begin"][:n] = begins[:-1]
        used = int(begins[-1])
        tail = tab[n:]
        tail[:] = np.zeros(1, ITEM_DTYPE)
        tail["out"] = self.dummy.data_ptr()
        tail["out_stride"] = CHUNK
        tail["out_scale"] = 1.0
        tail["origin"] = 0.5
        tail["chunk_begin"] = bucket
        if bucket > used:
            tail["nu"][0], tail["nv"][0], tail["chunk_begin"][0] = CHUNK, bucket - used, used

    def launch(self, items: np.ndarray, model: _HashGridModel | None = None,
               slice_ptr: int = 0) -> torch.cuda.Event:
        """Items in one launch: the bucket's captured graph, or with slice_ptr
        (items of one request, on its time slice) a direct launch."""
        total = int(item_chunks(items).sum())
        bucket = next(b for b in BUCKETS if b >= total)
        if self.last is not None:
            self.last.synchronize()   # this lane's staging buffer has been consumed
        self._write(items, bucket)
        with torch.cuda.stream(self.stream):
            self.items_dev[:self.items_host.numel()].copy_(self.items_host, non_blocking=True)
            if slice_ptr:
                _call_points_slice(model, slice_ptr, self.items_dev.data_ptr(), MAX_ITEMS, bucket,
                                   self.counter_ptr(), self.stream.cuda_stream, self.max_blocks)
            else:
                self.graphs[bucket].replay()
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.last = ev
        return ev


class QueryServer:
    """Continuous-batching server for slice / volume / re-projection queries.

    The memory budget is split at start-up into slots: slices up to
    ``max_slice``^2, volumes up to ``max_volume``^3, re-projections of the
    geometry's detector with their sampler workspace (shares in the
    proportions ``slot_mix``).  A request waits until a slot of its class is
    free (admission by memory); nothing is allocated while serving.

    Slices run on ``n_fast`` high-priority lanes, packed several requests per
    launch.  Volumes and re-projections share ``n_slow`` low-priority lanes.
    Volume launches are persistent grids capped at ``slow_blocks`` (default
    three one-warpgroup blocks per SM, 384 of its 512 tensor-memory columns):
    an SM keeps room for a slice block while background work runs, which is
    what keeps slice p99 near its unloaded latency.  A
    re-projection runs as pieces of ``piece_pixels`` detector pixels, each a
    launch of about a millisecond with ``slow_warpgroups`` warpgroups per SM
    (4 take half of an SM's tensor memory and two thirds of its registers,
    leaving room for a slice block; a 4D mixed model runs on a time slice at
    the request's t), so a slice waits at most one piece for SMs.  Volumes of a
    4D mixed model are evaluated on a time slice at their t too, built once
    per request."""

    def __init__(self, model: _HashGridModel, geometry, memory_budget: int = 40 << 30, n_fast: int = 2,
                 n_slow: int = 1, minimum: float = 0.0, maximum: float = 1.0, points_per_ray: int | None = None,
                 slow_blocks: int | None = None, max_slice: int = 1024, max_volume: int = 256,
                 slot_mix=(0.25, 0.25, 0.5), max_slots: int = 64, piece_pixels: int = 16384,
                 slow_warpgroups: int = 4):
        self.model = model
        self.geometry = geometry
        self.dev = model.table.device
        self.scale, self.offset = denormalisation(geometry.max_distance_traveled, minimum, maximum)
        self.points_per_ray = points_per_ray
        sms = torch.cuda.get_device_properties(self.dev).multi_processor_count
        self.slow_blocks = slow_blocks if slow_blocks is not None else 3 * sms
        if not 1 <= slow_warpgroups <= 6 or piece_pixels < 1:
            raise ValueError("slow_warpgroups must be 1..6 and piece_pixels positive")
        self.slow_warpgroups = slow_warpgroups
        lo, hi = torch.cuda.Stream.priority_range()
        self.fast = [_Lane(self.dev, priority=hi) for _ in range(n_fast)]
        self.slow = [_Lane(self.dev, priority=lo, max_blocks=self.slow_blocks) for _ in range(n_slow)]
        for ln in self.fast + self.slow:
            ln.capture(model)
        P = geometry.nDetector[0] * geometry.nDetector[1]
        self.n_pixels = P
        self.piece_pixels = min(piece_pixels, P)
        ws = (reproject_workspace_bytes(model, geometry, self.piece_pixels) + 255) // 256 * 256
        # a volume of a 4D mixed model is evaluated on a time slice at its t, built once per request
        self.slice_bytes = (time_slice_bytes(model) + 511) // 512 * 512   # texture alignment
        per = {"slice": 8 * max_slice ** 2, "volume": 8 * max_volume ** 3 + self.slice_bytes, "reproject": 8 * P + ws}
        nslots = {k: max(1, min(max_slots, int(memory_budget * f // per[k])))
                  for k, f in zip(("slice", "reproject", "volume"), slot_mix)}
        self.pools = {"slice": _Pool(nslots["slice"], max_slice ** 2, self.dev),
                      "volume": _Pool(nslots["volume"], max_volume ** 3, self.dev, ws_bytes=self.slice_bytes),
                      "reproject": _Pool(nslots["reproject"], P, self.dev, ws_bytes=ws)}
        self.max_slice, self.max_volume = max_slice, max_volume
        self.queue: queue.Queue = queue.Queue()
        self.completed: list[Request] = []
        self._rr = {"fast": 0, "slow": 0}
        self._done_q: queue.Queue = queue.Queue()
        self._free_q: queue.Queue = queue.Queue()
        self._finisher = threading.Thread(target=self._finish_loop, daemon=True)
        self._finisher.start()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    # -- client side ------------------------------------------------------
    def submit(self, req: Request) -> Request:
        if req.kind == "slice" and req.size > self.max_slice or req.kind == "volume" and req.size > self.max_volume:
            raise ValueError(f"{req.kind} of size {req.size} exceeds the server's slots")
        req.arrival = time.perf_counter()
        self.queue.put(req)
        return req

    def close(self):
        self.queue.put(None)
        self._thread.join()
        self._done_q.put(None)
        self._finisher.join()

    def _finish_loop(self):
        """Copies finished results out of their pinned slots and releases the
        slots, off the scheduler thread (a 64 MB volume copy must not stall
        the launches of other requests)."""
        while True:
            st = self._done_q.get()
            if st is None:
                return
            r, pool = st["req"], self.pools[st["req"].kind]
            r.result = pool.host_buf[st["slot"], :st["n"]].numpy().reshape(st["shape"]).copy()
            self._free_q.put((r.kind, st["slot"]))
            self.completed.append(r)
            r.event.set()

    # -- scheduler --------------------------------------------------------
    def _lane(self, kind: str, want_idle: bool = False):
        lanes = self.fast if kind == "fast" else self.slow
        if not want_idle:  # prefer an idle lane, so the launch never waits for a staging buffer
            for k in range(len(lanes)):
                ln = lanes[(self._rr[kind] + k) % len(lanes)]
                if ln.idle():
                    self._rr[kind] += k + 1
                    return ln
        for k in range(len(lanes)):
            ln = lanes[(self._rr[kind] + k) % len(lanes)]
            if not want_idle or ln.idle():
                self._rr[kind] += k + 1
                return ln
        return None

    def _finish_on(self, st: dict, ln: _Lane):
        pool, slot, n = self.pools[st["req"].kind], st["slot"], st["n"]
        with torch.cuda.stream(ln.stream):
            pool.host_buf[slot, :n].copy_(pool.dev_buf[slot, :n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(ln.stream)
        st["events"].append(ev)

    @staticmethod
    def _pack(active: list[dict], limit_chunks: int):
        parts, chunks, touched = [], 0, []
        for st in active:
            it, ch = st["items"], st["chunks"]
            k = 0
            while k < it.size and chunks + ch[k] <= limit_chunks and sum(p.size for p in parts) + k < MAX_ITEMS - 1:
                chunks += int(ch[k])
                k += 1
            if k:
                parts.append(it[:k])
                st["items"], st["chunks"] = it[k:], ch[k:]
                touched.append(st)
            if k < it.size:
                break
        return (np.concatenate(parts) if parts else np.zeros(0, ITEM_DTYPE)), touched

    def _admit(self, r: Request):
        pool = self.pools[r.kind]
        if not pool.free:
            return None
        slot = pool.free.pop(0)
        shape = r.out_shape(self.geometry)
        n = int(np.prod(shape))
        addr = pool.dev_buf[slot].data_ptr()
        st = {"req": r, "slot": slot, "n": n, "shape": shape, "events": []}
        if r.kind == "slice":
            st["items"] = slice_items(addr, shape, r.t, r.centre, r.u, r.v, self.scale, self.offset)
        elif r.kind == "volume":
            st["items"] = volume_items(addr, shape, r.t, self.scale, self.offset)
        if "items" in st:
            st["chunks"] = item_chunks(st["items"])
        return st

    def _run(self):
        torch.cuda.set_device(self.dev)
        waiting: list[Request] = []
        slices: list[dict] = []
        volumes: list[dict] = []
        reprojs: list[dict] = []
        flying: list[dict] = []
        closing = False
        while True:
            idle = not (waiting or slices or volumes or reprojs or flying)
            if closing and idle:
                return
            if idle and waiting == [] and self._free_q.qsize():
                idle = False
            try:
                r = self.queue.get(block=idle)
                while True:
                    if r is None:
                        closing = True
                    else:
                        waiting.append(r)
                    r = self.queue.get_nowait()
            except queue.Empty:
                pass
            # slots released by the finisher thread
            try:
                while True:
                    kind, slot = self._free_q.get_nowait()
                    self.pools[kind].free.append(slot)
            except queue.Empty:
                pass
            # admission: in arrival order within each class, when a slot is free
            still = []
            for r in waiting:
                st = self._admit(r)
                if st is None:
                    still.append(r)
                else:
                    {"slice": slices, "volume": volumes, "reproject": reprojs}[r.kind].append(st)
            waiting = still
            # slices: every pending slice item, packed across requests, on a fast lane
            while slices:
                batch, touched = self._pack(slices, BUCKETS[-1])
                if batch.size == 0:
                    break
                ln = self._lane("fast")
                ev = ln.launch(batch)
                for st in touched:
                    st["events"].append(ev)
                    if st["items"].size == 0:
                        st["req"].launched = time.perf_counter()
                        self._finish_on(st, ln)
                        slices.remove(st)
                        flying.append(st)
            # background: one launch per idle slow lane, oldest request first;
            # a re-projection's pieces run in order on the lane of its first piece
            while reprojs or volumes:
                ln = self._lane("slow", want_idle=True)
                if ln is None:
                    break
                st = next((x for x in reprojs if x.get("lane") in (None, ln)), None)
                if st is not None and (not volumes or st["req"].arrival <= volumes[0]["req"].arrival):
                    if self._reproject_piece(st, ln):
                        reprojs.remove(st)
                        self._finish_on(st, ln)
                        flying.append(st)
                elif not (volumes and self._volume_launch(volumes, ln, flying)):
                    break
            # completions
            for st in list(flying):
                if all(e.query() for e in st["events"]):
                    st["req"].done = time.perf_counter()
                    flying.remove(st)
                    self._done_q.put(st)
            if self.queue.empty() and not slices and (flying or reprojs or volumes or waiting):
                time.sleep(0.0001)

    def _volume_launch(self, volumes: list[dict], ln: _Lane, flying: list[dict]) -> bool:
        """One launch of at most 4096 chunks of volume items on lane ln: the
        oldest requests' items packed together, or, for a 4D mixed model, the
        oldest request's items on its time slice (built at its first launch,
        on the lane that then runs all of its launches).  False when there was
        nothing to launch on this lane."""
        if self.slice_bytes:
            st = next((x for x in volumes if x.get("lane") in (None, ln)), None)
            if st is None:
                return False
            slc = self.pools["volume"].ws[st["slot"]]
            if "lane" not in st:
                time_slice(self.model, st["req"].t, out=slc, stream=ln.stream)
                st["lane"] = ln
            batch, touched = self._pack([st], 4096)
            ev = ln.launch(batch, self.model, slc.data_ptr())
        else:
            batch, touched = self._pack(volumes, 4096)
            ev = ln.launch(batch)
        for st in touched:
            st["events"].append(ev)
            if st["items"].size == 0:
                st["req"].launched = time.perf_counter()
                self._finish_on(st, ln)
                volumes.remove(st)
                flying.append(st)
        return True

    def _reproject_piece(self, st: dict, ln: _Lane) -> bool:
        """Launches the next piece of a re-projection on lane ln; True when it
        was the last one."""
        r, pool = st["req"], self.pools["reproject"]
        begin = st.get("next", 0)
        count = min(self.piece_pixels, self.n_pixels - begin)
        with torch.cuda.stream(ln.stream):
            reproject(self.model, self.geometry, r.angle, r.t, self.points_per_ray, out=pool.dev_buf[st["slot"]],
                      workspace=pool.ws[st["slot"]], stream=ln.stream, pixels=(begin, count),
                      warpgroups=self.slow_warpgroups)
            ev = torch.cuda.Event()
            ev.record(ln.stream)
        ln.last = ev
        if begin == 0:
            r.launched = time.perf_counter()
            st["lane"] = ln
        st["next"] = begin + count
        if st["next"] < self.n_pixels:
            return False
        st["events"].append(ev)
        return True

    def device_errors(self) -> int:
        """OR of the error words of every lane (0 = no tensor-core wait timed out)."""
        err = 0
        for ln in self.fast + self.slow:
            err |= ln.error_word()
        return err

    # -- statistics ---------------------------------------------------------
    def latency_stats(self) -> dict:
        out = {}
        for kind in ("slice", "reproject", "volume"):
            done = [r for r in self.completed if r.kind == kind]
            lat = np.array([r.latency_ms() for r in done])
            if lat.size:
                wait = np.array([r.wait_ms() for r in done])
                out[kind] = {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
                             "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                             "wait_p99_ms": float(np.percentile(wait, 99))}
        return out
