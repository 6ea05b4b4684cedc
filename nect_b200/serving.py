"""Queries against a trained model and a continuous-batching query server.

The reference answers queries offline, one request at a time, one model call
per slice (create_volume, nect/trainers/base_trainer.py:402-450;
export_volume, nect/static_export.py:15-144; export_volumes/_at_timesteps and
export_video, nect/dynamic_export.py:145-544).  Here:

* ``slice_items`` / ``volume_items`` describe the points of a request as
  compact work items (origin + step vectors); ``query_points`` evaluates any
  set of items of any requests in ONE persistent launch (nectb_query_points),
  generating coordinates on the fly and writing de-normalised values
  (``/max_distance_traveled * (max - min) + min``, as the reference exports).
* ``reproject`` computes a detector view at (angle, t) with the training
  sampler (nectb_query_reproject).
* ``QueryServer`` keeps the model on the device and serves a stream of mixed
  requests: each request is admitted when its output and workspace fit in the
  memory budget; admitted point requests are cut into chunk slices and packed,
  several requests per launch, into persistent launches that are replayed from
  CUDA graphs captured per chunk-count bucket; launches rotate over several
  streams so new requests start while earlier ones are still running; each
  request completes when its last launch has finished and its result has been
  copied to pinned host memory.  Latencies are arrival-to-result.
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


class NectbQueryItem(ctypes.Structure):
    _fields_ = [
        ("origin", ctypes.c_float * 3),
        ("du", ctypes.c_float * 3),
        ("dv", ctypes.c_float * 3),
        ("nu", ctypes.c_int32),
        ("nv", ctypes.c_int32),
        ("t", ctypes.c_float),
        ("out_scale", ctypes.c_float),
        ("out_offset", ctypes.c_float),
        ("out", ctypes.c_void_p),
        ("out_stride", ctypes.c_int64),
        ("chunk_begin", ctypes.c_int64),
    ]


ITEM_BYTES = ctypes.sizeof(NectbQueryItem)

_lib.lib.nectb_query_points.restype = ctypes.c_int32
_lib.lib.nectb_query_points.argtypes = [ctypes.POINTER(_lib.NectbHashGrid), ctypes.POINTER(_lib.NectbMLP),
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                        ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
_lib.lib.nectb_query_reproject.restype = ctypes.c_int32
_lib.lib.nectb_query_reproject.argtypes = [ctypes.POINTER(_lib.NectbGeometry), ctypes.POINTER(_lib.NectbHashGrid),
                                           ctypes.POINTER(_lib.NectbMLP), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_void_p]


@dataclass
class Item:
    """Host description of one work item (an nu x nv grid of points)."""
    origin: tuple
    du: tuple
    dv: tuple
    nu: int
    nv: int
    t: float
    out: int          # device address of the first output value
    out_stride: int   # floats between rows
    scale: float = 1.0
    offset: float = 0.0

    @property
    def chunks(self) -> int:
        return -(-self.nu * self.nv // CHUNK)


def denormalisation(max_distance_traveled: float, minimum: float = 0.0, maximum: float = 1.0):
    """(scale, offset) of sigma/max_distance_traveled*(max-min)+min (static_export.py:139-140)."""
    return (maximum - minimum) / max_distance_traveled, minimum


def centres(n: int) -> np.ndarray:
    """Voxel centres linspace(0.5/n, 1-0.5/n, n) as create_volume uses (base_trainer.py:411-432)."""
    return (np.arange(n) + 0.5) / n


def volume_items(out: torch.Tensor, t: float, scale: float = 1.0, offset: float = 0.0,
                 rows_per_item: int | None = None) -> list[Item]:
    """Volume [nz, ny, nx] at voxel centres, z-slices (or slabs of rows) as items."""
    nz, ny, nx = out.shape
    rows = rows_per_item or ny
    items = []
    base = out.data_ptr()
    for k in range(nz):
        for r0 in range(0, ny, rows):
            nr = min(rows, ny - r0)
            items.append(Item(origin=((k + 0.5) / nz, (r0 + 0.5) / ny, 0.5 / nx), du=(0.0, 0.0, 1.0 / nx),
                              dv=(0.0, 1.0 / ny, 0.0), nu=nx, nv=nr, t=t,
                              out=base + 4 * (k * ny * nx + r0 * nx), out_stride=nx, scale=scale, offset=offset))
    return items


def slice_items(out: torch.Tensor, t: float, centre=(0.5, 0.5, 0.5), u=(0.0, 0.0, 1.0), v=(0.0, 1.0, 0.0),
                scale: float = 1.0, offset: float = 0.0, rows_per_item: int = 64) -> list[Item]:
    """n x n plane through ``centre`` spanned by unit vectors u (columns) and v
    (rows), sampled at cell centres over a unit-sized square (axis-aligned
    slices reproduce create_volume's grid; oblique ones rotate it)."""
    nv_, nu_ = out.shape
    c = np.asarray(centre, np.float64)
    u = np.asarray(u, np.float64) / np.linalg.norm(u)
    v = np.asarray(v, np.float64) / np.linalg.norm(v)
    items = []
    for r0 in range(0, nv_, rows_per_item):
        nr = min(rows_per_item, nv_ - r0)
        o = c + ((0.5 / nu_) - 0.5) * u + ((r0 + 0.5) / nv_ - 0.5) * v
        items.append(Item(origin=tuple(o), du=tuple(u / nu_), dv=tuple(v / nv_), nu=nu_, nv=nr, t=t,
                          out=out.data_ptr() + 4 * r0 * nu_, out_stride=nu_, scale=scale, offset=offset))
    return items


def pack_items(items: list[Item]) -> tuple[ctypes.Array, int]:
    arr = (NectbQueryItem * len(items))()
    total = 0
    for i, it in enumerate(items):
        a = arr[i]
        for k in range(3):
            a.origin[k], a.du[k], a.dv[k] = it.origin[k], it.du[k], it.dv[k]
        a.nu, a.nv, a.t = it.nu, it.nv, it.t
        a.out_scale, a.out_offset = it.scale, it.offset
        a.out, a.out_stride, a.chunk_begin = it.out, it.out_stride, total
        total += it.chunks
    return arr, total


def _call_points(model: _HashGridModel, items_dev: int, n_items: int, total_chunks: int, counter_dev: int,
                 stream: int):
    rc = _lib.lib.nectb_query_points(ctypes.byref(model.grid_desc), ctypes.byref(model.mlp_desc),
                                     model.grid_table.data_ptr(), model.mlp.data_ptr(), items_dev, n_items,
                                     total_chunks, counter_dev, stream)
    _lib.check(rc, "nectb_query_points")


def query_points(model: _HashGridModel, items: list[Item], stream: torch.cuda.Stream | None = None):
    """Evaluate the items in one launch on ``stream`` (outputs are written in place)."""
    if not items:
        return
    stream = stream or torch.cuda.current_stream()
    arr, total = pack_items(items)
    dev = model.table.device
    buf = torch.empty(ctypes.sizeof(arr) + 16, dtype=torch.uint8, device=dev)
    host = torch.frombuffer(bytearray(arr), dtype=torch.uint8)
    with torch.cuda.stream(stream):
        buf[:ctypes.sizeof(arr)].copy_(host, non_blocking=False)
        counter = buf[ctypes.sizeof(arr):ctypes.sizeof(arr) + 4]
        _call_points(model, buf.data_ptr(), len(items), total, counter.data_ptr(), stream.cuda_stream)


def reproject(model: _HashGridModel, geometry, angle: float, t: float = 0.0, points_per_ray: int | None = None,
              out: torch.Tensor | None = None, workspace: torch.Tensor | None = None,
              stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """Detector view [nDetector] at (angle, t): sum of sigma * distance / max_distance_traveled per ray."""
    cg = geometry.get_c_geometry()
    S = points_per_ray or int(math.ceil(1.5 * max(geometry.nDetector)))
    P = geometry.nDetector[0] * geometry.nDetector[1]
    dev = model.table.device
    if out is None:
        out = torch.empty(P, device=dev)
    need = _lib.lib.nectb_train_workspace_bytes(ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc),
                                                ctypes.byref(model.mlp_desc), P)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    stream = stream or torch.cuda.current_stream()
    rc = _lib.lib.nectb_query_reproject(ctypes.byref(cg.c_struct), ctypes.byref(model.grid_desc),
                                        ctypes.byref(model.mlp_desc), model.grid_table.data_ptr(),
                                        model.mlp.data_ptr(), float(angle), float(t), S,
                                        geometry.max_distance_traveled / S, geometry.max_distance_traveled,
                                        out.data_ptr(), workspace.data_ptr(), workspace.numel(), stream.cuda_stream)
    _lib.check(rc, "nectb_query_reproject")
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


BUCKETS = (64, 256, 1024, 4096, 16384)   # chunks per launch (128 points each)
MAX_ITEMS = 512


class _Lane:
    """One stream with its graph-captured launches (one per bucket)."""

    def __init__(self, server: "QueryServer", dev):
        self.stream = torch.cuda.Stream(device=dev)
        self.items_dev = torch.empty(MAX_ITEMS * ITEM_BYTES + 64, dtype=torch.uint8, device=dev)
        self.items_host = torch.empty(MAX_ITEMS * ITEM_BYTES, dtype=torch.uint8).pin_memory()
        self.dummy = torch.empty(CHUNK * BUCKETS[-1], device=dev)   # sink for padding chunks
        self.graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self.busy_event: torch.cuda.Event | None = None
        self.server = server

    def counter_ptr(self) -> int:
        return self.items_dev.data_ptr() + MAX_ITEMS * ITEM_BYTES

    def capture(self, model):
        for b in BUCKETS:
            g = torch.cuda.CUDAGraph()
            # warm up outside capture (sets kernel attributes), then capture
            self._write_padding(b, 0, 0)
            with torch.cuda.stream(self.stream):
                self.items_dev[:MAX_ITEMS * ITEM_BYTES].copy_(self.items_host, non_blocking=True)
                _call_points(model, self.items_dev.data_ptr(), MAX_ITEMS, b, self.counter_ptr(),
                             self.stream.cuda_stream)
            self.stream.synchronize()
            with torch.cuda.graph(g, stream=self.stream, capture_error_mode="relaxed"):
                _call_points(model, self.items_dev.data_ptr(), MAX_ITEMS, b, self.counter_ptr(),
                             torch.cuda.current_stream().cuda_stream)
            self.graphs[b] = g

    def _write_padding(self, bucket: int, n_items: int, used_chunks: int):
        """Fill items n_items.. with one padding item covering the unused chunks
        of the bucket (written to the dummy sink) and empty items after it."""
        arr = (NectbQueryItem * MAX_ITEMS).from_buffer(self.items_host.numpy())
        pad = bucket - used_chunks
        for i in range(n_items, MAX_ITEMS):
            a = arr[i]
            a.nu = CHUNK if (i == n_items and pad > 0) else 0
            a.nv = pad if (i == n_items and pad > 0) else 0
            a.out = self.dummy.data_ptr()
            a.out_stride = CHUNK
            a.t = 0.0
            a.out_scale, a.out_offset = 1.0, 0.0
            a.chunk_begin = used_chunks if i == n_items else bucket
            for k in range(3):
                a.origin[k], a.du[k], a.dv[k] = 0.5, 0.0, 0.0

    def launch(self, items: list[Item]) -> torch.cuda.Event:
        """Pack items (<= MAX_ITEMS - 1 of them, <= the largest bucket of chunks) and replay the graph."""
        total = sum(it.chunks for it in items)
        bucket = next(b for b in BUCKETS if b >= total)
        arr = (NectbQueryItem * MAX_ITEMS).from_buffer(self.items_host.numpy())
        if self.busy_event is not None:
            self.busy_event.synchronize()   # the host staging buffer of the previous launch is free
        c = 0
        for i, it in enumerate(items):
            a = arr[i]
            for k in range(3):
                a.origin[k], a.du[k], a.dv[k] = it.origin[k], it.du[k], it.dv[k]
            a.nu, a.nv, a.t = it.nu, it.nv, it.t
            a.out_scale, a.out_offset = it.scale, it.offset
            a.out, a.out_stride, a.chunk_begin = it.out, it.out_stride, c
            c += it.chunks
        self._write_padding(bucket, len(items), total)
        with torch.cuda.stream(self.stream):
            self.items_dev[:MAX_ITEMS * ITEM_BYTES].copy_(self.items_host, non_blocking=True)
            self.graphs[bucket].replay()
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.busy_event = ev
        return ev


class QueryServer:
    """Continuous-batching server for slice / volume / re-projection queries."""

    def __init__(self, model: _HashGridModel, geometry, memory_budget: int = 40 << 30, n_streams: int = 3,
                 max_chunks_per_launch: int = BUCKETS[-1], minimum: float = 0.0, maximum: float = 1.0,
                 points_per_ray: int | None = None):
        self.model = model
        self.geometry = geometry
        self.dev = model.table.device
        self.budget = memory_budget
        self.in_use = 0
        self.scale, self.offset = denormalisation(geometry.max_distance_traveled, minimum, maximum)
        self.points_per_ray = points_per_ray
        self.max_chunks = max_chunks_per_launch
        self.queue: queue.Queue = queue.Queue()
        self.lanes = [_Lane(self, self.dev) for _ in range(n_streams)]
        for ln in self.lanes:
            ln.capture(model)
        cg = geometry.get_c_geometry()
        P = geometry.nDetector[0] * geometry.nDetector[1]
        self.reproj_ws_bytes = _lib.lib.nectb_train_workspace_bytes(ctypes.byref(cg.c_struct),
                                                                    ctypes.byref(model.grid_desc),
                                                                    ctypes.byref(model.mlp_desc), P)
        self._stop = False
        self._thread = threading.Thread(target=self._run, daemon=True)
        self.completed: list[Request] = []
        self._lane_rr = 0
        self._thread.start()

    # -- client side ------------------------------------------------------
    def submit(self, req: Request) -> Request:
        req.arrival = time.perf_counter()
        self.queue.put(req)
        return req

    def close(self):
        self._stop = True
        self.queue.put(None)
        self._thread.join()

    # -- scheduler --------------------------------------------------------
    def _bytes(self, req: Request) -> int:
        n = int(np.prod(req.out_shape(self.geometry))) * 4
        return 2 * n + (self.reproj_ws_bytes if req.kind == "reproject" else 0)  # device + pinned host

    def _next_lane(self) -> _Lane:
        ln = self.lanes[self._lane_rr % len(self.lanes)]
        self._lane_rr += 1
        return ln

    def _run(self):
        torch.cuda.set_device(self.dev)
        waiting: list[Request] = []
        active: list[dict] = []       # admitted requests with their remaining work
        flying: list[dict] = []       # requests whose work is all launched
        while True:
            # take new arrivals without blocking while there is work
            block = not (waiting or active or flying)
            try:
                r = self.queue.get(block=block, timeout=None if block else 0.0)
                if r is None:
                    if not (waiting or active or flying):
                        return
                else:
                    waiting.append(r)
                while True:
                    r = self.queue.get_nowait()
                    if r is not None:
                        waiting.append(r)
            except queue.Empty:
                pass
            # admission by memory, in arrival order
            while waiting and self.in_use + self._bytes(waiting[0]) <= self.budget:
                r = waiting.pop(0)
                self.in_use += self._bytes(r)
                out = torch.empty(r.out_shape(self.geometry), device=self.dev)
                st = {"req": r, "out": out, "events": [], "host": torch.empty(out.shape, pin_memory=True)}
                if r.kind == "reproject":
                    ln = self._next_lane()
                    with torch.cuda.stream(ln.stream):
                        ws = torch.empty(self.reproj_ws_bytes, dtype=torch.uint8, device=self.dev)
                        reproject(self.model, self.geometry, r.angle, r.t, self.points_per_ray, out=out.view(-1),
                                  workspace=ws, stream=ln.stream)
                        st["host"].copy_(out, non_blocking=True)
                        ev = torch.cuda.Event()
                        ev.record(ln.stream)
                    st["ws"] = ws
                    st["events"].append(ev)
                    flying.append(st)
                else:
                    items = (slice_items(out, r.t, r.centre, r.u, r.v, self.scale, self.offset)
                             if r.kind == "slice" else volume_items(out, r.t, self.scale, self.offset))
                    st["items"] = items
                    active.append(st)
            # pack pending items of all active requests into launches (continuous batching)
            while active:
                ln = self._next_lane()
                batch, chunks, touched = [], 0, []
                for st in active:
                    while st["items"] and len(batch) < MAX_ITEMS - 1:
                        c = st["items"][0].chunks
                        if chunks + c > self.max_chunks:
                            break
                        batch.append(st["items"].pop(0))
                        chunks += c
                        if st not in touched:
                            touched.append(st)
                    if chunks >= self.max_chunks or len(batch) >= MAX_ITEMS - 1:
                        break
                if not batch:
                    break
                ev = ln.launch(batch)
                for st in touched:
                    st["events"].append(ev)
                    if not st["items"]:
                        with torch.cuda.stream(ln.stream):
                            st["host"].copy_(st["out"], non_blocking=True)
                            e2 = torch.cuda.Event()
                            e2.record(ln.stream)
                        st["events"].append(e2)
                for st in [s for s in active if not s["items"]]:
                    active.remove(st)
                    flying.append(st)
                if self.queue.qsize():
                    break   # admit newcomers between launches
            # completions
            for st in list(flying):
                if all(e.query() for e in st["events"]):
                    r = st["req"]
                    r.result = st["host"].numpy()
                    r.done = time.perf_counter()
                    self.in_use -= self._bytes(r)
                    flying.remove(st)
                    self.completed.append(r)
                    r.event.set()
            if not (waiting or active) and flying:
                time.sleep(0.0002)

    # -- statistics ---------------------------------------------------------
    def latency_stats(self) -> dict:
        out = {}
        for kind in ("slice", "reproject", "volume"):
            lat = np.array([r.latency_ms() for r in self.completed if r.kind == kind])
            if lat.size:
                out[kind] = {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
                             "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean())}
        return out
