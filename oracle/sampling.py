"""ctypes wrapper of the C sampling oracle (oracle/sampling.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
baseline of bench.py as the checker and CPU reference path; the product path
never imports it.  Builds ``oracle/_build/liboracle.so`` with ``make`` on first
use.  Calls release the GIL, so ``oracle_sample`` splits the rays over a thread
pool to use all host cores.
"""
from __future__ import annotations

import concurrent.futures
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"


class Geometry(ctypes.Structure):
    """Same layout as NectbGeometry in include/nectb.h."""
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("nDetector", ctypes.c_int32 * 2),
        ("dDetector", ctypes.c_float * 2),
        ("offOrigin", ctypes.c_float * 3),
        ("offDetector", ctypes.c_float * 2),
        ("rotDetector", ctypes.c_float * 3),
        ("COR", ctypes.c_float),
        ("distance_source_to_origin", ctypes.c_float),
        ("distance_origin_to_detector", ctypes.c_float),
        ("sVoxel", ctypes.c_float * 3),
        ("dVoxel", ctypes.c_float * 3),
        ("object_radius", ctypes.c_float),
        ("object_height", ctypes.c_float),
        ("remove_factor_top", ctypes.c_float),
        ("remove_factor_bottom", ctypes.c_float),
    ]


def build() -> Path:
    src = HERE / "sampling.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        P = ctypes.c_void_p
        _lib.oracle_sample.argtypes = [ctypes.POINTER(Geometry), P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, P, P, P, P, P, P]
        _lib.oracle_sample.restype = ctypes.c_int
        _lib.oracle_trig.argtypes = [ctypes.POINTER(Geometry), ctypes.c_float, P]
        _lib.oracle_trig.restype = None
    return _lib


def to_struct(geom) -> Geometry:
    """Copy any object exposing the NectbGeometry fields (e.g. the product's
    geometry classes or a dict) into the oracle's struct."""
    g = Geometry()
    src = geom.c_struct if hasattr(geom, "c_struct") else geom
    for name, ctype in Geometry._fields_:
        val = src[name] if isinstance(src, dict) else getattr(src, name)
        if name == "kind":
            g.kind = int(val)
        elif ctype is ctypes.c_float:
            setattr(g, name, float(val))
        else:
            arr = getattr(g, name)
            for i, v in enumerate(val):
                arr[i] = v
    return g


def host_trig(g: Geometry, angle: float) -> np.ndarray:
    out = np.zeros(8, np.float32)
    lib().oracle_trig(ctypes.byref(g), ctypes.c_float(angle), out.ctypes.data)
    return out


def oracle_sample(g: Geometry, perm: np.ndarray, start: int, num_rays: int, S: int, angle: float, maxd: float,
                  uniform: bool, jitter: np.ndarray, det_off: np.ndarray, trig: np.ndarray | None = None,
                  want_points: bool = True, threads: int | None = None):
    """Returns (points [R,S,3] or None, distances [R], counts [R]) as numpy."""
    perm = np.ascontiguousarray(perm, np.int64)
    jitter = np.ascontiguousarray(jitter, np.float32)
    det_off = np.ascontiguousarray(det_off, np.float32).reshape(-1)
    if trig is None:
        trig = host_trig(g, angle)
    trig = np.ascontiguousarray(trig, np.float32)
    points = np.empty((num_rays, S, 3), np.float32) if want_points else None
    dist = np.empty(num_rays, np.float32)
    counts = np.empty(num_rays, np.int32)
    threads = threads or os.cpu_count() or 1
    chunk = max(1, -(-num_rays // (threads * 4)))
    L = lib()

    def run(lo):
        hi = min(num_rays, lo + chunk)
        n = hi - lo
        # rays [lo, hi) are rays [start+lo, start+hi) of perm
        L.oracle_sample(ctypes.byref(g), perm.ctypes.data, perm.size, start + lo, n, S, ctypes.c_float(angle),
                        ctypes.c_float(maxd), 1 if uniform else 0, jitter[lo:].ctypes.data,
                        det_off[2 * lo:].ctypes.data, trig.ctypes.data,
                        points[lo:].ctypes.data if points is not None else None, dist[lo:].ctypes.data,
                        counts[lo:].ctypes.data)

    if threads == 1 or num_rays <= chunk:
        for lo in range(0, num_rays, chunk):
            run(lo)
    else:
        with concurrent.futures.ThreadPoolExecutor(threads) as ex:
            list(ex.map(run, range(0, num_rays, chunk)))
    return points, dist, counts
