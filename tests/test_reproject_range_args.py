"""Argument checks of the piecewise re-projection (nectb_query_reproject_range)
and the size of its time-slice room (nectb_query_reproject_slice_bytes).
Host-side only: every call here fails validation before a pointer is
dereferenced or a kernel launched, and the file is skipped where a GPU is
visible so that nothing here can reach a device."""
import ctypes

import pytest
import torch

from nect_b200 import _lib
from nect_b200.sampling import Geometry

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="host-side validation only")

NECTB_ERR_INVALID, NECTB_ERR_WORKSPACE = 1, 3
FAKE = ctypes.c_void_p(16)  # never dereferenced: validation fails first


def grid(n_dims, dtype=_lib.F16, log2_T=12):
    return _lib.NectbHashGrid(n_dims=n_dims, n_levels=16, n_features=2, log2_hashmap_size=log2_T,
                              feature_dtype=dtype, base_resolution=4.0, per_level_scale=1.3,
                              base_resolution_t=2.0 if n_dims == 4 else 0.0)


def mlp(dtype=_lib.BF16):
    return _lib.NectbMLP(n_input=32, n_hidden_layers=2, width=64, activation=_lib.ACT["relu"],
                         output_activation=_lib.ACT["softplus"], compute_dtype=dtype)


GEO = Geometry(nDetector=[48, 40], dDetector=[1.2, 1.2], mode="cone", DSD=250.0, DSO=160.0, nVoxel=[32] * 3,
               dVoxel=[1.0] * 3)


def call(begin, count, ws_bytes, warpgroups=3):
    cg = GEO.get_c_geometry()
    g, m = grid(4), mlp()
    return _lib.lib.nectb_query_reproject_range(ctypes.byref(cg.c_struct), ctypes.byref(g), ctypes.byref(m), FAKE,
                                                FAKE, 0.5, 0.5, 64, 1.0, 64.0, FAKE, begin, count, FAKE, ws_bytes, 0,
                                                warpgroups, None)


@pytest.mark.parametrize("begin,count,warpgroups,message", [
    (0, 48 * 40 + 1, 3, "pixel range"),     # past the last detector pixel
    (-1, 10, 3, "pixel range"),
    (1900, 30, 3, "pixel range"),
    (0, 0, 3, "pixel range"),
    (0, 100, 7, "warpgroups_per_sm"),
])
def test_bad_ranges_are_rejected(begin, count, warpgroups, message):
    assert call(begin, count, 1 << 30, warpgroups) == NECTB_ERR_INVALID
    assert message in _lib.lib.nectb_last_error().decode()


def test_small_workspace_is_rejected():
    assert call(0, 100, 64 * 100) == NECTB_ERR_WORKSPACE   # the ray records alone


def test_slice_room_only_for_4d_mixed_models():
    g4, g3 = grid(4), grid(3)
    assert _lib.lib.nectb_query_reproject_slice_bytes(ctypes.byref(g3), ctypes.byref(mlp()), 100) == 0
    assert _lib.lib.nectb_query_reproject_slice_bytes(ctypes.byref(grid(4, _lib.F32)),
                                                      ctypes.byref(mlp(_lib.F32)), 100) == 0
    # the fp16 slice of every level: the 4D level's hashed size, or its dense 3D vertices (rounded up to 8)
    L = 16
    res = (ctypes.c_int32 * L)()
    rt = (ctypes.c_int32 * L)()
    off = (ctypes.c_int64 * L)()
    ent = (ctypes.c_int64 * L)()
    hsh = (ctypes.c_int32 * L)()
    assert _lib.lib.nectb_hashgrid_layout(ctypes.byref(g4), ctypes.addressof(res), ctypes.addressof(rt),
                                          ctypes.addressof(off), ctypes.addressof(ent), ctypes.addressof(hsh)) > 0
    n3 = sum(1 << 12 if hsh[l] else ((res[l] + 1) ** 3 + 7) // 8 * 8 for l in range(L))
    want = (n3 * 2 * 2 + 255) // 256 * 256 + 512
    assert _lib.lib.nectb_query_reproject_slice_bytes(ctypes.byref(g4), ctypes.byref(mlp()), 100) == want


def test_time_slice_arguments():
    """nectb_time_slice_bytes is the fp16 slice alone (0 without a slice);
    nectb_time_slice rejects t outside [0, 1], a small buffer, 3D grids and
    fp32 tables before any device work."""
    g4 = grid(4)
    n = _lib.lib.nectb_time_slice_bytes(ctypes.byref(g4))
    assert n > 0
    assert (n + 255) // 256 * 256 + 512 == _lib.lib.nectb_query_reproject_slice_bytes(ctypes.byref(g4),
                                                                                       ctypes.byref(mlp()), 1)
    assert _lib.lib.nectb_time_slice_bytes(ctypes.byref(grid(3))) == 0
    assert _lib.lib.nectb_time_slice_bytes(ctypes.byref(grid(4, _lib.F32))) == 0
    ts = _lib.lib.nectb_time_slice
    assert ts(ctypes.byref(g4), FAKE, 1.5, FAKE, n, None) == NECTB_ERR_INVALID
    assert ts(ctypes.byref(g4), FAKE, float("nan"), FAKE, n, None) == NECTB_ERR_INVALID
    assert ts(ctypes.byref(g4), FAKE, 0.5, FAKE, n - 2, None) == NECTB_ERR_WORKSPACE
    assert ts(ctypes.byref(grid(3)), FAKE, 0.5, FAKE, n, None) == NECTB_ERR_INVALID
    assert ts(ctypes.byref(g4), None, 0.5, FAKE, n, None) == NECTB_ERR_INVALID
    q = _lib.lib.nectb_query_points_slice
    assert q(ctypes.byref(grid(3)), ctypes.byref(mlp()), FAKE, FAKE, FAKE, 1, 1, FAKE, 0, None) == NECTB_ERR_INVALID
