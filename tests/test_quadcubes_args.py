"""Argument checks and workspace size of QuadCubes' composite encoder
(nectb_quadcubes_workspace_bytes, nectb_quadcubes_encode, _backward).
Host-side only: every call here fails validation (or has n = 0) before a
pointer is dereferenced or a kernel launched, and the file is skipped where a
GPU is visible so that nothing here can reach a device."""
import ctypes

import pytest
import torch

from nect_b200 import _lib

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="host-side validation only")

NECTB_OK, NECTB_ERR_INVALID, NECTB_ERR_WORKSPACE = 0, 1, 3
A16 = ctypes.c_void_p(256)   # 16-byte aligned, never dereferenced
A4 = ctypes.c_void_p(260)    # 4-byte aligned only


def grid(n_dims=3, F=4, dtype=_lib.F32, log2_T=11, L=6):
    return _lib.NectbHashGrid(n_dims=n_dims, n_levels=L, n_features=F, log2_hashmap_size=log2_T, feature_dtype=dtype,
                              base_resolution=4.0, per_level_scale=1.65, base_resolution_t=0.0)


def ptrs(*p):
    return (ctypes.c_void_p * 4)(*p)


def plane_bytes(g):
    """Per level the (res+1)^2 vertices of the plane, or the T hashed entries
    where those are more, each rounded up to 8 entries; fp32 features."""
    L = g.n_levels
    res = (ctypes.c_int32 * L)()
    assert _lib.lib.nectb_hashgrid_layout(ctypes.byref(g), ctypes.addressof(res), None, None, None, None) > 0
    T = 1 << g.log2_hashmap_size
    total = sum(-(-min((r + 1) ** 2, T) // 8) * 8 for r in res)
    return -(-total * g.n_features * 4 // 256) * 256


def encode(g, n=100, tables=None, out=A16, ld=None, dtype=_lib.BF16, ws=A16, ws_bytes=1 << 30, identity=1):
    ld = ld if ld is not None else 128
    tables = tables if tables is not None else ptrs(A16, A16, A16, A16)
    return _lib.lib.nectb_quadcubes_encode(ctypes.byref(g), tables, A16, n, A16, identity, out, ld, dtype, ws,
                                           ws_bytes, None)


def backward(g, n=100, grads=None, dout=A16, ld=128, dtype=_lib.BF16, ws=A16, ws_bytes=1 << 30):
    grads = grads if grads is not None else ptrs(A16, A16, A16, A16)
    return _lib.lib.nectb_quadcubes_encode_backward(ctypes.byref(g), A16, n, A16, dout, ld, dtype, grads, ws,
                                                    ws_bytes, None)


def error():
    return _lib.lib.nectb_last_error().decode()


def test_workspace_bytes_is_one_fp32_plane():
    for g in (grid(), grid(F=2), grid(log2_T=19, L=12), grid(log2_T=8)):
        assert _lib.lib.nectb_quadcubes_workspace_bytes(ctypes.byref(g)) == plane_bytes(g)
    assert _lib.lib.nectb_quadcubes_workspace_bytes(ctypes.byref(grid(n_dims=4))) == 0
    assert _lib.lib.nectb_quadcubes_workspace_bytes(None) == 0


@pytest.mark.parametrize("kw,message", [
    ({"g": grid(n_dims=4)}, "3D with fp32 tables"),
    ({"g": grid(dtype=_lib.F16)}, "3D with fp32 tables"),
    ({"g": grid(F=3)}, "n_features"),
    ({"tables": ptrs(A16, A16, A4, A16)}, "16-byte aligned"),
    ({"tables": ptrs(A16, None, A16, A16)}, "16-byte aligned"),
    ({"dtype": _lib.F16}, "out_dtype"),
    ({"ld": 6 * 4 * 4 + 3}, "out_ld"),
    ({"identity": 0, "ld": 6 * 4 * 4 - 1}, "out_ld"),
    ({"ld": 100}, "16-byte aligned"),          # 100 bf16 = 200 bytes a row
    ({"out": A4}, "16-byte aligned"),
    ({"ws": A4}, "16-byte aligned"),
    ({"n": -1}, "negative"),
])
def test_encode_rejects(kw, message):
    g = kw.pop("g", grid())
    assert encode(g, **kw) == NECTB_ERR_INVALID
    assert message in error(), error()


def test_encode_small_workspace_and_empty_call():
    g = grid()
    assert encode(g, ws_bytes=plane_bytes(g) - 256) == NECTB_ERR_WORKSPACE
    assert encode(g, n=0, tables=ptrs(None, None, None, None), out=None) == NECTB_OK   # nothing to do


@pytest.mark.parametrize("kw,message", [
    ({"g": grid(n_dims=4)}, "3D with fp32 tables"),
    ({"grads": ptrs(A16, A16, A16, A4)}, "16-byte aligned"),
    ({"dtype": _lib.F16}, "dout_dtype"),
    ({"ld": 6 * 4 * 4 - 1}, "dout_ld"),
    ({"ld": 100}, "16-byte aligned"),
    ({"dout": A4}, "16-byte aligned"),
])
def test_backward_rejects(kw, message):
    g = kw.pop("g", grid())
    assert backward(g, **kw) == NECTB_ERR_INVALID
    assert message in error(), error()


def test_backward_small_workspace():
    g = grid()
    assert backward(g, ws_bytes=plane_bytes(g) - 256) == NECTB_ERR_WORKSPACE
