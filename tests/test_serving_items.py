"""Host-side query items of the serving path (CPU): the points an item
describes (point k = origin + (k % nu) du + (k // nu) dv, written to
out + ((k // nu) * out_stride + k % nu) floats, as the query kernels
evaluate them) reproduce create_volume's voxel-centre grid
(base_trainer.py:411-432) for volumes and axis-aligned slices; rows split
into items; chunk counts; and the request packing of the server."""
import numpy as np
import pytest

from nect_b200 import serving


def item_points(it):
    """(points [nv*nu, 3], float offsets of their outputs) of one item."""
    k = np.arange(int(it["nu"]) * int(it["nv"]))
    i, j = k % it["nu"], k // it["nu"]
    p = it["origin"][None, :] + i[:, None] * it["du"][None, :] + j[:, None] * it["dv"][None, :]
    return np.clip(p, 0, 1), j * it["out_stride"] + i


def test_volume_items_cover_the_voxel_centre_grid():
    nz, ny, nx = 3, 5, 4
    base = 1 << 20
    its = serving.volume_items(base, (nz, ny, nx), t=0.25, scale=2.0, offset=-1.0)
    assert its.size == nz
    vol = np.zeros((nz, ny, nx, 3))
    z, y, x = serving.centres(nz), serving.centres(ny), serving.centres(nx)
    for n, it in enumerate(its):
        assert (it["t"], it["out_scale"], it["out_offset"]) == (0.25, 2.0, -1.0)
        assert int(it["out"]) == base + 4 * n * ny * nx
        p, off = item_points(it)
        vol.reshape(-1, 3)[n * ny * nx + off] = p
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    assert np.allclose(vol, np.stack([Z, Y, X], -1), atol=1e-6)


def test_axis_aligned_slice_items_and_row_split():
    nv, nu = 10, 6
    its = serving.slice_items(0, (nv, nu), t=0.0, centre=(0.5, 0.5, 0.5), rows_per_item=4)
    assert list(its["nv"]) == [4, 4, 2] and list(its["out"]) == [0, 4 * 4 * nu, 4 * 8 * nu]
    img = np.zeros((nv, nu, 3))
    for it in its:
        p, off = item_points(it)
        img.reshape(-1, 3)[int(it["out"]) // 4 + off] = p
    Y, X = np.meshgrid(serving.centres(nv), serving.centres(nu), indexing="ij")
    assert np.allclose(img[..., 0], 0.5) and np.allclose(img[..., 1], Y) and np.allclose(img[..., 2], X)


def test_item_chunks_round_up():
    its = serving.volume_items(0, (2, 10, 13), 0.0)       # 130 points per item
    assert list(serving.item_chunks(its)) == [2, 2]
    assert serving.item_chunks(serving.volume_items(0, (1, 8, 16), 0.0))[0] == 1


def test_pack_fills_requests_in_order_within_the_chunk_limit():
    a = {"items": serving.volume_items(0, (3, 16, 16), 0.0)}     # 2 chunks per item
    b = {"items": serving.volume_items(0, (2, 8, 16), 0.0)}      # 1 chunk per item
    for st in (a, b):
        st["chunks"] = serving.item_chunks(st["items"])
    packed, touched = serving.QueryServer._pack([a, b], limit_chunks=7)
    assert packed.size == 4 and touched == [a, b]                # a's three items, one of b's
    assert a["items"].size == 0 and b["items"].size == 1
    packed, touched = serving.QueryServer._pack([b], limit_chunks=0)
    assert packed.size == 0 and touched == []
    c = {"items": serving.volume_items(0, (5, 16, 16), 0.0)}
    c["chunks"] = serving.item_chunks(c["items"])
    d = {"items": serving.volume_items(0, (1, 8, 16), 0.0)}
    d["chunks"] = serving.item_chunks(d["items"])
    packed, touched = serving.QueryServer._pack([c, d], limit_chunks=5)
    assert packed.size == 2 and touched == [c]                  # c unfinished: d waits its turn


def test_denormalisation_matches_create_volume():
    scale, offset = serving.denormalisation(4.0, minimum=1.0, maximum=3.0)
    sigma = np.array([0.0, 2.0, 8.0])
    assert np.allclose(sigma * scale + offset, sigma / 4.0 * (3.0 - 1.0) + 1.0)
    assert scale == pytest.approx(0.5)
