"""The allocation-free training entry point, called through the C ABI.

nectb_train_step_static serves callers that cannot allocate device memory
(a foreign runtime binding the library's C ABI without a CUDA allocator, or a
loop that must not call cudaMalloc): its scratch is a library-owned
__device__ array instead of a caller workspace.  Two calls in a row must each
reproduce the workspace entry point (nectb_train_step) on the same batch, to
the tolerance the parity tests use for run-to-run differences of fp32
atomics (1e-5 relative on y_pred/loss, 1e-4 of the largest gradient entry).
This file is collected last so a failure here leaves every other test run.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(precision):
    from nect_b200.config import HashEncoderConfig, MLPNetConfig
    from nect_b200.network import HashGrid
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import RayBatch

    torch.manual_seed(5)
    geo = Geometry(nDetector=[64, 64], dDetector=[1.0, 1.0], mode="cone", DSD=300.0, DSO=200.0, nVoxel=[48] * 3,
                   dVoxel=[1.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=14, base_resolution=4,
                            finest_resolution=256)
    net = MLPNetConfig(n_hidden_layers=2, n_neurons=64, activation="ReLU", output_activation="Softplus")
    m = HashGrid(enc, net, precision=precision, device="cuda")
    with torch.no_grad():
        g = torch.Generator(device="cpu").manual_seed(2)
        m.table.copy_((torch.rand(m.table.shape, generator=g) * 2 - 1) * 0.3)
        m.refresh_half()
    P, S, R = 64 * 64, 96, 3000
    batch = RayBatch(perm=torch.randperm(P, device="cuda"), start=0, num_rays=R, points_per_ray=S, angle=1.3,
                     max_ray_distance_per_point=geo.max_distance_traveled / S,
                     jitter=torch.rand(R, device="cuda") - 0.5, detector_offset=torch.zeros(R, 2, device="cuda"),
                     projection=torch.rand(P, device="cuda"))
    return geo, m, batch


def _static_step(m, cg, batch, max_dist):
    from nect_b200 import _lib
    from nect_b200.trainer import c_batch

    tg = torch.zeros_like(m.table)
    mg = torch.zeros_like(m.mlp)
    y = torch.empty(batch.num_rays, device="cuda")
    loss = torch.empty(1, device="cuda")
    cb = c_batch(batch, max_dist, "l2")
    rc = _lib.lib.nectb_train_step_static(ctypes.byref(cg.c_struct), ctypes.byref(m.grid_desc),
                                          ctypes.byref(m.mlp_desc), m.grid_table.data_ptr(), m.mlp.data_ptr(),
                                          ctypes.byref(cb), tg.data_ptr(), mg.data_ptr(), y.data_ptr(),
                                          loss.data_ptr(), _lib.stream_ptr())
    _lib.check(rc, "nectb_train_step_static")
    return y, loss, tg, mg


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp(min=1e-30))


@pytest.mark.parametrize("precision", ["plain_fp32", "mixed"])
def test_static_entry_matches_workspace_entry_twice(cuda_device, precision):
    from nect_b200.trainer import Workspace, train_step

    geo, m, batch = _setup(precision)
    cg = geo.get_c_geometry()
    tg = torch.zeros_like(m.table)
    mg = torch.zeros_like(m.mlp)
    loss_ref, y_ref = train_step(m, cg, batch, geo.max_distance_traveled, tg, mg, Workspace(), "l2")
    for _ in range(2):
        y, loss, tg2, mg2 = _static_step(m, cg, batch, geo.max_distance_traveled)
        torch.cuda.synchronize()
        assert _rel(y, y_ref) < 1e-5
        assert abs(float(loss) - float(loss_ref)) <= 1e-5 * abs(float(loss_ref))
        assert _rel(tg2, tg) < 1e-4
        assert _rel(mg2, mg) < 1e-4


def test_static_entry_rejects_oversized_batches(cuda_device):
    from nect_b200 import _lib
    from nect_b200.trainer import c_batch

    geo, m, batch = _setup("plain_fp32")
    cap = _lib.lib.nectb_train_static_scratch_bytes()
    assert cap == (20 << 20) + 4096
    big = batch
    big.num_rays = 1 << 20  # needs 64 MiB of ray records: refused before any launch
    cb = c_batch(big, geo.max_distance_traveled, "l2")
    cg = geo.get_c_geometry()
    rc = _lib.lib.nectb_train_step_static(ctypes.byref(cg.c_struct), ctypes.byref(m.grid_desc),
                                          ctypes.byref(m.mlp_desc), m.grid_table.data_ptr(), m.mlp.data_ptr(),
                                          ctypes.byref(cb), 0, 0, 0, 0, _lib.stream_ptr())
    assert rc == 4  # NECTB_ERR_TOO_LARGE
    assert b"static scratch" in _lib.lib.nectb_last_error()
