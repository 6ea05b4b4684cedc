"""The device-side error word of the bounded tensor-core waits.

Failure is made without any fault: the self-test kernel waits on an mbarrier
that nothing arrives at, with a small poll limit, and must end with its error
word set; the context must stay usable for a training step afterwards, whose
own error word must read 0."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(cuda_device):
    from nect_b200 import _lib
    from nect_b200.config import HashEncoderConfig, MLPNetConfig, ModelConfig, get_model
    from nect_b200.sampling import Geometry
    from nect_b200.trainer import Trainer

    word = torch.full((1,), 7, dtype=torch.int32, device=cuda_device)
    rc = _lib.lib.nectb_selftest_bounded_wait(word.data_ptr(), 256, _lib.stream_ptr(cuda_device))
    _lib.check(rc, "nectb_selftest_bounded_wait")
    assert int(word.item()) == 1, "a wait that nothing completes must give up and set the error word"
    with pytest.raises(RuntimeError):
        _lib.check(_lib.lib.nectb_selftest_bounded_wait(word.data_ptr(), 0, _lib.stream_ptr(cuda_device)), "x")

    # the context is still usable: a mixed (tcgen05) training step runs and reports no time-out
    geo = Geometry(nDetector=[64, 64], dDetector=[2.0, 2.0], mode="cone", DSD=1000.0, DSO=500.0,
                   nVoxel=[32] * 3, dVoxel=[2.0] * 3)
    enc = HashEncoderConfig(n_levels=16, n_features_per_level=2, log2_hashmap_size=14, base_resolution=4,
                            finest_resolution=64)
    model = get_model(ModelConfig("hash_grid", enc, MLPNetConfig(n_hidden_layers=2), "mixed"), device=cuda_device)
    tr = Trainer(model, geo, points_per_batch=4096 * 64, points_per_ray=64, device=cuda_device)
    proj = torch.rand(64 * 64, device=cuda_device)
    loss = tr.train_projection(proj, 0.3)
    torch.cuda.synchronize()
    assert torch.isfinite(loss).all()
    assert tr.device_error() == 0


def test_error_word_address_checks_arguments(cuda_device):
    from nect_b200 import _lib
    from nect_b200.sampling import Geometry

    geo = Geometry(nDetector=[16, 16], dDetector=[1.0, 1.0], mode="parallel", nVoxel=[8] * 3, dVoxel=[2.0] * 3)
    cg = geo.get_c_geometry()
    assert not _lib.lib.nectb_train_error_word(ctypes.byref(cg.c_struct), 0, None)
    addr = _lib.lib.nectb_train_error_word(ctypes.byref(cg.c_struct), 256, None)   # static scratch
    assert addr
    # more rays than the static scratch holds: no address (NECTB_ERR_TOO_LARGE), not one past its end
    assert not _lib.lib.nectb_train_error_word(ctypes.byref(cg.c_struct), 1 << 20, None)
    assert b"static scratch" in _lib.lib.nectb_last_error()
    # a geometry the library rejects gives no address either
    bad = Geometry(nDetector=[16, 16], dDetector=[1.0, 1.0], mode="parallel", nVoxel=[8] * 3,
                   dVoxel=[2.0] * 3).get_c_geometry()
    bad.c_struct.nDetector[0] = -16
    assert not _lib.lib.nectb_train_error_word(ctypes.byref(bad.c_struct), 256, None)
