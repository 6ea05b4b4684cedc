"""Model shapes outside the instantiated set (dispatch_shape: 16 levels of 2 or
4 features with 2 or 3 hidden layers in 3D and 4D, and the reference's
default static model of 19 levels of 4 features with 6 hidden layers) are
rejected through the C ABI
with NECTB_ERR_INVALID and a message, before any device work (they are not
run on another path).  Host-side checks only: the calls fail validation, so
no pointer is dereferenced and no kernel is launched; they are skipped where
a GPU is visible so that nothing here can reach a device."""
import ctypes

import pytest
import torch

from nect_b200 import _lib

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="host-side validation only")

NECTB_ERR_INVALID = 1
FAKE = ctypes.c_void_p(16)  # never dereferenced: validation fails first


def grid(n_dims=3, n_levels=16, F=2, dtype=_lib.F32):
    return _lib.NectbHashGrid(n_dims=n_dims, n_levels=n_levels, n_features=F, log2_hashmap_size=12,
                              feature_dtype=dtype, base_resolution=4.0, per_level_scale=1.3,
                              base_resolution_t=2.0 if n_dims == 4 else 0.0)


def mlp(n_input, H=2, width=64, act="relu"):
    return _lib.NectbMLP(n_input=n_input, n_hidden_layers=H, width=width, activation=_lib.ACT[act],
                         output_activation=_lib.ACT["softplus"], compute_dtype=_lib.F32)


def model_forward(g, m):
    return _lib.lib.nectb_model_forward(ctypes.byref(g), ctypes.byref(m), FAKE, FAKE, FAKE, 10, 0.0, FAKE, None)


def model_backward(g, m):
    return _lib.lib.nectb_model_backward(ctypes.byref(g), ctypes.byref(m), FAKE, FAKE, FAKE, 10, 0.0, FAKE, FAKE,
                                         FAKE, None)


def last_error():
    return _lib.lib.nectb_last_error().decode()


@pytest.mark.parametrize("call", [model_forward, model_backward])
@pytest.mark.parametrize("n_dims,n_levels,F,H,width,act,message", [
    (3, 16, 8, 2, 64, "relu", "unsupported configuration"),   # 8 features per level
    (4, 16, 1, 2, 64, "relu", "unsupported configuration"),   # 1 feature per level
    (3, 16, 2, 1, 64, "relu", "unsupported configuration"),   # one hidden layer
    (3, 16, 4, 6, 64, "relu", "unsupported configuration"),  # six hidden layers over 16 levels
    (3, 19, 4, 2, 64, "relu", "unsupported configuration"),  # 19 levels with two hidden layers
    (3, 19, 4, 7, 64, "leakyrelu", "n_hidden_layers"),       # seven hidden layers
    (4, 19, 4, 6, 64, "leakyrelu", "unsupported configuration"),  # the reference's static shape, in 4D
    (3, 16, 2, 2, 128, "relu", "width"),                     # width 128
    (3, 16, 2, 2, 64, "sigmoid", "hidden activation"),       # sigmoid hidden layers
])
def test_unsupported_model_shapes_are_rejected(call, n_dims, n_levels, F, H, width, act, message):
    g = grid(n_dims, n_levels, F)
    rc = call(g, mlp(n_levels * F, H, width, act))
    assert rc == NECTB_ERR_INVALID
    assert message in last_error(), last_error()
