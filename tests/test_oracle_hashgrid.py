"""Known answers for the oracle's hash-grid index rules (CPU), worked out
here with plain integer arithmetic from the published method (Mueller et al.,
ACM TOG 41(4), 2022, section 3): per-level resolution, dense strides and the
multiple-of-8 rounding of dense levels, the XOR-of-primes hash modulo T, the
cell clamp at x = 1 and d-linear weights.  The kernels are compared with the
oracle bit for bit on GPUs; these cases pin the oracle itself."""
import pytest
import torch

from oracle import hashgrid as ohg


def hand_hash(v, T):
    primes = (1, 2654435761, 805459861, 2246822519)
    h = 0
    for k, vk in enumerate(v):
        h ^= (vk * primes[k]) & 0xFFFFFFFF
    return h % T


def test_layout_resolutions_rounding_and_offsets():
    levels, total = ohg.layout(3, 4, 12, 4.0, 2.0)
    assert [lv.res for lv in levels] == [(4, 4, 4), (8, 8, 8), (16, 16, 16), (32, 32, 32)]
    # 5^3 = 125 -> 128 entries; 9^3 = 729 -> 736; 17^3 = 4913 > 4096 -> hashed
    assert [(lv.entries, lv.hashed) for lv in levels] == [(128, False), (736, False), (4096, True), (4096, True)]
    assert [lv.offset for lv in levels] == [0, 128, 864, 4960] and total == 9056
    levels4, _ = ohg.layout(4, 2, 12, 4.0, 1.5, base_t=2.0)
    assert [lv.res for lv in levels4] == [(4, 4, 4, 2), (6, 6, 6, 3)]
    assert [(lv.entries, lv.hashed) for lv in levels4] == [(376, False), (1376, False)]   # 375, 1372 rounded up


def test_dense_level_indices_and_weights():
    lv = ohg.layout(3, 1, 12, 4.0, 2.0)[0][0]          # resolution 4, stride (1, 5, 25)
    x = torch.tensor([[0.3, 0.55, 0.9]])                # cell (1, 2, 3), fractions (0.2, 0.2, 0.6)
    idx, w = ohg.corner_indices(x, lv, 12)
    for corner in range(8):
        b = [(corner >> k) & 1 for k in range(3)]
        v = (1 + b[0], 2 + b[1], 3 + b[2])
        assert int(idx[0, corner]) == v[0] + 5 * v[1] + 25 * v[2]
        frac = (0.2, 0.2, 0.6)
        expect = 1.0
        for k in range(3):
            expect *= frac[k] if b[k] else 1 - frac[k]
        assert float(w[0, corner]) == pytest.approx(expect, abs=1e-6)
    assert float(w.sum()) == pytest.approx(1.0, abs=1e-6)


def test_hashed_level_indices_3d_and_4d():
    lv = ohg.layout(3, 6, 12, 4.0, 2.0)[0][5]          # resolution 128, hashed into 4096
    assert lv.hashed and lv.res == (128, 128, 128)
    x = torch.tensor([[0.5, 0.25, 0.75], [0.0123, 0.987, 0.5]])
    idx, _ = ohg.corner_indices(x, lv, 12)
    cells = [(64, 32, 96), (int(0.0123 * 128), int(0.987 * 128), 64)]
    for n, c in enumerate(cells):
        for corner in range(8):
            v = [c[k] + ((corner >> k) & 1) for k in range(3)]
            assert int(idx[n, corner]) == hand_hash(v, 4096)
    lv4 = ohg.layout(4, 4, 10, 4.0, 2.0, base_t=2.0)[0][3]   # (32, 32, 32, 16): 33^3 * 17 > 1024
    assert lv4.hashed and lv4.res == (32, 32, 32, 16)
    x4 = torch.tensor([[0.1, 0.2, 0.3, 0.4]])
    idx4, _ = ohg.corner_indices(x4, lv4, 10)
    c4 = (int(0.1 * 32), int(0.2 * 32), int(0.3 * 32), int(0.4 * 16))
    for corner in range(16):
        v = [c4[k] + ((corner >> k) & 1) for k in range(4)]
        assert int(idx4[0, corner]) == hand_hash(v, 1024)


def test_cell_clamp_at_the_upper_face():
    lv = ohg.layout(3, 1, 12, 4.0, 2.0)[0][0]
    idx, w = ohg.corner_indices(torch.tensor([[1.0, 1.0, 1.0]]), lv, 12)
    # x * 4 = 4 -> cell clamped to 3 with fraction 1: all weight on vertex (4, 4, 4)
    assert int(idx[0, 7]) == 4 + 5 * 4 + 25 * 4 and float(w[0, 7]) == 1.0
    assert float(w[0, :7].abs().sum()) == 0.0
