"""CPU checks of the network oracle: its backward pass against central finite
differences of its own forward pass (FP64), and the BF16 rounding helper."""
import numpy as np

import oracle


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], dtype=np.float32)
    r = oracle.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert np.all(np.abs(r[:4] - x[:4]) <= 2.0 ** -8 * np.abs(x[:4]))


def test_network_gradient_finite_differences():
    p = oracle.cnn_init(1).astype(np.float64)
    rng = np.random.default_rng(0)
    fbp = rng.normal(size=(1, 32, 32))
    tgt = fbp + 0.1 * rng.normal(size=fbp.shape)
    _, g = oracle.cnn_loss_and_grads(p, fbp, tgt, scale=1.5)
    # one weight with a non-zero gradient from every layer, plus a bias
    picks = []
    off = 0
    for ci, co, _ in oracle.CNN_LAYERS:
        n = co * 9 * ci
        seg = np.flatnonzero(np.abs(g[off:off + n]) > 1e-6 * np.abs(g).max())
        picks.append(off + int(seg[len(seg) // 2]))
        off += n + co
    picks.append(off - 16)  # bias of output channel 0
    for i in picks:
        h = 1e-5 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (oracle.cnn_loss_and_grads(pp, fbp, tgt, scale=1.5)[0] -
              oracle.cnn_loss_and_grads(pm, fbp, tgt, scale=1.5)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(g[i]), 1e-8) + 1e-12, (i, fd, g[i])


def test_pack_unpack_round_trip():
    p = oracle.cnn_init(3)
    assert p.size == oracle.cnn_num_params()
    assert np.array_equal(oracle.cnn_pack(oracle.cnn_unpack(p)).astype(np.float32), p)
