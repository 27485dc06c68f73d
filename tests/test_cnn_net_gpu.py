"""Sparse-view correction network: forward pass and full-network gradients
against the FP64 oracle (with BF16 rounding emulated at the points where the
engine stores BF16), checkpoint round trip, and a short overfit."""
import numpy as np
import pytest

import oracle
from ufob import cnn as ucnn

pytestmark = pytest.mark.gpu


def _inputs(seed, B=2, N=64):
    rng = np.random.default_rng(seed)
    fbp = rng.normal(size=(B, N, N)).astype(np.float32)
    tgt = (fbp + 0.2 * rng.normal(size=fbp.shape)).astype(np.float32)
    return fbp, tgt


def _net_with(params, scale=1.0):
    net = ucnn.SparseViewNet(seed=3, scale=scale)
    net.set_state(ucnn.PARAMS, params)
    return net


@pytest.mark.parametrize("B,N,scale", [(2, 64, 1.0), (1, 128, 2.0), (3, 32, 0.5)])
def test_forward_matches_oracle(cuda, B, N, scale):
    import torch
    params = oracle.cnn_init(11)
    net = _net_with(params, scale)
    fbp, _ = _inputs(5, B, N)
    out = net.forward(torch.from_numpy(fbp).cuda()).cpu().numpy()
    ref = oracle.cnn_forward(params, fbp, scale=scale, bf16=True)
    # compare the correction (output minus input), the part the network computes
    err = oracle.rel_l2(out - fbp, ref - fbp)
    assert err < 1e-2, err
    ref64 = oracle.cnn_forward(params, fbp, scale=scale, bf16=False)
    assert oracle.rel_l2(out - fbp, ref64 - fbp) < 5e-2


@pytest.mark.parametrize("B,N", [(1, 512), (3, 64), (2, 96), (5, 32)])
def test_inference_path_matches_training_path(cuda, B, N):
    """The persistent padded-layout kernels (inference) against the NHWC
    kernels the gradients are taken through (training)."""
    import torch
    params = oracle.cnn_init(31)
    net = _net_with(params, scale=1.5)
    fbp = torch.from_numpy(_inputs(4, B, N)[0]).cuda()
    fast = net.forward(fbp)
    ref = net.forward_nhwc(fbp)
    torch.cuda.synchronize()
    err = oracle.rel_l2((fast - fbp).cpu().numpy(), (ref - fbp).cpu().numpy())
    assert err < 5e-3, err
    # weights changed by a train step are picked up by the inference path
    net.train_step(fbp, fbp, 1e-2)
    fast2, ref2 = net.forward(fbp), net.forward_nhwc(fbp)
    assert oracle.rel_l2((fast2 - fbp).cpu().numpy(), (ref2 - fbp).cpu().numpy()) < 5e-3
    assert oracle.rel_l2((fast2 - fbp).cpu().numpy(), (fast - fbp).cpu().numpy()) > 1e-3


def _layer_slices():
    off = 0
    for ci, co, _ in oracle.CNN_LAYERS:
        n = co * 9 * ci
        yield slice(off, off + n), slice(off + n, off + n + co)
        off += n + co


def test_gradients_match_oracle(cuda):
    import torch
    params = oracle.cnn_init(21)
    net = _net_with(params)
    fbp, tgt = _inputs(9, 2, 64)
    loss = net.train_step(torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda(), lr=0.0)
    g = net.get_state(ucnn.GRADS)
    ref_loss, ref_g = oracle.cnn_loss_and_grads(params, fbp, tgt, bf16=True)
    assert abs(loss - ref_loss) / ref_loss < 1e-3, (loss, ref_loss)
    _, g64 = oracle.cnn_loss_and_grads(params, fbp, tgt, bf16=False)
    for i, (sw, sb) in enumerate(_layer_slices()):
        ew = oracle.rel_l2(g[sw], ref_g[sw])
        eb = oracle.rel_l2(g[sb], ref_g[sb])
        assert ew < 2e-2 and eb < 2e-2, (i, ew, eb)
        assert oracle.rel_l2(g[sw], g64[sw]) < 1e-1, i
    # lr = 0 leaves the parameters untouched
    assert np.array_equal(net.get_state(ucnn.PARAMS), params)


def test_checkpoint_round_trip(cuda, tmp_path):
    import torch
    net = ucnn.SparseViewNet(seed=5)
    fbp, tgt = _inputs(1, 2, 64)
    x, y = torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda()
    for _ in range(3):
        net.train_step(x, y, 1e-3)
    path = str(tmp_path / "ck.npz")
    net.save(path, train_step=3)
    other = ucnn.SparseViewNet(seed=99)
    extra = other.load(path)
    assert int(extra["train_step"]) == 3 and other.step == net.step == 3
    for which in (ucnn.PARAMS, ucnn.ADAM_M, ucnn.ADAM_V):
        assert np.array_equal(other.get_state(which), net.get_state(which))
    # resumed and uninterrupted training take the same next step
    la = net.train_step(x, y, 1e-3)
    lb = other.train_step(x, y, 1e-3)
    assert la == pytest.approx(lb, rel=1e-6)
    assert np.allclose(other.get_state(ucnn.PARAMS), net.get_state(ucnn.PARAMS), rtol=0, atol=1e-6)


def test_overfit_reduces_loss(cuda):
    import torch
    net = ucnn.SparseViewNet(seed=7)
    fbp, tgt = _inputs(2, 4, 64)
    x, y = torch.from_numpy(fbp).cuda(), torch.from_numpy(tgt).cuda()
    first = net.train_step(x, y, 2e-3)
    for _ in range(60):
        last = net.train_step(x, y, 2e-3)
    assert last < 0.7 * first, (first, last)


def test_rejects_bad_shape(cuda):
    import torch
    from ufob import UfobError
    net = ucnn.SparseViewNet(seed=1)
    with pytest.raises(UfobError):
        net.forward(torch.zeros((1, 40, 40), device="cuda"))


def test_pairs_are_engine_made(cuda):
    import torch
    maker = ucnn.PairMaker(N=128, sparse=90, dense=720)
    x, y, imgs = maker.pair([1, 2])
    assert x.shape == y.shape == imgs.shape == (2, 128, 128)
    # the dense FBP is closer to the phantom than the sparse one
    e_sparse = ucnn.rel_l2(x, imgs)
    e_dense = ucnn.rel_l2(y, imgs)
    assert bool((e_dense < e_sparse).all())
    assert torch.isfinite(x).all() and torch.isfinite(y).all()


def test_pretrained_network_beats_plain_sparse_fbp(cuda):
    """The shipped weights (trained on engine-made pairs) lower the error of a
    90-angle FBP against the 1800-angle FBP on phantoms outside the training
    and evaluation seed ranges."""
    import torch
    net = ucnn.SparseViewNet.pretrained()
    maker = ucnn.PairMaker()
    x, y, _ = maker.pair(list(range(2_000_000, 2_000_008)))
    e_plain = ucnn.rel_l2(x, y)
    e_net = ucnn.rel_l2(net.forward(x), y)
    torch.cuda.synchronize()
    assert float(e_net.mean()) < 0.5 * float(e_plain.mean()), (float(e_net.mean()), float(e_plain.mean()))
    assert bool((e_net < e_plain).all())
