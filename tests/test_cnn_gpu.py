"""The surrogate network on a B200: forward pass and gradients of the tcgen05
convolutions against the FP64 CPU oracle (with the device's bfloat16
rounding points), and training that learns."""
import numpy as np
import pytest

from oracle import cnn as ocnn
from gpu_2dising_b200 import engine, surrogate

pytestmark = pytest.mark.gpu

L = 64


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _data(B, seed):
    rs = np.random.default_rng(seed)
    # grids with varied magnetisation: a random fraction of +1 spins per grid
    f = rs.uniform(0.05, 0.95, size=B)
    g = np.where(rs.random((B, L, L)) < f[:, None, None], 1, -1).astype(np.int8)
    y = 1.0 / (1.0 + np.exp(-6.0 * g.reshape(B, -1).mean(axis=1)))
    return g, y.astype(np.float32)


def test_forward_matches_oracle():
    g, _ = _data(6, 1)
    params = surrogate.init_params(3)
    net = surrogate.CommittorCNN(L, 8, params)
    q = net.predict(g)
    ref = ocnn.forward(params.astype(np.float64), g.astype(np.float64), bf16=True)["q"]
    assert np.max(np.abs(q - ref)) < 2e-3, (q, ref)
    # and close to the exact FP64 network
    exact = ocnn.forward(params.astype(np.float64), g.astype(np.float64))["q"]
    assert np.max(np.abs(q - exact)) < 2e-2


def test_gradients_match_oracle():
    g, y = _data(4, 2)
    params = surrogate.init_params(5)
    # give the head and biases non-trivial values so every gradient is exercised
    params[-33:] = np.random.default_rng(0).normal(0, 0.5, 33).astype(np.float32)
    net = surrogate.CommittorCNN(L, 8, params)
    loss, grad = net.gradients(g, y)
    rloss, rgrad, _ = ocnn.loss_and_grads(params.astype(np.float64), g.astype(np.float64),
                                          y.astype(np.float64), bf16=True)
    assert abs(loss - rloss) < 1e-3 * max(1.0, abs(rloss))
    o = 0
    for name, shp in ocnn.SHAPES:
        n = int(np.prod(shp))
        a, b = grad[o:o + n].astype(np.float64), rgrad[o:o + n]
        o += n
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 2e-2, (name, rel)
        if np.linalg.norm(b) > 0:
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            assert cos > 0.999, (name, cos)


@pytest.mark.parametrize("Lo", [32, 128])
def test_other_sizes_forward_and_gradients_match_oracle(Lo):
    """The window convolutions at the other lattice sides with a row-aligned
    tile (a 128-pixel tile is 4 rows of 32 or 1 row of 128): forward and the
    loss gradient against the FP64 oracle."""
    rs = np.random.default_rng(Lo)
    f = rs.uniform(0.1, 0.9, size=3)
    g = np.where(rs.random((3, Lo, Lo)) < f[:, None, None], 1, -1).astype(np.int8)
    y = (1.0 / (1.0 + np.exp(-6.0 * g.reshape(3, -1).mean(axis=1)))).astype(np.float32)
    params = surrogate.init_params(9)
    params[-33:] = np.random.default_rng(1).normal(0, 0.5, 33).astype(np.float32)
    net = surrogate.CommittorCNN(Lo, 4, params)
    q = net.predict(g)
    ref = ocnn.forward(params.astype(np.float64), g.astype(np.float64), bf16=True)["q"]
    assert np.max(np.abs(q - ref)) < 2e-3, (q, ref)
    loss, grad = net.gradients(g, y)
    rloss, rgrad, _ = ocnn.loss_and_grads(params.astype(np.float64), g.astype(np.float64),
                                          y.astype(np.float64), bf16=True)
    assert abs(loss - rloss) < 1e-3 * max(1.0, abs(rloss))
    rel = np.linalg.norm(grad - rgrad) / np.linalg.norm(rgrad)
    assert rel < 2e-2, rel


def test_training_learns():
    g, y = _data(512, 3)
    gv, yv = _data(128, 4)
    net = surrogate.CommittorCNN(L, 256, surrogate.init_params(7))
    mae0 = float(np.mean(np.abs(net.predict(gv) - yv)))
    hist = net.train(g, y, epochs=12, batch=64, lr=3e-3, val=(gv, yv), augment=False)
    mae1 = hist[-1]["val_mae"]
    assert hist[-1]["loss"] < hist[0]["loss"]
    assert mae1 < 0.5 * mae0 and mae1 < 0.05, (mae0, hist)


def test_predict_returns_magnetisation_and_screen_shoots_out_of_window_grids():
    """gasp_cnn_predict_ex gives each grid's magnetisation from the upload;
    screening shoots grids outside the training window whatever the network
    predicts."""
    g, _ = _data(70, 5)  # more than one 32-grid batch of the 64-grid handle
    net = surrogate.CommittorCNN(L, 64, surrogate.init_params(2))
    q, m = net.predict(g, with_mag=True)
    # the pooled sums are accumulated with float atomics, so the last bit of q
    # may differ between calls
    assert np.allclose(q, net.predict(g), rtol=0, atol=1e-6)
    assert np.array_equal(m, (g.reshape(70, -1).astype(np.int64).sum(axis=1) / (L * L))
                          .astype(np.float32))
    inside = np.full((2, L, L), -1, np.int8)
    inside[:, :, :7] = 1  # m = -1 + 2*7/64, inside (-0.93, -0.65)
    grids = np.concatenate([inside, np.ones((1, L, L), np.int8), -np.ones((1, L, L), np.int8)])
    pb, shot, _ = surrogate.screen(net, grids, 0.54, 0.07, fallback_shots=16, band=0.0,
                                   window=(-0.93, -0.65), seed=4)
    assert shot.tolist() == [False, False, True, True]
    assert pb[2] == 1.0 and pb[3] == 0.0  # all up is in B, all down in A at once


def test_fused_forward_matches_layer_by_layer_and_oracle():
    """The whole-network kernel of the L=64 prediction path (one band of 8
    rows per work item, activations on the chip, ghost columns for the wrap)
    against the layer-by-layer kernels and the FP64 oracle with the same BF16
    rounding points; biases and head non-zero.  37 grids in a 16-grid handle:
    the chunked path with a ragged last chunk."""
    from gpu_2dising_b200._native import check, lib
    rs = np.random.default_rng(11)
    f = rs.uniform(0.05, 0.95, size=37)
    g = np.where(rs.random((37, L, L)) < f[:, None, None], 1, -1).astype(np.int8)
    params = surrogate.init_params(13)
    params[288:320] = rs.normal(0, 0.3, 32)                    # layer-1 bias
    for l in range(3):                                          # layer 2-4 biases
        o = 320 + 9216 + l * (9216 + 32)
        params[o:o + 32] = rs.normal(0, 0.2, 32)
    params[-33:] = rs.normal(0, 0.5, 33).astype(np.float32)
    net = surrogate.CommittorCNN(L, 16, params)
    check(lib().gasp_cnn_set_fused(net._h, 1))
    q_fused = net.predict(g)
    check(lib().gasp_cnn_set_fused(net._h, 0))
    q_layers = net.predict(g)
    check(lib().gasp_cnn_set_fused(net._h, 1))
    assert np.max(np.abs(q_fused - q_layers)) < 2e-5, np.max(np.abs(q_fused - q_layers))
    ref = ocnn.forward(params.astype(np.float64), g[:6].astype(np.float64), bf16=True)["q"]
    assert np.max(np.abs(q_fused[:6] - ref)) < 2e-3, (q_fused[:6], ref)
    assert np.max(np.abs(net.predict(g[:5]) - q_fused[:5])) < 2e-5  # one unchunked batch
