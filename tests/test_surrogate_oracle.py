"""The surrogate's CPU restatement (oracle/surrogate_oracle.py) checked by
finite differences, and its input/output stages by their defining identities.
These are the references the GPU kernels are compared with."""
import numpy as np

from oracle import surrogate_oracle as SO


def _fd(f, a, idx, h=1e-6):
    a1, a2 = a.copy(), a.copy()
    a1[idx] += h
    a2[idx] -= h
    return (f(a1) - f(a2)) / (2 * h)


def test_conv_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    B, T, C, N, dil = 2, 40, 3, 4, 5
    x = rng.standard_normal((B, T, C))
    w = rng.standard_normal((N, 3, C))
    b = rng.standard_normal(N)
    dy = rng.standard_normal((B, T, N))
    f_x = lambda xx: float(np.sum(SO.conv(xx, w, b, dil) * dy))  # noqa: E731
    f_w = lambda ww: float(np.sum(SO.conv(x, ww, b, dil) * dy))  # noqa: E731
    gx = SO.conv_input_grad(dy, w, dil)
    gw, gb = SO.conv_weight_grad(dy, x, dil)
    for idx in [(0, 0, 0), (1, 7, 2), (0, T - 1, 1), (1, 3, 0)]:
        assert abs(_fd(f_x, x, idx) - gx[idx]) < 1e-6
    for idx in [(0, 0, 0), (3, 2, 2), (1, 1, 1)]:
        assert abs(_fd(f_w, w, idx) - gw[idx]) < 1e-6
    f_b = lambda bb: float(np.sum(SO.conv(x, w, bb, dil) * dy))  # noqa: E731
    assert abs(_fd(f_b, b, (2,)) - gb[2]) < 1e-6


def test_projected_output_layer_gradient():
    """With outputs z = P (W x + b) (P removes the channel mean), dL/dW equals
    the weight gradient of the projected upstream gradient."""
    rng = np.random.default_rng(1)
    B, T, C, N, cv, dil, margin = 1, 30, 4, 5, 5, 2, 3
    x = rng.standard_normal((B, T, C))
    w = rng.standard_normal((N, 3, C))
    b = rng.standard_normal(N)
    tgt = rng.standard_normal((B, T, N))

    def loss_of(ww, bb):
        wp, bp = SO.project_outputs(ww, bb)
        out = SO.conv(x, wp, bp, dil)
        return SO.mse_residual(out, None, tgt, cv, margin)[0]

    wp, bp = SO.project_outputs(w, b)
    out = SO.conv(x, wp, bp, dil)
    assert np.allclose(out.sum(axis=-1), 0.0, atol=1e-12)
    _, g = SO.mse_residual(out, None, tgt, cv, margin, project=True)
    assert np.allclose(g.sum(axis=-1), 0.0, atol=1e-15)
    gw, gb = SO.conv_weight_grad(g, x, dil)
    for idx in [(0, 0, 0), (4, 2, 3), (2, 1, 1)]:
        assert abs(_fd(lambda ww: loss_of(ww, b), w, idx) - gw[idx]) < 1e-7
    assert abs(_fd(lambda bb: loss_of(w, bb), b, (3,)) - gb[3]) < 1e-7


def test_huber_gradient():
    rng = np.random.default_rng(4)
    out = rng.standard_normal((1, 20, 4))
    tgt = rng.standard_normal((1, 20, 4))
    _, g = SO.mse_residual(out, None, tgt, 3, 2, delta=0.7)
    f = lambda o: SO.mse_residual(o, None, tgt, 3, 2, delta=0.7)[0]  # noqa: E731
    for idx in [(0, 2, 0), (0, 10, 2), (0, 17, 1), (0, 5, 3), (0, 0, 0)]:
        assert abs(_fd(f, out, idx) - g[idx]) < 1e-8


def test_two_layer_chain_with_relu():
    rng = np.random.default_rng(2)
    B, T, C, H, N, margin = 1, 50, 3, 6, 3, 4
    x = rng.standard_normal((B, T, C))
    w1, b1 = rng.standard_normal((H, 3, C)), rng.standard_normal(H)
    w2, b2 = rng.standard_normal((N, 3, H)), rng.standard_normal(N)
    tgt = rng.standard_normal((B, T, N))

    def loss_of(ww1):
        a = np.maximum(SO.conv(x, ww1, b1, 1), 0)
        return SO.mse_residual(SO.conv(a, w2, b2, 2), None, tgt, N, margin)[0]

    z1 = SO.conv(x, w1, b1, 1)
    a1 = np.maximum(z1, 0)
    _, g = SO.mse_residual(SO.conv(a1, w2, b2, 2), None, tgt, N, margin)
    ga = SO.conv_input_grad(g, w2, 2) * (a1 > 0)
    gw1, _ = SO.conv_weight_grad(ga, x, 1)
    for idx in [(0, 0, 0), (5, 2, 2), (3, 1, 1)]:
        assert abs(_fd(loss_of, w1, idx) - gw1[idx]) < 1e-6


def test_stages_identities():
    rng = np.random.default_rng(3)
    S, K, N = 3, 10, 200
    count = rng.integers(1, 9, size=(S, K)).astype(np.int32)
    count[2, 9] = 0
    imf_sum = rng.standard_normal((S, K, N)) * count[:, :, None]
    imf_sum[2, 9] = 0.0
    x = rng.standard_normal((S, N))
    scale = SO.rms(x)
    inp = SO.prepare(imf_sum, count, x, scale)
    # channels times the scale sum back to x
    assert np.allclose((inp[:, :, :K + 1].sum(axis=-1)) * scale[:, None], x, atol=1e-12)
    # a zero network output serves the small-ensemble decomposition exactly
    imfs, res, recon, _, _, _ = SO.combine(imf_sum, count, x, scale, np.zeros((S, N, 16)), 6)
    means, r = SO.means_and_residual(imf_sum, count, x)
    assert np.array_equal(imfs, means) and np.array_equal(res, r)
    assert np.all(recon < 1e-15)
    # any correction of the first P modes keeps the reconstruction and leaves
    # the later modes alone
    net = rng.standard_normal((S, N, 16))
    imfs, res, recon, _, _, _ = SO.combine(imf_sum, count, x, scale, net, 6)
    assert np.all(recon < 1e-12)
    assert np.array_equal(imfs[:, 6:], means[:, 6:])
    # orthogonal components have index 0; two equal components have index 1/2
    t = np.arange(1000) / 1000
    c = np.vstack([np.sin(2 * np.pi * 5 * t), np.sin(2 * np.pi * 11 * t)])
    assert abs(SO.orthogonality_index(c, c.sum(axis=0))) < 1e-12
    d = np.vstack([c[0], c[0]])
    assert abs(SO.orthogonality_index(d, d.sum(axis=0)) - 0.5) < 1e-12
