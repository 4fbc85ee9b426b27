"""The surrogate end to end on the GPU: the projected output layer, the input
and output stages and the gate against oracle/surrogate_oracle.py, the whole
network's gradient against an oracle backpropagation, and a short training
run that must beat the small-ensemble mean it starts from."""
import numpy as np
import pytest

from oracle import surrogate_oracle as SO

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from eemd4cuda_b200 import _sg  # noqa: E402
from eemd4cuda_b200 import surrogate as SU  # noqa: E402


def bf16r(a):
    """round to bfloat16 (nearest even), back to float64"""
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).double().numpy()


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


def test_projected_pack_bias_and_loss():
    rng = np.random.default_rng(11)
    nv, cv, N, C = 11, 64, 16, 64
    w = rng.standard_normal((nv, 3, cv)).astype(np.float32)
    b = rng.standard_normal(nv).astype(np.float32)
    wd, bd = dev(w), dev(b)
    wp = torch.empty((N * 3 * C,), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty((C * 3 * N,), dtype=torch.bfloat16, device="cuda")
    bias = torch.empty((N,), dtype=torch.float32, device="cuda")
    _sg.pack(wd, wp, N, C, nv, cv, project=True)
    _sg.pack(wd, wt, C, N, cv, nv, transpose=True, project=True)
    _sg.bias(bd, bias, N, nv, project=True)
    # a convolution with the projected operands has outputs of zero channel sum
    B, T = 2, 500
    x = rng.standard_normal((B, T, C)).astype(np.float32)
    y = torch.empty((B, T, N), dtype=torch.bfloat16, device="cuda")
    _sg.conv(dev(x, torch.bfloat16), wp, bias, y, B, T, C, N, 4)
    torch.cuda.synchronize()
    ye = y.double().cpu().numpy()
    wq, bq = SO.project_outputs(w.astype(np.float64), b.astype(np.float64))
    ref = SO.conv(bf16r(x), bf16r(wq), bq, 4)
    assert np.allclose(ye[..., nv:], 0.0)
    assert np.max(np.abs(ye[..., :nv] - ref)) <= 2 ** -7 * np.max(np.abs(ref)) + 1e-2
    assert np.max(np.abs(ye[..., :nv].sum(axis=-1))) <= nv * 2 ** -8 * np.max(np.abs(ref))
    assert np.allclose(bias.cpu().numpy()[:nv], bq, atol=1e-6)
    assert np.allclose(bias.cpu().numpy()[nv:], 0.0)
    # the transposed operand is the transpose of the projected one
    dy = rng.standard_normal((B, T, N)).astype(np.float32)
    dy[..., nv:] = 0
    dx = torch.empty((B, T, C), dtype=torch.bfloat16, device="cuda")
    _sg.conv(dev(dy, torch.bfloat16), wt, None, dx, B, T, N, C, 4, direction=-1)
    torch.cuda.synchronize()
    gi = SO.conv_input_grad(bf16r(dy)[..., :nv], bf16r(wq), 4)
    assert np.max(np.abs(dx.double().cpu().numpy() - gi)) <= 2 ** -7 * np.max(np.abs(gi)) + 1e-2
    # loss with the projected gradient and no base
    out = rng.standard_normal((B, T, 16)).astype(np.float32)
    tgt = rng.standard_normal((B, T, 16)).astype(np.float32)
    dout = torch.empty((B, T, 16), dtype=torch.bfloat16, device="cuda")
    acc = torch.zeros((1,), dtype=torch.float32, device="cuda")
    _sg.loss(dev(out, torch.bfloat16), None, dev(tgt, torch.bfloat16), dout, acc, B, T, 16, nv, 30, project=True)
    torch.cuda.synchronize()
    lo, go = SO.mse_residual(bf16r(out), None, bf16r(tgt), nv, 30, project=True)
    assert abs(float(acc.item()) - lo) <= 1e-4 * lo
    assert np.max(np.abs(dout.double().cpu().numpy() - go)) <= 2 ** -7 * np.max(np.abs(go))
    # the Huber form with channel weights
    wch = rng.random(nv).astype(np.float32) + 0.5
    acc.zero_()
    _sg.loss(dev(out, torch.bfloat16), None, dev(tgt, torch.bfloat16), dout, acc, B, T, 16, nv, 30, project=True,
             delta=0.5, weights=dev(wch))
    torch.cuda.synchronize()
    lo, go = SO.mse_residual(bf16r(out), None, bf16r(tgt), nv, 30, project=True, delta=0.5, weights=wch)
    assert abs(float(acc.item()) - lo) <= 1e-4 * lo
    assert np.max(np.abs(dout.double().cpu().numpy() - go)) <= 2 ** -7 * np.max(np.abs(go))


def test_scale_prepare_combine_and_gate():
    rng = np.random.default_rng(12)
    S, K, N, C = 5, 10, 3000, 16
    count = rng.integers(1, 9, size=(S, K)).astype(np.int32)
    count[4, 8:] = 0
    x = rng.standard_normal((S, N)).astype(np.float32) * np.array([1, 2, 0.5, 3, 1], np.float32)[:, None]
    imf_sum = rng.standard_normal((S, K, N)) * 0.3 * count[:, :, None]
    imf_sum[4, 8:] = 0.0
    count2 = count + 3
    imf_sum2 = imf_sum * 1.1 + 0.01
    xd = dev(x)
    sd, cd = dev(imf_sum, torch.float64), dev(count, torch.int32)
    s2, c2 = dev(imf_sum2, torch.float64), dev(count2, torch.int32)
    scale = torch.empty((S,), dtype=torch.float32, device="cuda")
    _sg.scale(xd, scale, S, N)
    inp = torch.empty((S, N, C), dtype=torch.bfloat16, device="cuda")
    dif = torch.empty_like(inp)
    _sg.prepare(sd, cd, xd, scale, inp, S, N, K, C)
    _sg.prepare(sd, cd, xd, scale, dif, S, N, K, C, imf_sum2=s2, mode_count2=c2)
    torch.cuda.synchronize()
    sc = SO.rms(x)
    assert np.allclose(scale.cpu().numpy(), sc, rtol=1e-6)
    ref = SO.prepare(imf_sum, count, x, sc.astype(np.float32).astype(np.float64), C)
    got = inp.double().cpu().numpy()
    assert np.max(np.abs(got - bf16r(ref))) <= 2 ** -8 * np.max(np.abs(ref))
    ref2 = ref - SO.prepare(imf_sum2, count2, x, sc.astype(np.float32).astype(np.float64), C)
    assert np.max(np.abs(dif.double().cpu().numpy() - ref2)) <= 2 ** -8 * np.max(np.abs(ref2))
    # combine: corrections of the first P modes; a non-finite output planted
    # in the test's network output for signal 4
    P = 6
    net = rng.standard_normal((S, N, C)).astype(np.float32) * 0.05
    net[4, 100, 2] = np.nan
    netq = bf16r(net)
    imfs = torch.empty((S, K, N), dtype=torch.float64, device="cuda")
    res = torch.empty((S, N), dtype=torch.float64, device="cuda")
    chunks = 7
    part = torch.empty((S * chunks * _sg.stat_count(),), dtype=torch.float64, device="cuda")
    met = torch.empty((S, 4), dtype=torch.float64, device="cuda")
    fb = torch.empty((S,), dtype=torch.int32, device="cuda")
    sc32 = sc.astype(np.float32).astype(np.float64)
    oi, orr, orec, oio, oio_all, oio_ref = SO.combine(imf_sum, count, x, sc32, netq, P)
    io_bound = float(np.median(np.abs(oio[:4])))
    _sg.combine(sd, cd, xd, scale, dev(net, torch.bfloat16), imfs, res, part, chunks, S, N, K, C, P, 1e-3,
                io_bound, met, fb, io_relative=False)
    torch.cuda.synchronize()
    gi, gr, m = imfs.cpu().numpy(), res.cpu().numpy(), met.cpu().numpy()
    assert np.allclose(gi[:4], oi[:4], rtol=1e-12, atol=1e-12)
    assert np.allclose(gr[:4], orr[:4], rtol=1e-12, atol=1e-12)
    assert np.array_equal(gi[:, P:], oi[:, P:])
    assert np.all(m[:4, 0] < 1e-12)
    assert np.allclose(m[:4, 1], oio[:4], rtol=1e-9, atol=1e-12)
    assert np.allclose(m[:4, 2], oio_all[:4], rtol=1e-9, atol=1e-12)
    assert np.allclose(m[:, 3], oio_ref, rtol=1e-9, atol=1e-12)
    assert not np.isfinite(m[4, 0])
    flags = fb.cpu().numpy().tolist()
    assert flags[:4] == [int(abs(v) > io_bound) for v in oio[:4]]
    assert flags[4] == 1
    # the relative form: the bound applies to |io| - |io of the small-ensemble modes|
    rel = np.abs(oio[:4]) - np.abs(oio_ref[:4])
    rb = float(np.median(rel))
    _sg.combine(sd, cd, xd, scale, dev(net, torch.bfloat16), imfs, res, part, chunks, S, N, K, C, P, 1e-3, rb,
                met, fb, io_relative=True)
    torch.cuda.synchronize()
    flags = fb.cpu().numpy().tolist()
    assert flags[:4] == [int(v > rb) for v in rel]
    assert flags[4] == 1


def _oracle_backprop(net, x, tgt, margin):
    """float64 forward and backward of the network on bf16-rounded weights and
    activations (the precision the kernels keep between layers)."""
    params = net.state().astype(np.float64)
    acts, ws = [bf16r(x)], []
    off = 0
    for lay in net.layers:
        nw = lay["cout_v"] * 3 * lay["cin_v"]
        w = params[off:off + nw].reshape(lay["cout_v"], 3, lay["cin_v"])
        b = params[off + nw:off + nw + lay["cout_v"]]
        off += nw + lay["cout_v"]
        if lay["project"]:
            w, b = SO.project_outputs(w, b)
        wq = np.zeros((lay["cout_p"], 3, lay["cin_p"]))
        wq[:lay["cout_v"], :, :lay["cin_v"]] = bf16r(w)
        bp = np.zeros(lay["cout_p"])
        bp[:lay["cout_v"]] = b
        ws.append(wq)
        z = SO.conv(acts[-1], wq, bp, lay["dil"])
        acts.append(bf16r(np.maximum(z, 0) if lay["relu"] else z))
    _, g = SO.mse_residual(acts[-1], None, bf16r(tgt), SU.P_CORR, margin)
    g = bf16r(g)
    grads = []
    for li in range(len(net.layers) - 1, -1, -1):
        lay = net.layers[li]
        dw, db = SO.conv_weight_grad(g, acts[li], lay["dil"])
        grads.append((li, dw[:lay["cout_v"], :, :lay["cin_v"]], db[:lay["cout_v"]]))
        if li > 0:
            g = bf16r(SO.conv_input_grad(g, ws[li], lay["dil"]) * (acts[li] > 0))
    return dict((li, (dw, db)) for li, dw, db in grads)


def test_network_gradient_matches_oracle_backprop():
    rng = np.random.default_rng(13)
    net = SU.Net(seed=3)
    # a trained-looking output layer (the initial one is nearly zero)
    st = net.state()
    st += (rng.standard_normal(st.shape) * 0.02).astype(np.float32)
    net.load_state(st)
    B, T, margin = 1, 900, 40
    x = np.zeros((B, T, SU.CH), np.float32)
    x[..., :SU.NCH] = rng.standard_normal((B, T, SU.NCH))
    tgt = np.zeros_like(x)
    tgt[..., :SU.NCH] = rng.standard_normal((B, T, SU.NCH)) * 0.1
    xd = dev(x, torch.bfloat16)
    acts = net.forward(xd, B, T)
    dout = torch.empty((B, T, SU.CH), dtype=torch.bfloat16, device="cuda")
    acc = torch.zeros((1,), dtype=torch.float32, device="cuda")
    _sg.loss(acts[-1], None, dev(tgt, torch.bfloat16), dout, acc, B, T, SU.CH, SU.P_CORR, margin)
    net.backward(acts, dout, B, T)
    torch.cuda.synchronize()
    net.check()
    ref = _oracle_backprop(net, x, tgt, margin)
    grads = net.grads.cpu().numpy().astype(np.float64)
    off = 0
    for li, lay in enumerate(net.layers):
        nw = lay["cout_v"] * 3 * lay["cin_v"]
        gw = grads[off:off + nw].reshape(lay["cout_v"], 3, lay["cin_v"])
        gb = grads[off + nw:off + nw + lay["cout_v"]]
        off += nw + lay["cout_v"]
        rw, rb = ref[li]
        # bf16 activations and gradients round at different points in the two
        # computations: compare whole-layer gradients
        assert np.linalg.norm(gw - rw) <= 0.03 * np.linalg.norm(rw), li
        assert np.linalg.norm(gb - rb) <= 0.03 * np.linalg.norm(rb) + 1e-12, li


def test_training_gains_over_the_small_ensemble_and_gates_fall_back():
    """A short training run: on the noise-dominated first modes the
    surrogate's IMFs must lie closer to the 256-trial mean than the 8-trial
    mean it starts from, the served decomposition must reconstruct the signal,
    and the gate must hand flagged signals to the plain EEMD."""
    N, E_small, E_big = 65536, 8, 256
    inp, tgt = SU.generate_pairs(range(10000, 10064), N, E_small, E_big)
    vinp, vtgt = SU.generate_pairs(range(20000, 20008), N, E_small, E_big)
    net, rep = SU.fit(inp, tgt, vinp, vtgt, candidates=2, steps=3000)
    del inp, tgt, vinp, vtgt
    for c in rep["candidates"]:
        hist = [h[1] for h in c["loss_history"]]
        assert min(hist[-3:]) < hist[0]
    ev = SU.evaluate(net, range(30000, 30008), N, E_small, E_big, group=8, plain_group=8)
    summ = SU.summarize(ev)
    e8, es = summ["median_err_8_per_imf"], summ["median_err_per_imf"]
    print(f"median rel. L2 error per IMF vs the {E_big}-trial mean: {E_small}-trial {e8}, surrogate {es}")
    # what the network gains: the first mode holds most of the averaged noise,
    # where the 8-trial mean is about 4x further from the 256-trial mean than
    # two independent 256-trial means are from each other
    assert es[0] < 0.6 * e8[0]
    assert np.mean([a / b for a, b in zip(es[:SU.P_CORR], e8[:SU.P_CORR])]) < 0.8
    assert summ["max_recon"] < 1e-12
    # gate: an orthogonality bound of 0 flags every signal; the served result
    # is then the plain EEMD
    N = 16384
    xs = SU.make_signals(range(30000, 30002), N)
    sur = SU.SurrogateEEMD(net, 2, N, E_small, E_big, io_bound=0.0, io_relative=False)
    served = sur.decompose(xs)
    plain = SU.plain_eemd(xs, N, E_big)
    for (m, r, st), (pm, pr) in zip(served, plain):
        assert st["fallback"]
        assert np.array_equal(m, pm) and np.array_equal(r, pr)
    sur = SU.SurrogateEEMD(net, 2, N, E_small, E_big, io_bound=1e30)
    for m, r, st in sur.decompose(xs):
        assert not st["fallback"]
        assert st["recon"] < 1e-12
