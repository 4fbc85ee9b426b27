"""The surrogate's GPU kernels against the CPU restatement (oracle/surrogate_oracle.py)
and the tensor-core convolution against the CUDA-core reference kernel."""
import numpy as np
import pytest

from oracle import surrogate_oracle as SO

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from eemd4cuda_b200 import _sg  # noqa: E402


def bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16)


def f64(t):
    return t.float().cpu().numpy().astype(np.float64)


def packed(w, n_rows, c, transpose=False):
    """w: f32 [nv][3][cv] -> packed bf16 device operand."""
    wd = torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).cuda()
    out = torch.empty((n_rows * 3 * c,), dtype=torch.bfloat16, device="cuda")
    nv, cv = (w.shape[2], w.shape[0]) if transpose else (w.shape[0], w.shape[2])
    _sg.pack(wd, out, n_rows, c, nv, cv, transpose=transpose)
    return out


@pytest.mark.parametrize("cin,cout", [(16, 64), (64, 64), (64, 16)])
@pytest.mark.parametrize("dil", [1, 7, 128])
def test_tensor_core_conv_matches_reference_and_oracle(cin, cout, dil):
    rng = np.random.default_rng(cin * 1000 + cout + dil)
    B, T = 2, 1000
    x = rng.standard_normal((B, T, cin)).astype(np.float32)
    w = (rng.standard_normal((cout, 3, cin)) / np.sqrt(3 * cin)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    xd = bf16(x).cuda()
    wp = packed(w, cout, cin)
    bd = torch.from_numpy(b).cuda()
    err = torch.zeros((1,), dtype=torch.int32, device="cuda")
    for relu in (False, True):
        y_tc = torch.empty((B, T, cout), dtype=torch.bfloat16, device="cuda")
        y_ref = torch.empty_like(y_tc)
        _sg.conv(xd, wp, bd, y_tc, B, T, cin, cout, dil, relu=relu, tensor_cores=True, err=err)
        _sg.conv(xd, wp, bd, y_ref, B, T, cin, cout, dil, relu=relu, tensor_cores=False)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        a, r = f64(y_tc), f64(y_ref)
        # both round an f32 sum to bf16: at most one bf16 step apart
        assert np.max(np.abs(a - r) / (np.abs(r) + 1e-2)) < 2 ** -6
        xq = f64(bf16(x))
        wq = f64(bf16(w))
        o = SO.conv(xq, wq, b, dil)
        if relu:
            o = np.maximum(o, 0)
        assert np.max(np.abs(a - o)) <= 2 ** -7 * np.max(np.abs(o)) + 1e-3


@pytest.mark.parametrize("cin,cout", [(16, 64), (64, 64), (64, 16)])
def test_input_gradient_conv_with_mask(cin, cout):
    rng = np.random.default_rng(7 + cin + cout)
    B, T, dil = 2, 700, 16
    dy = rng.standard_normal((B, T, cout)).astype(np.float32)
    w = (rng.standard_normal((cout, 3, cin)) / np.sqrt(3 * cin)).astype(np.float32)
    mask = (rng.random((B, T, cin)) > 0.5).astype(np.float32)
    dyd, md = bf16(dy).cuda(), bf16(mask).cuda()
    wpt = packed(w, cin, cout, transpose=True)  # N = cin rows, K = 3*cout
    dx = torch.empty((B, T, cin), dtype=torch.bfloat16, device="cuda")
    _sg.conv(dyd, wpt, None, dx, B, T, cout, cin, dil, direction=-1, mask=md, tensor_cores=True)
    torch.cuda.synchronize()
    o = SO.conv_input_grad(f64(bf16(dy)), f64(bf16(w)), dil) * mask
    assert np.max(np.abs(f64(dx) - o)) <= 2 ** -7 * np.max(np.abs(o)) + 1e-3


@pytest.mark.parametrize("N,C,nv,cv", [(64, 16, 64, 16), (64, 64, 64, 64), (16, 64, 10, 64), (64, 16, 64, 11)])
@pytest.mark.parametrize("tensor_cores", [True, False])
def test_weight_gradient(N, C, nv, cv, tensor_cores):
    """Weight and bias gradients (tcgen05 implicit GEMM over time, and the
    CUDA-core kernel) against the float64 oracle on the same bf16 operands."""
    rng = np.random.default_rng(3)
    B, T, dil = 2, 500, 8
    dy = rng.standard_normal((B, T, N)).astype(np.float32)
    x = rng.standard_normal((B, T, C)).astype(np.float32)
    dw = torch.zeros((nv, 3, cv), dtype=torch.float32, device="cuda")
    db = torch.zeros((nv,), dtype=torch.float32, device="cuda")
    err = torch.zeros((1,), dtype=torch.int32, device="cuda")
    _sg.wgrad(bf16(dy).cuda(), bf16(x).cuda(), dw, db, B, T, N, C, nv, cv, dil, tensor_cores=tensor_cores, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ow, ob = SO.conv_weight_grad(f64(bf16(dy)), f64(bf16(x)), dil)
    assert np.allclose(dw.cpu().numpy(), ow[:nv, :, :cv], rtol=1e-4, atol=1e-3)
    assert np.allclose(db.cpu().numpy(), ob[:nv], rtol=1e-4, atol=1e-3)


def test_loss_and_adam():
    rng = np.random.default_rng(5)
    B, T, C, cv, margin = 2, 300, 16, 10, 20
    out, base, tgt = (rng.standard_normal((B, T, C)).astype(np.float32) for _ in range(3))
    dout = torch.empty((B, T, C), dtype=torch.bfloat16, device="cuda")
    acc = torch.zeros((1,), dtype=torch.float32, device="cuda")
    _sg.loss(bf16(out).cuda(), bf16(base).cuda(), bf16(tgt).cuda(), dout, acc, B, T, C, cv, margin)
    torch.cuda.synchronize()
    l, g = SO.mse_residual(f64(bf16(out)), f64(bf16(base)), f64(bf16(tgt)), cv, margin)
    assert abs(float(acc.item()) - l) <= 1e-4 * l
    assert np.max(np.abs(f64(dout) - g)) <= 2 ** -7 * np.max(np.abs(g))
    p, gr = rng.standard_normal(1000).astype(np.float32), rng.standard_normal(1000).astype(np.float32)
    m, v = np.zeros(1000, np.float32), np.zeros(1000, np.float32)
    pd, gd, md, vd = (torch.from_numpy(a.copy()).cuda() for a in (p, gr, m, v))
    _sg.adam(pd, gd, md, vd, 1e-3, 1)
    torch.cuda.synchronize()
    op, om, ov = SO.adam(p.astype(np.float64), gr, m, v, 1e-3, 1)
    assert np.allclose(pd.cpu().numpy(), op, rtol=1e-5, atol=1e-6)
    # with the gradient clipped to norm 2 (its norm is about 31), twice
    pd, gd, md, vd = (torch.from_numpy(a.copy()).cuda() for a in (p, gr, m, v))
    work = torch.zeros((1,), dtype=torch.float32, device="cuda")
    op, om, ov = p.astype(np.float64), m.astype(np.float64), v.astype(np.float64)
    for step in (1, 2):
        _sg.adam(pd, gd, md, vd, 1e-2, step, max_norm=2.0, work=work)
        op, om, ov = SO.adam(op, gr.astype(np.float64), om, ov, 1e-2, step, max_norm=2.0)
    torch.cuda.synchronize()
    assert np.allclose(pd.cpu().numpy(), op, rtol=1e-5, atol=1e-6)
    assert np.allclose(md.cpu().numpy(), om, rtol=1e-5, atol=1e-7)
    # a non-finite gradient leaves everything unchanged
    before = pd.clone()
    gd[3] = float("nan")
    _sg.adam(pd, gd, md, vd, 1e-2, 3, max_norm=2.0, work=work)
    torch.cuda.synchronize()
    assert torch.equal(pd, before)


@pytest.mark.parametrize("cin,cout", [(16, 64), (64, 64), (64, 16)])
@pytest.mark.parametrize("dil", [1, 13, 128])
def test_double_buffered_kernels_equal_single_buffered(cin, cout, dil):
    """tensor_cores=2 (two input buffers and accumulators, epilogue of tile
    k-1 overlapping MMA k), 3 (the same fed by bulk-tensor copies) and 4
    (warp-specialised, swizzled operands, bulk-tensor stores) against
    tensor_cores=1, forward and
    masked input gradient, with more tiles than CTAs, a ragged last tile and
    halo rows outside the signal."""
    rng = np.random.default_rng(100 + cin + cout + dil)
    B, T = 8, 10000
    x = rng.standard_normal((B, T, cin)).astype(np.float32)
    w = (rng.standard_normal((cout, 3, cin)) / np.sqrt(3 * cin)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    xd, bd = bf16(x).cuda(), torch.from_numpy(b).cuda()
    wp = packed(w, cout, cin)
    err = torch.zeros((1,), dtype=torch.int32, device="cuda")
    ys = []
    for mode in (1, 2, 3, 4):
        y = torch.full((B, T, cout), 7.0, dtype=torch.bfloat16, device="cuda")
        _sg.conv(xd, wp, bd, y, B, T, cin, cout, dil, relu=True, tensor_cores=mode, err=err)
        ys.append(y)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert all(torch.equal(ys[0], y) for y in ys[1:])
    # masked input gradient
    dy = rng.standard_normal((B, T, cout)).astype(np.float32)
    mask = (rng.random((B, T, cin)) > 0.3).astype(np.float32)
    wpt = packed(w, cin, cout, transpose=True)
    gs = []
    for mode in (1, 2, 3, 4):
        g = torch.full((B, T, cin), 7.0, dtype=torch.bfloat16, device="cuda")
        _sg.conv(bf16(dy).cuda(), wpt, None, g, B, T, cout, cin, dil, direction=-1, mask=bf16(mask).cuda(),
                 tensor_cores=mode, err=err)
        gs.append(g)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert all(torch.equal(gs[0], g) for g in gs[1:])


@pytest.mark.parametrize("cin,cout", [(64, 64), (64, 16), (16, 64)])
@pytest.mark.parametrize("dil", [1, 64])
def test_warp_specialised_conv_over_many_tiles(cin, cout, dil):
    """tensor_cores=4 over 16 x 65536 samples (55 or 56 tiles per CTA: every
    input stage and accumulator reused many times) equals tensor_cores=3."""
    rng = np.random.default_rng(500 + cin + cout + dil)
    B, T = 16, 65536
    xd = (torch.randn((B, T, cin), generator=torch.Generator().manual_seed(cin + cout + dil)) * 0.5).to(
        torch.bfloat16).cuda()
    w = (rng.standard_normal((cout, 3, cin)) / np.sqrt(3 * cin)).astype(np.float32)
    bd = torch.from_numpy(rng.standard_normal(cout).astype(np.float32)).cuda()
    wp = packed(w, cout, cin)
    err = torch.zeros((1,), dtype=torch.int32, device="cuda")
    ys = []
    for mode in (3, 4):
        y = torch.full((B, T, cout), 7.0, dtype=torch.bfloat16, device="cuda")
        _sg.conv(xd, wp, bd, y, B, T, cin, cout, dil, relu=True, tensor_cores=mode, err=err)
        ys.append(y)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(ys[0], ys[1])
