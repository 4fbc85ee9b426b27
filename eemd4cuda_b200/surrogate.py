"""Learned ensemble surrogate: small-ensemble mean IMFs -> large-ensemble mean.

For a signal x the plain EEMD engine gives the ensemble-mean IMFs of trials
[0, 8) (the network input) and of trials [0, 256) of the same Philox stream
(the target).  A dilated 1-D convolution network (8 layers, 64 channels,
kernel 3, dilations 1, 2, ..., 128; bfloat16 weights and activations,
float32 accumulation) reads 11 channels -- the 10 mean IMFs and the residual
x - sum(IMFs), divided by the signal's RMS -- and predicts corrections of
the first P_CORR = 6 modes:

    IMF_k ~ IMF8_k + RMS(x) * net_k          (k < 6; later modes unchanged)
    resid = resid8 - RMS(x) * sum_k net_k    (the IMFs and residual still sum to x)

The residual of an ensemble mean, x - sum(mean IMFs), carries minus the mean
of the added noise; the noise the first modes lose moves to the residual,
which is what the large ensemble's residual does as its noise averages out.
The last modes and the trend of single trials swing far beyond the signal
(end effects of the spline envelopes), so their ensemble means are not a
learnable target and are passed through.

All network arithmetic runs in libeemd_surrogate.so: the convolutions and
their input gradients as tcgen05 implicit GEMMs, the weight gradients, the
loss and Adam on CUDA cores, and the input (means, residual, scaling) and
output (served IMFs and residual, reconstruction error, orthogonality index)
stages.  PyTorch holds the device buffers and gathers training crops.

The plain large-ensemble EEMD remains the fallback: a signal whose served
decomposition has a relative reconstruction error above 1e-3, or whose
corrected modes are less orthogonal than the small-ensemble modes they
refine by more than a bound (orthogonality index, Huang et al. 1998, in
magnitude), is decomposed by it instead.  The bound is calibrated on
held-out pairs as the largest increase genuine 256-trial modes show over the
8-trial ones, and is at least 0.05: averaging more trials raises the index
(the index of the first modes is near 0.33 for 8 trials and 0.42 for 256 on
the harmonic test signals, whose partials are shared by neighbouring modes).
io_relative=False applies 0.05 to the index itself, which the plain
256-trial EEMD's own output exceeds on nearly every such signal.  The index
over all modes and the residual is reported too (not gated: the last modes
and the residual of this EEMD reach magnitudes of several units).

    python -m eemd4cuda_b200.surrogate --train-signals 20000 --eval-signals 1000 --steps 20000 \
        --save eemd4cuda_b200/weights/surrogate_n65536.npz
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import _lib as L
from . import _sg as SG
from . import emd_par as M
from . import signals
from .hostcopy import copy_into, prefault

CH = 16           # padded channels of the network's input and output
K_IMF = 10        # IMF channels
NCH = K_IMF + 1   # IMFs + residual: the network's input channels
P_CORR = 6        # modes the network corrects: its output channels
HIDDEN = 64
DILATIONS = (1, 2, 4, 8, 16, 32, 64, 128)
MARGIN = 255      # sum of the dilations: a crop's outputs nearer its edge see its zero padding
RECON_BOUND = 1e-3
IO_BOUND = 0.05
HUBER = 0.2       # loss threshold in RMS(x) units
CLIP = 1.0        # gradient norm bound of an Adam step
WARMUP = 500      # steps of linear learning-rate warm-up


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the surrogate needs a CUDA device")
    return torch


def make_signals(seeds, N):
    """Synthetic audio as the float32 ensemble workload: a harmonic tone, pink
    noise and decaying clicks (signals.harmonic_clicks), one seed per signal."""
    return [signals.harmonic_clicks(N, seed=int(s)).astype(np.float32) for s in seeds]


def engine_params(eps=0.2, seed=0, max_sifts=10, max_imf=K_IMF):
    """The ensemble settings of the training pairs: float32 data with the
    float64 spline solve, Philox noise of std eps * std(x), a fixed number of
    sifts per IMF (tau = 0)."""
    return M.make_params(dtype=np.float32, noise_mode=L.EEMD_NOISE_PHILOX, eps=eps, seed=seed, tau=0.0,
                         max_sifts=max_sifts, max_imf=max_imf)


class Ensembles:
    """Engine buffers for groups of up to S equal-length signals: per-mode
    ensemble sums of a trial range, and the plain EEMD's finalised result."""

    def __init__(self, S, N, max_trials, p=None):
        torch = _torch()
        self.torch = torch
        self.S, self.N = S, N
        # p_base: the caller's settings; p: the same with the launch shape of
        # the group's largest launch from the autotune table (the workspace is
        # sized for it, and every launch of the group uses it)
        self.p_base = p if p is not None else engine_params()
        self.p = M.tuned(self.p_base, [N] * S, max_trials)
        self.K = int(self.p.max_imf)
        self.ws = torch.empty((L.workspace_size(self.p, [N] * S, max_trials, False),), dtype=torch.uint8,
                              device="cuda")
        self.max_trials = max_trials

    def sums(self, xd, S, b0, count, imf_sum, mode_count, times=None):
        """imf_sum / mode_count += the sums of trials [b0, b0 + count) (with
        `times`, the first launch sequence fills per-kernel event timings)."""
        done = 0
        while done < count:
            c = min(self.max_trials, count - done)
            L.run(self.p, xd, [self.N] * S, b0 + done, c, self.ws, imf_sum=imf_sum, mode_count=mode_count,
                  times=times if done == 0 else None)
            done += c

    def plain(self, xd, S, E, imf_sum, mode_count, imf_mean, resid, n_modes):
        """The plain E-trial EEMD of the group: sums, then eemd_finalize."""
        imf_sum.zero_()
        mode_count.zero_()
        self.sums(xd, S, 0, E, imf_sum, mode_count)
        L.finalize(self.p, xd, [self.N] * S, imf_sum, mode_count, imf_mean, resid, n_modes)


# ---------------------------------------------------------------------------
# the network
# ---------------------------------------------------------------------------
class Net:
    """Weights (f32 master copy, bf16 packed operands) and the kernel calls of
    the forward and backward passes over a batch [B][T][CH]."""

    def __init__(self, seed=0):
        torch = _torch()
        self.torch = torch
        rng = np.random.default_rng(seed)
        self.layers = []
        sizes = []
        last = len(DILATIONS) - 1
        for i, d in enumerate(DILATIONS):
            lay = dict(cin_v=NCH if i == 0 else HIDDEN, cout_v=P_CORR if i == last else HIDDEN,
                       cin_p=CH if i == 0 else HIDDEN, cout_p=CH if i == last else HIDDEN, dil=d,
                       relu=i < last, project=False)
            self.layers.append(lay)
            sizes.append((lay["cout_v"] * 3 * lay["cin_v"], lay["cout_v"]))
        n = sum(a + b for a, b in sizes)
        self.n_params = n
        self.params = torch.zeros((n,), dtype=torch.float32, device="cuda")
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        host = np.zeros(n, dtype=np.float32)
        off = 0
        for lay, (nw, nb) in zip(self.layers, sizes):
            fan_in = 3 * lay["cin_v"]
            std = math.sqrt(2.0 / fan_in) if lay["relu"] else 0.1 / math.sqrt(fan_in)
            host[off:off + nw] = rng.standard_normal(nw) * std
            lay["w"], lay["dw"] = self.params[off:off + nw], self.grads[off:off + nw]
            off += nw
            lay["b"], lay["db"] = self.params[off:off + nb], self.grads[off:off + nb]
            off += nb
            lay["wp"] = torch.empty((lay["cout_p"] * 3 * lay["cin_p"],), dtype=torch.bfloat16, device="cuda")
            lay["wt"] = torch.empty((lay["cin_p"] * 3 * lay["cout_p"],), dtype=torch.bfloat16, device="cuda")
            lay["bias"] = torch.empty((lay["cout_p"],), dtype=torch.float32, device="cuda")
        self.params.copy_(torch.from_numpy(host))
        self.step_count = 0
        self.err = torch.zeros((1,), dtype=torch.int32, device="cuda")
        self.work = torch.zeros((1,), dtype=torch.float32, device="cuda")
        self.io_increase = None  # calibrated gate bound (load_model / fit)
        # eemd_sg_conv's tensor_cores: 4 warp-specialised with swizzled operands (the fastest:
        # the 8-layer pass over 16 x 65536 samples in 0.54 ms with it on the 64-channel
        # inputs, against 1.29 ms for 3, double-buffered with bulk-tensor loads, and 1.47 (2)
        # and 1.71 (1)); all four bit-identical
        self.conv_kernel = 4
        self.pack()

    def pack(self):
        """bf16 operands (forward and transposed) and the padded bias from the master weights."""
        for lay in self.layers:
            SG.pack(lay["w"], lay["wp"], lay["cout_p"], lay["cin_p"], lay["cout_v"], lay["cin_v"],
                    project=lay["project"])
            SG.pack(lay["w"], lay["wt"], lay["cin_p"], lay["cout_p"], lay["cin_v"], lay["cout_v"], transpose=True,
                    project=lay["project"])
            SG.bias(lay["b"], lay["bias"], lay["cout_p"], lay["cout_v"], project=lay["project"])

    def layer(self, i, src, dst, B, T, tensor_cores=True):
        lay = self.layers[i]
        mode = self.conv_kernel if tensor_cores else 0
        SG.conv(src, lay["wp"], lay["bias"], dst, B, T, lay["cin_p"], lay["cout_p"], lay["dil"], relu=lay["relu"],
                tensor_cores=mode, err=self.err)

    def forward(self, x, B, T, tensor_cores=True):
        """x: bf16 [B][T][CH] -> the activations (x, a1, ..., a8), kept for backward."""
        acts = [x]
        for i, lay in enumerate(self.layers):
            y = self.torch.empty((B, T, lay["cout_p"]), dtype=self.torch.bfloat16, device="cuda")
            self.layer(i, acts[-1], y, B, T, tensor_cores)
            acts.append(y)
        return acts

    def infer(self, x, out, S, T, chunk, bufs):
        """out[S][T][CH] = net(x[S][T][CH]) over chunks of `chunk` signals with
        two activation buffers bufs[0..1] of [chunk][T][HIDDEN] (nothing kept)."""
        last = len(self.layers) - 1
        for c0 in range(0, S, chunk):
            cs = min(chunk, S - c0)
            src = x[c0:c0 + cs]
            for i in range(len(self.layers)):
                dst = out[c0:c0 + cs] if i == last else bufs[i & 1][:cs]
                self.layer(i, src, dst, cs, T)
                src = dst

    def backward(self, acts, dout, B, T, tensor_cores=True):
        """Gradients of every layer from dL/d(output) (the loss kernel's dout)."""
        self.grads.zero_()
        g = dout
        for li in range(len(self.layers) - 1, -1, -1):
            lay = self.layers[li]
            SG.wgrad(g, acts[li], lay["dw"], lay["db"], B, T, lay["cout_p"], lay["cin_p"], lay["cout_v"],
                     lay["cin_v"], lay["dil"], tensor_cores=tensor_cores)
            if li > 0:
                gi = self.torch.empty((B, T, lay["cin_p"]), dtype=self.torch.bfloat16, device="cuda")
                # the input gradient times the ReLU derivative of the layer below (its output > 0)
                SG.conv(g, lay["wt"], None, gi, B, T, lay["cout_p"], lay["cin_p"], lay["dil"], direction=-1,
                        mask=acts[li], tensor_cores=self.conv_kernel if tensor_cores else 0, err=self.err)
                g = gi

    def adam_step(self, lr, max_norm=CLIP):
        self.step_count += 1
        SG.adam(self.params, self.grads, self.m, self.v, lr, self.step_count, max_norm=max_norm, work=self.work)
        self.pack()

    def check(self):
        e = int(self.err.item())
        if e != 0:
            raise SG.SurrogateError(e, "tensor-core convolution wait")

    def state(self) -> np.ndarray:
        return self.params.cpu().numpy()

    def load_state(self, params: np.ndarray):
        self.params.copy_(self.torch.from_numpy(np.asarray(params, np.float32)))
        self.pack()


# ---------------------------------------------------------------------------
# training pairs and training
# ---------------------------------------------------------------------------
def generate_pairs(seeds, N, E_small=8, E_big=256, group=16, p=None):
    """Device tensors inp, tgt [S][N][CH] bf16: the small-ensemble channels and
    the large-minus-small difference of every channel, both divided by RMS(x)
    (the loss reads the first P_CORR target channels)."""
    torch = _torch()
    seeds = list(seeds)
    S_all = len(seeds)
    inp = torch.empty((S_all, N, CH), dtype=torch.bfloat16, device="cuda")
    tgt = torch.empty_like(inp)
    ens = Ensembles(min(group, S_all), N, E_big - E_small, p)
    K = ens.K
    for g0 in range(0, S_all, group):
        xs = make_signals(seeds[g0:g0 + group], N)
        S = len(xs)
        xd = torch.from_numpy(np.concatenate(xs)).cuda()
        s_small = torch.zeros((S * K * N,), dtype=torch.float64, device="cuda")
        c_small = torch.zeros((S * K,), dtype=torch.int32, device="cuda")
        ens.sums(xd, S, 0, E_small, s_small, c_small)
        s_big, c_big = s_small.clone(), c_small.clone()
        ens.sums(xd, S, E_small, E_big - E_small, s_big, c_big)
        scale = torch.empty((S,), dtype=torch.float32, device="cuda")
        SG.scale(xd, scale, S, N)
        SG.prepare(s_small, c_small, xd, scale, inp[g0:g0 + S], S, N, K, CH)
        SG.prepare(s_big, c_big, xd, scale, tgt[g0:g0 + S], S, N, K, CH, imf_sum2=s_small, mode_count2=c_small)
    torch.cuda.synchronize()
    return inp, tgt


def channel_weights(tgt, sample=16):
    """Loss weight of each corrected mode: 1 / the mean square of its target
    channel over a sample of the training signals, normalised to mean 1, so
    that the faint first modes (mostly averaged noise) count as much as the
    energetic middle ones."""
    t = tgt[:sample, :, :P_CORR].float().cpu().numpy().astype(np.float64)
    ms = np.maximum(np.mean(t * t, axis=(0, 1)), 1e-12)
    w = 1.0 / ms
    return (w / w.mean()).astype(np.float32)


def train(net: Net, inp, tgt, steps=2000, batch=32, crop=4096, lr=1e-3, seed=1, log_every=100, delta=HUBER,
          weights=None):
    """Adam on random crops (gradient norm clipped to CLIP, linear warm-up
    over WARMUP steps, then cosine decay) with the Huber loss (threshold delta
    in RMS(x) units) and per-mode weights (default channel_weights(tgt));
    returns the loss history."""
    torch = net.torch
    rng = np.random.default_rng(seed)
    S, N = inp.shape[0], inp.shape[1]
    crop = min(crop, N)
    w = channel_weights(tgt) if weights is None else np.asarray(weights, np.float32)
    wd = torch.from_numpy(w).cuda()
    flat_in, flat_tg = inp.view(-1, CH), tgt.view(-1, CH)
    loss_acc = torch.zeros((1,), dtype=torch.float32, device="cuda")
    dout = torch.empty((batch, crop, CH), dtype=torch.bfloat16, device="cuda")
    ar = torch.arange(crop, device="cuda")
    history = []
    best, snap, since = float("inf"), None, 0
    loss_acc.zero_()
    t0 = time.time()
    for step in range(1, steps + 1):
        idx = rng.integers(0, S, size=batch)
        off = rng.integers(0, N - crop + 1, size=batch)
        rows = (torch.from_numpy(idx * N + off).cuda()[:, None] + ar[None, :]).reshape(-1)
        xb = flat_in.index_select(0, rows).view(batch, crop, CH)
        tb = flat_tg.index_select(0, rows).view(batch, crop, CH)
        acts = net.forward(xb, batch, crop)
        SG.loss(acts[-1], None, tb, dout, loss_acc, batch, crop, CH, P_CORR, MARGIN, delta=delta, weights=wd)
        net.backward(acts, dout, batch, crop)
        warm = min(1.0, step / WARMUP)
        net.adam_step(lr * warm * 0.5 * (1 + math.cos(math.pi * (step - 1) / steps)))
        since += 1
        if step % log_every == 0 or step == steps:
            mean = float(loss_acc.item()) / since  # the kernel adds every step's loss
            loss_acc.zero_()
            since = 0
            history.append((step, mean, math.sqrt(float(net.work.item()))))  # with the last gradient norm
            if mean < best:
                best, snap = mean, net.params.clone()
    torch.cuda.synchronize()
    net.check()
    restored = False
    if snap is not None and history[-1][1] > 1.5 * best:
        # the run diverged late: keep the parameters of the best window
        net.load_state(snap.cpu().numpy())
        restored = True
    return dict(history=history, seconds=time.time() - t0, weights=w.tolist(), restored=restored)


def validation_loss(net: Net, inp, tgt, weights, delta=HUBER, chunk=4):
    """The training loss over whole held-out signals (forward passes only)."""
    torch = net.torch
    S, N = inp.shape[0], inp.shape[1]
    acc = torch.zeros((1,), dtype=torch.float32, device="cuda")
    wd = torch.from_numpy(np.asarray(weights, np.float32)).cuda()
    total = 0.0
    for c0 in range(0, S, chunk):
        cs = min(chunk, S - c0)
        acts = net.forward(inp[c0:c0 + cs], cs, N)
        dout = torch.empty((cs, N, CH), dtype=torch.bfloat16, device="cuda")
        acc.zero_()
        SG.loss(acts[-1], None, tgt[c0:c0 + cs], dout, acc, cs, N, CH, P_CORR, MARGIN, delta=delta, weights=wd)
        total += float(acc.item()) * cs
        del acts, dout
    net.check()
    return total / S


def calibrate_gate(vinp, vtgt, quantile=1.0):
    """The orthogonality-index increase that genuine large ensembles show:
    over held-out pairs, |IO| of the first P_CORR large-ensemble modes less
    |IO| of the same small-ensemble modes (IO is scale free, so the scaled
    channels serve); returns max(IO_BOUND, that quantile of it)."""
    a = vinp[..., :NCH].double().cpu().numpy()
    b = a + vtgt[..., :NCH].double().cpu().numpy()
    inc = []
    for s in range(a.shape[0]):
        x = a[s].sum(axis=1)
        inc.append(abs(orthogonality_index(b[s][:, :P_CORR].T, x)) - abs(orthogonality_index(a[s][:, :P_CORR].T, x)))
    return max(IO_BOUND, float(np.quantile(inc, quantile))), [round(float(v), 4) for v in inc]


def save_model(path, net, io_increase):
    np.savez(path, params=net.state(), io_increase=np.float64(io_increase), p_corr=P_CORR, k_imf=K_IMF,
             dilations=np.array(DILATIONS), hidden=HIDDEN)


def load_model(path, net):
    """Parameters into net; returns the calibrated orthogonality gate bound (None for a bare .npy)."""
    d = np.load(path)
    if isinstance(d, np.ndarray):
        net.load_state(d)
        return None
    if int(d["p_corr"]) != P_CORR or int(d["k_imf"]) != K_IMF or tuple(d["dilations"]) != DILATIONS:
        raise ValueError(f"{path}: network shape differs from this build")
    net.load_state(d["params"])
    return float(d["io_increase"])


def fit(inp, tgt, vinp, vtgt, candidates=3, steps=2000, batch=32, crop=4096, lr=1e-3, delta=HUBER):
    """Trains `candidates` networks from different initialisations and crop
    orders and keeps the one with the lowest validation loss (some runs stay
    on a plateau where the first modes' averaged noise is not yet removed)."""
    w = channel_weights(tgt)
    best, report = None, []
    for c in range(candidates):
        net = Net(seed=c)
        tr = train(net, inp, tgt, steps=steps, batch=batch, crop=crop, lr=lr, seed=1 + c, delta=delta, weights=w)
        vl = validation_loss(net, vinp, vtgt, w, delta)
        report.append(dict(candidate=c, validation_loss=vl, seconds=round(tr["seconds"], 1),
                           restored_best=tr["restored"], loss_history=[(h[0], h[1]) for h in tr["history"][::10]]))
        if best is None or vl < best[1]:
            best = (net, vl, c)
        else:
            del net
    io_increase, inc = calibrate_gate(vinp, vtgt)
    return best[0], dict(chosen=best[2], candidates=report, channel_weights=[round(float(v), 3) for v in w],
                         io_increase=io_increase, io_increase_validation=inc)


# ---------------------------------------------------------------------------
# the served path
# ---------------------------------------------------------------------------
class SurrogateEEMD:
    """EEMD of groups of up to S equal-length signals through the surrogate:
    the E_small-trial ensemble, the network, the served IMFs and residual and
    the gate.  decompose() runs the fallback (the plain E_big-trial EEMD of
    the flagged signals)."""

    def __init__(self, net: Net, S, N, E_small=8, E_big=256, p=None, chunk=16, recon_bound=RECON_BOUND,
                 io_bound=None, io_relative=True, chunks_per_signal=32):
        torch = _torch()
        self.torch, self.net = torch, net
        self.S, self.N, self.E_small, self.E_big = S, N, E_small, E_big
        self.ens = Ensembles(S, N, E_small, p)
        K = self.K = self.ens.K
        if K != K_IMF:
            raise ValueError(f"the network reads {K_IMF} IMF channels")
        if io_bound is None:
            io_bound = (net.io_increase if io_relative and net.io_increase is not None else IO_BOUND)
        self.recon_bound, self.io_bound, self.io_relative = recon_bound, io_bound, io_relative
        self.chunk = min(chunk, S)
        self.cps = chunks_per_signal
        f = dict(device="cuda")
        self.xd = torch.empty((S * N,), dtype=torch.float32, **f)
        self.imf_sum = torch.empty((S * K * N,), dtype=torch.float64, **f)
        self.mode_count = torch.empty((S * K,), dtype=torch.int32, **f)
        self.scale = torch.empty((S,), dtype=torch.float32, **f)
        self.inp = torch.empty((S, N, CH), dtype=torch.bfloat16, **f)
        self.out = torch.empty_like(self.inp)
        self.bufs = [torch.empty((self.chunk, N, HIDDEN), dtype=torch.bfloat16, **f) for _ in range(2)]
        self.imfs = torch.empty((S, K, N), dtype=torch.float64, **f)
        self.resid = torch.empty((S, N), dtype=torch.float64, **f)
        self.partial = torch.empty((S * self.cps * SG.stat_count(),), dtype=torch.float64, **f)
        self.metrics = torch.empty((S, 4), dtype=torch.float64, **f)
        self.fallback = torch.empty((S,), dtype=torch.int32, **f)

    def run(self, S):
        """The surrogate decomposition of the first S signals in self.xd (device, asynchronous)."""
        N, K = self.N, self.K
        self.imf_sum.zero_()
        self.mode_count.zero_()
        self.ens.sums(self.xd, S, 0, self.E_small, self.imf_sum, self.mode_count)
        SG.scale(self.xd, self.scale, S, N)
        SG.prepare(self.imf_sum, self.mode_count, self.xd, self.scale, self.inp, S, N, K, CH)
        self.net.infer(self.inp, self.out, S, N, self.chunk, self.bufs)
        SG.combine(self.imf_sum, self.mode_count, self.xd, self.scale, self.out, self.imfs, self.resid,
                   self.partial, self.cps, S, N, K, CH, P_CORR, self.recon_bound, self.io_bound, self.metrics,
                   self.fallback, io_relative=self.io_relative)

    def _host_buffers(self):
        """Pinned host staging for decompose (allocated at its first call):
        the signals in, the served modes, residuals and gate results out."""
        if getattr(self, "_hbuf", None) is None:
            torch = self.torch
            pin = dict(pin_memory=True)
            self._hbuf = dict(x=torch.empty((self.S * self.N,), dtype=torch.float32, **pin),
                              imfs=torch.empty((self.S, self.K, self.N), dtype=torch.float64, **pin),
                              resid=torch.empty((self.S, self.N), dtype=torch.float64, **pin),
                              met=torch.empty((self.S, 4), dtype=torch.float64, **pin),
                              fb=torch.empty((self.S,), dtype=torch.int32, **pin))
        return self._hbuf

    def launches_per_run(self, S) -> int:
        """Kernels of libeemd_surrogate.so per run (the engine's are counted by the engine)."""
        return 2 + len(DILATIONS) * ((S + self.chunk - 1) // self.chunk) + 2

    def decompose(self, xs):
        """Served decompositions of host signals xs (equal length N, at most S):
        list of (imfs [K][N], residual [N], stats); flagged signals are replaced
        by the plain E_big-trial EEMD."""
        torch = self.torch
        S = len(xs)
        if S > self.S or any(len(x) != self.N for x in xs):
            raise ValueError(f"at most {self.S} signals of {self.N} samples")
        hb = self._host_buffers()
        n = S * self.N
        hb["x"][:n].numpy()[:] = np.concatenate([np.asarray(x, np.float32) for x in xs])
        self.xd[:n].copy_(hb["x"][:n], non_blocking=True)
        # the fresh result arrays are paged in on the copy threads while the device computes
        imfs = np.empty((S, self.K, self.N), dtype=np.float64)
        resid = np.empty((S, self.N), dtype=np.float64)
        paged = prefault([imfs, resid])
        self.run(S)
        for name, d in (("met", self.metrics), ("fb", self.fallback)):
            hb[name][:S].copy_(d[:S], non_blocking=True)
        # the served modes and residuals cross to the host in groups of signals, and the
        # host copies each group out of the pinned buffers (reused by the next call) into
        # fresh arrays while the later groups are still on their way
        G = max(1, -(-S // 8))
        marks = []
        for g0 in range(0, S, G):
            g1 = min(S, g0 + G)
            hb["imfs"][g0:g1].copy_(self.imfs[g0:g1], non_blocking=True)
            hb["resid"][g0:g1].copy_(self.resid[g0:g1], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            marks.append((g0, g1, ev))
        for f in paged:
            f.result()
        hi, hr = hb["imfs"].numpy(), hb["resid"].numpy()
        for g0, g1, ev in marks:
            ev.synchronize()
            copy_into(imfs[g0:g1], hi[g0:g1])
            copy_into(resid[g0:g1], hr[g0:g1])
        torch.cuda.current_stream().synchronize()
        self.net.check()
        met = hb["met"][:S].numpy().copy()
        fb = hb["fb"][:S].numpy().astype(bool)
        flagged = [i for i in range(S) if fb[i]]
        plain = {}
        if flagged:
            plain = dict(zip(flagged, plain_eemd([xs[i] for i in flagged], self.N, self.E_big, self.ens.p_base)))
        out = []
        for i in range(S):
            st = dict(method="surrogate", recon=float(met[i, 0]), io=float(met[i, 1]), io_all=float(met[i, 2]),
                      io_small=float(met[i, 3]), fallback=bool(fb[i]), E_small=self.E_small, E_big=self.E_big)
            out.append((*plain[i], st) if fb[i] else (imfs[i], resid[i], st))
        return out


def plain_eemd(xs, N, E, p=None, group=16):
    """The plain E-trial EEMD of host signals: list of (means [K][N], residual [N])."""
    torch = _torch()
    S_all = len(xs)
    g = min(group, S_all)
    ens = Ensembles(g, N, E, p)
    K = ens.K
    f = dict(device="cuda")
    s = torch.empty((g * K * N,), dtype=torch.float64, **f)
    c = torch.empty((g * K,), dtype=torch.int32, **f)
    mean = torch.empty((g * K * N,), dtype=torch.float64, **f)
    res = torch.empty((g * N,), dtype=torch.float64, **f)
    nm = torch.empty((g,), dtype=torch.int32, **f)
    out = []
    for g0 in range(0, S_all, g):
        part = xs[g0:g0 + g]
        S = len(part)
        xd = torch.from_numpy(np.concatenate([np.asarray(x, np.float32) for x in part])).cuda()
        ens.plain(xd, S, E, s[:S * K * N], c[:S * K], mean[:S * K * N], res[:S * N], nm[:S])
        mh = mean[:S * K * N].cpu().numpy().reshape(S, K, N)
        rh = res[:S * N].cpu().numpy().reshape(S, N)
        out.extend((mh[i], rh[i]) for i in range(S))
    return out


# ---------------------------------------------------------------------------
# evaluation
# ---------------------------------------------------------------------------
def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(b)), 1e-300))


def orthogonality_index(components, x):
    """Huang et al. (1998): sum over pairs j != k of <c_j, c_k> / ||x||^2."""
    g = components @ components.T
    return float((g.sum() - np.trace(g)) / max(float(x @ x), 1e-300))


def evaluate(net: Net, seeds, N, E_small=8, E_big=256, group=128, plain_group=16, p=None, floor_signals=0):
    """Held-out signals: per signal the relative L2 error (over the 10 IMFs)
    of the small-ensemble mean and of the surrogate against the plain
    large-ensemble mean, the gate metrics and fallbacks, and the device time
    (CUDA events) of the surrogate path and of the plain EEMD."""
    torch = net.torch
    seeds = list(seeds)
    sur = SurrogateEEMD(net, min(group, len(seeds)), N, E_small, E_big, p)
    io_bound = sur.io_bound
    ens_plain = Ensembles(min(plain_group, len(seeds)), N, E_big, p)
    K = sur.K
    g = ens_plain.S
    f = dict(device="cuda")
    ps = torch.empty((g * K * N,), dtype=torch.float64, **f)
    pc = torch.empty((g * K,), dtype=torch.int32, **f)
    pm = torch.empty((g * K * N,), dtype=torch.float64, **f)
    pr = torch.empty((g * N,), dtype=torch.float64, **f)
    pn = torch.empty((g,), dtype=torch.int32, **f)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rows = []
    t_sur = t_plain = 0.0
    # warm-up of both paths (first-launch costs are not part of the steady state)
    xw = torch.from_numpy(np.concatenate(make_signals(seeds[:1], N))).cuda()
    sur.xd[:N].copy_(xw)
    sur.run(1)
    ens_plain.plain(xw, 1, E_small, ps[:K * N], pc[:K], pm[:K * N], pr[:N], pn[:1])
    torch.cuda.synchronize()
    for g0 in range(0, len(seeds), sur.S):
        xs = make_signals(seeds[g0:g0 + sur.S], N)
        S = len(xs)
        sur.xd[:S * N].copy_(torch.from_numpy(np.concatenate(xs)))
        a, b = ev(), ev()
        a.record()
        sur.run(S)
        b.record()
        b.synchronize()
        t_sur += a.elapsed_time(b)
        net.check()
        imfs = sur.imfs[:S].cpu().numpy()
        met = sur.metrics[:S].cpu().numpy()
        fb = sur.fallback[:S].cpu().numpy().astype(bool)
        cnt = sur.mode_count[:S * K].cpu().numpy().reshape(S, K)
        m8 = sur.imf_sum[:S * K * N].cpu().numpy().reshape(S, K, N) / np.maximum(cnt, 1)[:, :, None]
        for q0 in range(0, S, g):
            qs = min(g, S - q0)
            xd = torch.from_numpy(np.concatenate(xs[q0:q0 + qs])).cuda()
            a, b = ev(), ev()
            a.record()
            ens_plain.plain(xd, qs, E_big, ps[:qs * K * N], pc[:qs * K], pm[:qs * K * N], pr[:qs * N], pn[:qs])
            b.record()
            b.synchronize()
            t_plain += a.elapsed_time(b)
            big = pm[:qs * K * N].cpu().numpy().reshape(qs, K, N)
            for j in range(qs):
                i = q0 + j
                e8 = rel_l2(m8[i], big[j])
                es = rel_l2(imfs[i], big[j])
                per_imf = [rel_l2(imfs[i][k], big[j][k]) for k in range(K)]
                per_imf_8 = [rel_l2(m8[i][k], big[j][k]) for k in range(K)]
                x = np.asarray(xs[i], np.float64)
                io_plain = orthogonality_index(big[j][:P_CORR], x)
                io_plain_all = orthogonality_index(np.vstack([big[j], x - big[j].sum(axis=0)]), x)
                rows.append(dict(seed=seeds[g0 + i], err_8=e8, err_surrogate=es, recon=float(met[i, 0]),
                                 io=float(met[i, 1]), io_all=float(met[i, 2]), io_small=float(met[i, 3]),
                                 io_plain=io_plain,
                                 io_plain_all=io_plain_all, fallback=bool(fb[i]),
                                 err_served=0.0 if fb[i] else es, err_per_imf=per_imf, err_8_per_imf=per_imf_8))
    floor = None
    if floor_signals:
        # two disjoint large ensembles of the same signals: how far apart two
        # plain E_big-trial results lie (the target's own trial noise)
        xs = make_signals(seeds[:floor_signals], N)
        pa = plain_eemd(xs, N, E_big, engine_params(seed=0))
        pb = plain_eemd(xs, N, E_big, engine_params(seed=1))
        floor = dict(stack=float(np.median([rel_l2(u[0], v[0]) for u, v in zip(pa, pb)])),
                     per_imf=[round(float(np.median([rel_l2(u[0][k], v[0][k]) for u, v in zip(pa, pb)])), 4)
                              for k in range(K)])
    return dict(rows=rows, surrogate_ms=t_sur, plain_ms=t_plain, ensemble_distance=floor, io_bound=io_bound)


def summarize(ev):
    rows = ev["rows"]
    med = lambda k: float(np.median([r[k] for r in rows]))  # noqa: E731
    n = len(rows)
    nf = sum(r["fallback"] for r in rows)
    # the served path pays the plain EEMD for every flagged signal
    served_ms = ev["surrogate_ms"] + ev["plain_ms"] * nf / max(n, 1)
    return dict(signals=n, io_gate_bound=ev.get("io_bound"),
                median_err_8=med("err_8"), median_err_surrogate=med("err_surrogate"),
                median_err_served=med("err_served"), gain=med("err_8") / max(med("err_surrogate"), 1e-300),
                median_err_per_imf=[round(float(np.median([r["err_per_imf"][k] for r in rows])), 4)
                                    for k in range(K_IMF)],
                median_err_8_per_imf=[round(float(np.median([r["err_8_per_imf"][k] for r in rows])), 4)
                                      for k in range(K_IMF)],
                fallbacks=nf, median_recon=med("recon"), max_recon=float(max(r["recon"] for r in rows)),
                median_abs_io=float(np.median([abs(r["io"]) for r in rows])),
                median_abs_io_plain=float(np.median([abs(r["io_plain"]) for r in rows])),
                plain_io_above_bound=sum(abs(r["io_plain"]) > IO_BOUND for r in rows),
                fallbacks_absolute_io=sum(abs(r["io"]) > IO_BOUND for r in rows),
                median_abs_io_small=float(np.median([abs(r["io_small"]) for r in rows])),
                median_abs_io_all=float(np.median([abs(r["io_all"]) for r in rows])),
                median_abs_io_all_plain=float(np.median([abs(r["io_plain_all"]) for r in rows])),
                surrogate_ms=round(ev["surrogate_ms"], 2), plain_ms=round(ev["plain_ms"], 2),
                served_ms=round(served_ms, 2), speedup=round(ev["plain_ms"] / ev["surrogate_ms"], 2),
                served_speedup=round(ev["plain_ms"] / served_ms, 2),
                ensemble_distance=ev["ensemble_distance"])


def network_flops_per_sample() -> int:
    """Algorithmic FLOPs of one forward pass per sample (valid channels, 2 per MAC)."""
    dims = [(NCH, HIDDEN)] + [(HIDDEN, HIDDEN)] * (len(DILATIONS) - 2) + [(HIDDEN, P_CORR)]
    return sum(2 * 3 * a * b for a, b in dims)


def time_network(net: Net, S, N, load="", reps=3, chunk=16):
    """Device time of the forward pass over S signals (random channels)."""
    torch = net.torch
    if load:
        net.load_state(np.load(load))
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((S, N, CH), generator=g, device="cuda").to(torch.bfloat16)
    x[..., NCH:] = 0
    out = torch.empty_like(x)
    c = min(chunk, S)
    bufs = [torch.empty((c, N, HIDDEN), dtype=torch.bfloat16, device="cuda") for _ in range(2)]
    net.infer(x, out, S, N, c, bufs)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        net.infer(x, out, S, N, c, bufs)
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    net.check()
    ms = min(ts)
    res = dict(signals=S, N=N, ms=round(ms, 4), launches=len(DILATIONS) * ((S + c - 1) // c),
               tflops=round(network_flops_per_sample() * S * N / (ms / 1e3) / 1e12, 2))
    print(json.dumps(res), flush=True)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--N", type=int, default=65536)
    ap.add_argument("--train-signals", type=int, default=2048)
    ap.add_argument("--eval-signals", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--crop", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--E-small", type=int, default=8)
    ap.add_argument("--E-big", type=int, default=256)
    ap.add_argument("--floor-signals", type=int, default=8)
    ap.add_argument("--delta", type=float, default=HUBER)
    ap.add_argument("--candidates", type=int, default=3)
    ap.add_argument("--val-signals", type=int, default=32)
    ap.add_argument("--save", default="", help="write the trained model (.npz: parameters and gate bound)")
    ap.add_argument("--load", default="", help="skip training: read a model (.npz, or bare parameters .npy)")
    ap.add_argument("--calibrate", action="store_true",
                    help="with --load: calibrate the orthogonality gate on validation pairs (and --save)")
    ap.add_argument("--time-network", type=int, default=0, metavar="S",
                    help="only time the network's forward pass over S signals of N samples")
    ap.add_argument("--conv-kernel", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="tensor-core convolution: 1 single-buffered, 2 double-buffered, 3 double-buffered "
                         "with bulk-tensor loads, 4 warp-specialised with swizzled operands (0: the default)")
    args = ap.parse_args(argv)
    t0 = time.time()
    if args.time_network:
        net = Net(seed=0)
        if args.conv_kernel:
            net.conv_kernel = args.conv_kernel
        return time_network(net, args.time_network, args.N, args.load)
    out = dict(N=args.N, E_small=args.E_small, E_big=args.E_big)
    if args.load:
        net = Net(seed=0)
        net.io_increase = load_model(args.load, net)
        if args.calibrate:
            vinp, vtgt = generate_pairs(range(20000, 20000 + args.val_signals), args.N, args.E_small, args.E_big)
            net.io_increase, inc = calibrate_gate(vinp, vtgt)
            del vinp, vtgt
            out.update(io_increase=net.io_increase, io_increase_validation=inc)
            if args.save:
                save_model(args.save, net, net.io_increase)
    else:
        inp, tgt = generate_pairs(range(10000, 10000 + args.train_signals), args.N, args.E_small, args.E_big)
        vinp, vtgt = generate_pairs(range(20000, 20000 + args.val_signals), args.N, args.E_small, args.E_big)
        out["data_seconds"] = round(time.time() - t0, 1)
        t1 = time.time()
        net, rep = fit(inp, tgt, vinp, vtgt, candidates=args.candidates, steps=args.steps, batch=args.batch,
                       crop=args.crop, lr=args.lr, delta=args.delta)
        del inp, tgt, vinp, vtgt
        out.update(train_signals=args.train_signals, val_signals=args.val_signals, steps=args.steps,
                   batch=args.batch, crop=args.crop, lr=args.lr, train_seconds=round(time.time() - t1, 1), fit=rep)
        net.io_increase = rep["io_increase"]
        if args.save:
            save_model(args.save, net, net.io_increase)
    out["params"] = net.n_params
    ev = evaluate(net, range(30000, 30000 + args.eval_signals), args.N, args.E_small, args.E_big,
                  floor_signals=args.floor_signals)
    out.update(summarize(ev))
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
