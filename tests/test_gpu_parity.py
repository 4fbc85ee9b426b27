"""Parity of the sm_100a engine with the CPU oracle and the reference's golden
vectors (test_emd_gpu.py A1-A5, test_phase3_gates.py G1-G5/G8 analogues).

Tolerances (float64):
  exact=True  (reference operation order): per-IMF max|d| <= 1e-12 * max|x|;
              integers (modes, sifts, per-sift knot counts) identical
  exact=False (fused-multiply-add, reciprocals): per-IMF <= 1e-9 relative
"""
import numpy as np
import pytest

from conftest import checksum_close
from eemd4cuda_b200 import _lib as L
from eemd4cuda_b200 import emd_par as M
from eemd4cuda_b200 import signals
from oracle import emd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def raw_run(X, *, tau=0.25, max_sifts=50, max_imf=16, rules="ref", exact=True, end="natural",
            dtype=np.float64, config=None, lengths=None, noise_mode=L.EEMD_NOISE_PREPERTURBED,
            trial_count=None, noise=None, eps=0.2, seed=0, x=None):
    """Per-trial results through eemd_run: imfs, resid, nsift, nmode, mode_sifts, knot_log."""
    dev = torch.device("cuda")
    if X is not None:
        X = np.ascontiguousarray(X, dtype=dtype)
    if lengths is None:
        E, N = X.shape
        lengths = [N]
        trial_count = E
    n_tasks = len(lengths) * trial_count
    p = M.make_params(dtype=dtype, noise_mode=noise_mode, tau=tau, max_sifts=max_sifts,
                      max_imf=max_imf, end=end, rules=rules, exact=exact, config=config,
                      eps=eps, seed=seed)
    src = X if x is None else np.ascontiguousarray(x, dtype=dtype)
    xd = torch.from_numpy(src.ravel()).to(dev)
    tot = sum(lengths) * trial_count
    imfs = torch.zeros((max_imf * tot,), dtype=torch.float64 if dtype == np.float64 else torch.float32,
                       device=dev)
    resid = torch.zeros((tot,), dtype=imfs.dtype, device=dev)
    nsift = torch.zeros((n_tasks,), dtype=torch.int32, device=dev)
    nmode = torch.zeros((n_tasks,), dtype=torch.int32, device=dev)
    msift = torch.zeros((n_tasks, max_imf), dtype=torch.int32, device=dev)
    klog = torch.zeros((n_tasks, max_imf, max_sifts, 2), dtype=torch.int32, device=dev)
    flags = torch.zeros((n_tasks,), dtype=torch.int32, device=dev)
    nz = None if noise is None else torch.from_numpy(np.ascontiguousarray(noise, dtype=dtype).ravel()).to(dev)
    ws = torch.empty((L.workspace_size(p, lengths, trial_count, True),), dtype=torch.uint8, device=dev)
    L.run(p, xd, lengths, 0, trial_count, ws, noise=nz, imfs=imfs, resid_out=resid, nsift=nsift,
          nmode=nmode, mode_sifts=msift, knot_log=klog, flags=flags)
    out = dict(nsift=nsift.cpu().numpy(), nmode=nmode.cpu().numpy(), mode_sifts=msift.cpu().numpy(),
               knot_log=klog.cpu().numpy(), flags=flags.cpu().numpy(), imfs=[], resid=[])
    im = imfs.to(torch.float64).cpu().numpy()
    rs = resid.to(torch.float64).cpu().numpy()
    io = ro = 0
    for s, n in enumerate(lengths):
        for e in range(trial_count):
            out["imfs"].append(im[io:io + max_imf * n].reshape(max_imf, n))
            out["resid"].append(rs[ro:ro + n])
            io += max_imf * n
            ro += n
    return out


def oracle_log(st):
    return [[list(k) for k in mode] for mode in st["knot_log"]]


def engine_log(res, task):
    log = []
    for m in range(int(res["nmode"][task])):
        row = []
        for k in range(res["knot_log"].shape[2]):
            a, b = res["knot_log"][task, m, k]
            if a < 0:
                break
            row.append([int(a), int(b)])
        log.append(row)
    return log


def max_imf_err(a_list, b_list, scale):
    return max((float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) for a, b in zip(a_list, b_list)),
               default=0.0) / scale


@pytest.mark.parametrize("exact", [True, False])
def test_A1_one_sift(small, exact):
    x = small["a1_x"]
    r = M.decompose(x, E=1, max_sifts=1, max_imf=1, exact=exact)
    d = float(np.max(np.abs(r.imfs[0] - small["a1_h1"])))
    assert d <= (1e-13 if exact else 1e-12), d


@pytest.mark.parametrize("exact", [True, False])
def test_plain_8k_mirror(known, small, exact):
    x = signals.plain_emd_8k()
    r = M.decompose(x, E=1, tau=0.2, max_sifts=10, max_imf=10, end="mirror", exact=exact)
    K = known["plain8k_mirror"]
    assert r.n_modes == K["n_modes"]
    assert r.stats["per_mode_sifts"] == K["per_mode_sifts"]
    err = max_imf_err(r.imfs, small["plain8k_imfs"], np.abs(x).max())
    assert err <= (1e-12 if exact else 1e-9), err
    assert r.recon_error() <= 1e-10


@pytest.mark.parametrize("end", ["natural", "mirror"])
@pytest.mark.parametrize("exact", [True, False])
def test_chirp2048(known, small, end, exact):
    x = small["a1_x"]
    r = M.decompose(x, E=1, tau=0.25, max_sifts=50, end=end, exact=exact)
    K = known[f"chirp2048_{end}"]
    assert r.n_modes == K["n_modes"]
    assert r.stats["per_mode_sifts"] == K["per_mode_sifts"]
    err = max_imf_err(r.imfs, small[f"chirp2048_{end}_imfs"], np.abs(x).max())
    assert err <= (1e-12 if exact else 1e-9), err


@pytest.mark.parametrize("exact", [True, False])
def test_config_A_known_answer(known, sweep, exact):
    """ref[:110250], E=1: 9 modes, 26 sifts, per-mode [2,3,7,3,2,2,2,2,3]."""
    x = sweep[:110250]
    res = raw_run(x[None, :], exact=exact)
    A = known["A"]
    assert int(res["nmode"][0]) == A["n_modes"]
    assert int(res["nsift"][0]) == A["total_sifts"]
    assert res["mode_sifts"][0, :A["n_modes"]].tolist() == A["per_mode_sifts"]
    imfs, resid, st = O.emd_1d(x, tau=0.25, max_sifts=50, max_imf=16, record_knots=True)
    assert engine_log(res, 0) == oracle_log(st)
    err = max_imf_err(res["imfs"][0][:A["n_modes"]], imfs, np.abs(x).max())
    assert err <= (1e-12 if exact else 1e-9), err
    for m, ck in zip(res["imfs"][0], A["imf"]):
        assert checksum_close(m, ck, rtol=1e-10 if exact else 1e-8)[0]


@pytest.mark.parametrize("exact", [True, False])
def test_config_B_same_noise(known, sweep, exact):
    """Identical injected perturbations: per-trial modes, sifts and every
    sift's knot counts equal the reference's (test_phase3_gates.py G2/G3)."""
    x = sweep[:110250]
    rng = np.random.default_rng(7)
    X = x[None, :] + 0.2 * np.std(x) * rng.standard_normal((8, len(x)))
    res = raw_run(X, exact=exact)
    B = known["B"]
    assert res["nmode"].tolist() == B["n_modes"]
    assert res["nsift"].tolist() == B["total_sifts"]
    for e in (0, 7):
        imfs, _, st = O.emd_1d(X[e], tau=0.25, max_sifts=50, max_imf=16, record_knots=True)
        assert engine_log(res, e) == oracle_log(st)
        err = max_imf_err(res["imfs"][e][:st["n_modes"]], imfs, np.abs(X[e]).max())
        assert err <= (1e-12 if exact else 1e-9), err


def test_numba_rules_vs_simulated_kernel(known, small):
    """rules='numba' against the reference numba kernel's own outputs."""
    K = known["numba_sim"]
    X = small["numba_X"]
    imfs, nsift, nmode = M.gpu_eemd_full(X, E=X.shape[0], tau=K["tau"], max_sifts=K["max_sifts"],
                                         max_imf=K["maximf"], exact=True)
    assert nsift.tolist() == K["nsift"]
    assert nmode.tolist() == K["nmode"]
    out = small["numba_out"]
    for e in range(X.shape[0]):
        for m in range(int(nmode[e])):
            assert np.max(np.abs(imfs[e, m] - out[e, m])) <= 1e-12


def test_pathological_spacing(known):
    """G8: modulated chirp, N=441000, integers as the reference."""
    x = signals.modulated_chirp()
    res = raw_run(x[None, :], exact=True)
    G = known["G8"]
    assert int(res["nmode"][0]) == G["n_modes"]
    assert int(res["nsift"][0]) == G["total_sifts"]
    assert res["mode_sifts"][0, :G["n_modes"]].tolist() == G["per_mode_sifts"]
    for m, ck in zip(res["imfs"][0], G["imf"]):
        assert checksum_close(m, ck, rtol=1e-9)[0]


def test_determinism_and_seed(sweep):
    """A3/G5 same input twice -> bit-identical; A4 other seed -> differs."""
    x = sweep[:20000]
    a = M.decompose(x, E=8, seed=7, tau=0.25, max_imf=8)
    b = M.decompose(x, E=8, seed=7, tau=0.25, max_imf=8)
    c = M.decompose(x, E=8, seed=8, tau=0.25, max_imf=8)
    assert np.array_equal(a.imfs, b.imfs) and np.array_equal(a.residual, b.residual)
    m = min(a.n_modes, c.n_modes)
    assert np.max(np.abs(a.imfs[:m] - c.imfs[:m])) > 0


@pytest.mark.parametrize("cluster_size", [1, 2, 4, 9])
def test_cluster_size_invariance(sweep, cluster_size):
    """Launch shape must not change results: the knot lists, the solve windows
    and the per-sample arithmetic do not depend on how many CTAs share a
    signal (only the SD sum order moves)."""
    x = sweep[:50000]
    base = raw_run(x[None, :], exact=True, config=M.EngineConfig(cluster_size=2))
    res = raw_run(x[None, :], exact=True, config=M.EngineConfig(cluster_size=cluster_size))
    assert res["nmode"].tolist() == base["nmode"].tolist()
    assert res["nsift"].tolist() == base["nsift"].tolist()
    for a, b in zip(res["imfs"][0], base["imfs"][0]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("B,S", [(16, 32), (250, 30), (272, 32), (64, 48)])
def test_block_thomas_windows(sweep, B, S):
    """Decay-seamed windows of any size agree with the exact serial result."""
    x = sweep[:50000]
    ref_imfs, _, st = O.emd_1d(x, tau=0.25, max_sifts=50, max_imf=16)
    res = raw_run(x[None, :], exact=True, config=M.EngineConfig(knots_per_block=B, halo=S))
    assert int(res["nmode"][0]) == st["n_modes"]
    assert int(res["nsift"][0]) == st["total_sifts"]
    err = max_imf_err(res["imfs"][0][:st["n_modes"]], ref_imfs, np.abs(x).max())
    assert err <= 1e-12, err


def test_ensemble_mean_reference_noise(sweep):
    """decompose with the reference GPU path's own noise stream equals the
    oracle EEMD on the identical perturbed trials (emd_par.py:225-250)."""
    x = sweep[:12000]
    E = 6
    r = M.decompose(x, E=E, seed=3, eps=0.2, tau=0.25, max_sifts=50, max_imf=10,
                    noise="reference-gpu", exact=True)
    X = x[None, :] + O.noise_gpu_stream(x, E, 0.2, 3)
    avg, resid, res = O.eemd(x, X, tau=0.25, max_sifts=50, max_imf=10)
    assert r.n_modes == avg.shape[0]
    assert r.stats["per_trial_total_sifts"].tolist() == [q[2]["total_sifts"] for q in res]
    assert np.max(np.abs(r.imfs - avg)) <= 1e-12 * np.abs(x).max()
    assert np.max(np.abs(r.residual - resid)) <= 1e-12 * np.abs(x).max()


def test_float32_storage():
    """float32 I/O with float64 solve: decomposition close to float64's."""
    x = signals.harmonic_clicks(4800, seed=1)
    a = M.decompose(x, E=4, seed=1, tau=0.0, max_sifts=10, max_imf=8, dtype=np.float64)
    b = M.decompose(x, E=4, seed=1, tau=0.0, max_sifts=10, max_imf=8, dtype=np.float32)
    assert a.n_modes == b.n_modes
    rel = np.linalg.norm(a.imfs[0] - b.imfs[0]) / np.linalg.norm(a.imfs[0])
    assert rel <= 1e-3, rel
    assert b.recon_error() <= 1e-5 * np.abs(x).max()


def test_philox_noise_statistics():
    """Recover each trial's noise as sum(IMFs)+residual-x: zero mean, std eps*std(x)."""
    N, E = 20000, 8
    x = np.sin(np.arange(N) * 0.05)
    res = raw_run(None, x=x, lengths=[N], trial_count=E, noise_mode=L.EEMD_NOISE_PHILOX,
                  eps=0.3, seed=11, exact=False, max_imf=24, tau=0.25)
    sigma = 0.3 * np.std(x)
    noises = []
    for e in range(E):
        nz = res["imfs"][e].sum(axis=0) + res["resid"][e] - x
        noises.append(nz / sigma)
        assert abs(nz.mean() / sigma) < 5.0 / np.sqrt(N)
        assert abs(nz.std() / sigma - 1.0) < 0.03
    c = np.corrcoef(np.stack(noises))
    assert np.max(np.abs(c - np.eye(E))) < 0.05


def test_batched_uneven_signals_equal_single_runs():
    """Many signals of different length in one launch == one launch each."""
    lengths = [4096, 9000, 3000]
    xs = [signals.harmonic_clicks(n, seed=1000 + i) for i, n in enumerate(lengths)]
    cfg = M.EngineConfig()
    E = 3
    batched = raw_run(None, x=np.concatenate(xs), lengths=lengths, trial_count=E,
                      noise_mode=L.EEMD_NOISE_PHILOX, eps=0.2, seed=5, exact=False, tau=0.0,
                      max_sifts=10, max_imf=8, config=cfg)
    assert batched["nmode"].min() >= 1
    # the Philox stream is keyed by (signal index, trial): signal 0 of the
    # batch has the same keys as a single-signal run of it
    one0 = raw_run(None, x=xs[0], lengths=[lengths[0]], trial_count=E, noise_mode=L.EEMD_NOISE_PHILOX,
                   eps=0.2, seed=5, exact=False, tau=0.0, max_sifts=10, max_imf=8, config=cfg)
    assert batched["nmode"][:E].tolist() == one0["nmode"].tolist()
    for e in range(E):
        assert np.array_equal(batched["imfs"][e], one0["imfs"][e])


def test_watchdog_reports_timeout_and_context_survives(small):
    """A bounded wait on a flag nothing sets returns EEMD_E_TIMEOUT; the next
    run on the same context succeeds."""
    x = np.tile(small["a1_x"], 4)
    with pytest.raises(L.EngineError) as ei:
        M.decompose(x, E=1, max_sifts=2, max_imf=2, config=M.EngineConfig(watchdog=-2000))
    assert ei.value.status == L.EEMD_E_TIMEOUT
    r = M.decompose(x, E=1, max_sifts=2, max_imf=2)
    assert r.n_modes == 2


def test_workspace_too_small_is_reported():
    dev = torch.device("cuda")
    p = M.make_params(max_imf=4)
    x = torch.zeros(1000, dtype=torch.float64, device=dev)
    need = L.workspace_size(p, [1000], 1, False)
    ws = torch.empty((need - 256,), dtype=torch.uint8, device=dev)
    with pytest.raises(L.EngineError) as ei:
        L.run(p, x, [1000], 0, 1, ws)
    assert ei.value.status == L.EEMD_E_NOMEM


def test_knot_capacity_overflow_is_reported_and_context_survives():
    """The survey's forced knot-capacity overflow: the bounds-checked build
    honours params.reserved as a cap on the knot lists (knots of one kind per
    warp segment).  A cap far below what a 48 000-sample signal needs returns
    EEMD_E_KNOT_OVERFLOW as a status (the task stops at the step that
    overflowed; nothing is written past the cap), and the next call on the
    same context -- with the cap lifted -- succeeds and equals the release
    build.  (The reference's own bound is K = max(16, N // 2), emd_gpu.py:297-298.)"""
    chk = L.load_variant(L.LIB_DIR / "libeemd_b200_checked.so")
    dev = torch.device("cuda")
    x = signals.harmonic_clicks(48000, seed=1)
    N = len(x)
    xd = torch.from_numpy(x).to(dev)
    for cap in (16, 64):
        p = M.make_params(tau=0.0, max_sifts=10, max_imf=8)
        p.reserved = cap
        ws = torch.empty((L.workspace_size(p, [N], 1, False),), dtype=torch.uint8, device=dev)
        with pytest.raises(L.EngineError) as ei:
            L.run(p, xd, [N], 0, 1, ws, lib=chk)
        assert ei.value.status == L.EEMD_E_KNOT_OVERFLOW
    p = M.make_params(tau=0.0, max_sifts=10, max_imf=8)
    outs = []
    for lib in (chk, None):
        ws = torch.empty((L.workspace_size(p, [N], 1, False),), dtype=torch.uint8, device=dev)
        imfs = torch.zeros((8 * N,), dtype=torch.float64, device=dev)
        nmode = torch.zeros((1,), dtype=torch.int32, device=dev)
        L.run(p, xd, [N], 0, 1, ws, imfs=imfs, nmode=nmode, lib=lib)
        outs.append((imfs.cpu().numpy(), int(nmode.item())))
    assert outs[0][1] == outs[1][1] == 8
    assert np.array_equal(outs[0][0], outs[1][0])


@pytest.mark.parametrize("cta_warps,cluster", [(5, 4), (5, 13), (5, 16), (4, 16)])
def test_launch_shapes_give_identical_results(cta_warps, cluster):
    """Every launch shape the autotune table may choose -- 4- or 5-warp CTAs,
    up to 16 CTAs per task (80 knot segments) -- gives the same IMFs bit for
    bit as 4-warp CTAs in clusters of 4 (fixed sift counts, so no decision
    depends on how the SD sums are grouped)."""
    x = signals.harmonic_clicks(65536, seed=3)
    kw = dict(tau=0.0, max_sifts=5, max_imf=3, exact=False, noise_mode=L.EEMD_NOISE_PHILOX, eps=0.2, seed=4,
              lengths=[len(x)], trial_count=2)
    base = raw_run(None, x=x, config=M.EngineConfig(cta_warps=4, cluster_size=4), **kw)
    other = raw_run(None, x=x, config=M.EngineConfig(cta_warps=cta_warps, cluster_size=cluster), **kw)
    assert other["nmode"].tolist() == base["nmode"].tolist()
    assert np.array_equal(other["knot_log"], base["knot_log"])
    for a, b in zip(other["imfs"], base["imfs"]):
        assert np.array_equal(a, b)


def test_results_stay_valid_across_calls():
    """decompose returns its IMFs and residual as views of pinned host memory
    of that call: a later call (same shape, and a different one) leaves an
    earlier result untouched, plain EMD and EEMD alike."""
    x1 = signals.harmonic_clicks(12000, seed=5)
    x2 = signals.harmonic_clicks(12000, seed=6)
    for kw in (dict(E=1, tau=0.25, max_sifts=20), dict(E=4, tau=0.25, max_sifts=20, seed=3)):
        r1 = M.decompose(x1, **kw)
        keep = (r1.imfs.copy(), r1.residual.copy())
        r2 = M.decompose(x2, **kw)
        r3 = M.decompose(signals.plain_emd_8k(), **kw)
        assert np.array_equal(r1.imfs, keep[0]) and np.array_equal(r1.residual, keep[1])
        assert r2.imfs.shape[1] == 12000 and r3.imfs.shape[1] == 8192
        assert np.allclose(r1.imfs.sum(axis=0) + r1.residual, x1, atol=1e-9)
