"""eemd_run_static: the engine without a caller workspace.

Some callers cannot allocate device memory at the moment they need a
decomposition: code running inside a CUDA-graph capture, a real-time audio
callback, or a host that lets another allocator own all device memory.  For
them the library keeps its own fixed-size scratch array on the device; this
file checks that the entry point built on it gives the same results as the
workspace entry point (eemd_run) on two calls in a row, and that a problem
larger than the static scratch is refused with a clear status.

The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from eemd4cuda_b200 import _lib as L
from eemd4cuda_b200 import emd_par as M
from eemd4cuda_b200 import signals

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ensemble(x, E, seed, static):
    """Ensemble sums, counts and per-trial counters of one batch, through
    eemd_run_static (static=True) or eemd_run with a torch workspace."""
    dev = torch.device("cuda")
    N = len(x)
    p = M.make_params(noise_mode=L.EEMD_NOISE_PHILOX, eps=0.2, seed=seed, tau=0.25,
                      max_sifts=20, max_imf=10)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev)
    imf_sum = torch.zeros((10, N), dtype=torch.float64, device=dev)
    count = torch.zeros((10,), dtype=torch.int32, device=dev)
    nsift = torch.zeros((E,), dtype=torch.int32, device=dev)
    nmode = torch.zeros((E,), dtype=torch.int32, device=dev)
    if static:
        L.run_static(p, xd, [N], 0, E, imf_sum=imf_sum, mode_count=count, nsift=nsift,
                     nmode=nmode)
    else:
        ws = torch.empty((L.workspace_size(p, [N], E, False),), dtype=torch.uint8, device=dev)
        L.run(p, xd, [N], 0, E, ws, imf_sum=imf_sum, mode_count=count, nsift=nsift, nmode=nmode)
    torch.cuda.synchronize()
    return (imf_sum.cpu().numpy(), count.cpu().numpy(), nsift.cpu().numpy(),
            nmode.cpu().numpy())


def test_static_entry_matches_workspace_entry_twice():
    # two different problems back to back: the shared static scratch keeps the
    # first call's contents, which must not leak into the second result
    for x, E, seed in ((signals.harmonic_clicks(12000, seed=3), 6, 11),
                       (signals.plain_emd_8k(), 4, 12)):
        a = _ensemble(x, E, seed, static=True)
        b = _ensemble(x, E, seed, static=False)
        scale = float(np.abs(x).max())
        np.testing.assert_allclose(a[0], b[0], rtol=0, atol=1e-12 * scale * E)
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(a[2], b[2])
        assert np.array_equal(a[3], b[3])
        assert a[1][0] == E


def test_static_entry_refuses_problems_beyond_its_scratch():
    p = M.make_params(noise_mode=L.EEMD_NOISE_PHILOX, max_imf=10)
    N = 1 << 20
    assert L.workspace_size(p, [N], 8, False) > L.STATIC_SCRATCH_BYTES
    x = torch.zeros((N,), dtype=torch.float64, device="cuda")
    with pytest.raises(L.EngineError) as ei:
        L.run_static(p, x, [N], 0, 8)
    assert ei.value.status == L.EEMD_E_STATIC_CAPACITY
