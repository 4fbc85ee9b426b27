"""eemd_run_static: the engine without a caller workspace.

Some callers cannot allocate device memory themselves: a host application
whose device memory belongs to another allocator or framework, or a plugin
host that forbids device allocations from its plugins.  For them the library
keeps its own fixed-size scratch array on the device; this file checks that
the entry point built on it gives the same results as the workspace entry
point (eemd_run) on two calls in a row, that those calls take no device
memory from the caller's allocator, and that a problem larger than the static
scratch is refused with a clear status.

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
    # two different problems back to back, the larger first: the shared static
    # scratch keeps the first call's contents, which must not leak into the
    # second result.  Both entry points launch the same kernels on the same
    # inputs; every sum is taken in a fixed order and no result depends on
    # which cluster slot (scratch region) ran a task, so the results are
    # identical bit for bit, not merely close.
    for x, E, seed in ((signals.harmonic_clicks(12000, seed=3), 6, 11),
                       (signals.plain_emd_8k(), 4, 12)):
        a = _ensemble(x, E, seed, static=True)
        b = _ensemble(x, E, seed, static=False)
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(a[2], b[2])
        assert np.array_equal(a[3], b[3])
        assert a[1][0] == E


def test_static_entry_takes_no_device_memory():
    """After a first call (which looks up the static array's address), a
    further call leaves torch's allocator statistics unchanged: the engine's
    scratch is the library's own array, not caller memory."""
    x = signals.harmonic_clicks(12000, seed=3)
    dev = torch.device("cuda")
    p = M.make_params(noise_mode=L.EEMD_NOISE_PHILOX, eps=0.2, seed=5, tau=0.25,
                      max_sifts=20, max_imf=10)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev)
    imf_sum = torch.zeros((10, len(x)), dtype=torch.float64, device=dev)
    count = torch.zeros((10,), dtype=torch.int32, device=dev)
    L.run_static(p, xd, [len(x)], 0, 4, imf_sum=imf_sum, mode_count=count)
    torch.cuda.synchronize()
    alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    free0, _ = torch.cuda.mem_get_info()
    L.run_static(p, xd, [len(x)], 0, 4, imf_sum=imf_sum, mode_count=count)
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0
    free1, _ = torch.cuda.mem_get_info()
    # no device allocation of the size of a workspace happened behind torch's back
    assert free0 - free1 < L.workspace_size(p, [len(x)], 4, False)


def test_static_entry_refuses_problems_beyond_its_scratch():
    p = M.make_params(noise_mode=L.EEMD_NOISE_PHILOX, max_imf=10)
    N = 1 << 20
    assert L.workspace_size(p, [N], 8, False) > L.STATIC_SCRATCH_BYTES
    x = torch.zeros((N,), dtype=torch.float64, device="cuda")
    with pytest.raises(L.EngineError) as ei:
        L.run_static(p, x, [N], 0, 8)
    assert ei.value.status == L.EEMD_E_STATIC_CAPACITY
