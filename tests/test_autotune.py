"""Lookup of the threads-per-trial table (eemd4cuda_b200/autotune.py) and its
use by the Python entry points (no GPU needed)."""
import numpy as np

from eemd4cuda_b200 import _lib as L
from eemd4cuda_b200 import autotune as A
from eemd4cuda_b200 import emd_par as M

TABLE = [(4096, 1, 2, 4), (4096, 1024, 1, 4), (65536, 1, 16, 4), (65536, 100, 4, 5), (65536, 4096, 1, 4),
         (1 << 22, 64, 8, 4)]


def test_lookup_nearest_bucket_and_task_count(monkeypatch):
    monkeypatch.setattr(A, "_table", lambda dtype: TABLE if dtype == "f32" else None)
    assert A.cluster_size(48000, 100, "f32") == 4       # nearest bucket 65536, 100 tasks
    assert A.launch_shape(48000, 100, "f32") == (4, 5)
    assert A.cluster_size(70000, 2, "f32") == 16        # 1 task is the nearest count
    assert A.cluster_size(70000, 3000, "f32") == 1
    assert A.cluster_size(5000, 1, "f32") == 2
    assert A.cluster_size(3_000_000, 256, "f32") == 8
    assert A.cluster_size(48000, 100, "f64") == 0       # no table: the engine's own rule
    # never below 2048 samples per CTA
    assert A.cluster_size(20000, 1, "f32") == 9
    # an uneven launch: looked up by its median length, capped by its shortest signal
    assert A.launch_shape(65536, 1, "f32", n_min=8192) == (4, 4)
    assert A.launch_shape(65536, 1, "f32", n_min=65536) == (16, 4)


def test_uneven_batch_uses_the_median_length(monkeypatch):
    """tuned() looks an uneven batch up by its median length (the long
    signals' bucket), not by its shortest signal's."""
    monkeypatch.setattr(A, "_table", lambda dtype: TABLE)
    p = M.make_params(dtype=np.float32)
    q = M.tuned(p, [4096] + [65536] * 4, 1)
    assert (q.cluster_size, q.cta_warps) == (2, 4)   # 65536, 5 tasks -> 16 CTAs of 4 warps, capped to 2 by 4096


def test_tuned_params_respect_an_explicit_choice(monkeypatch):
    monkeypatch.setattr(A, "_table", lambda dtype: TABLE)
    p = M.make_params(dtype=np.float32)
    q = M.tuned(p, [48000], 100)
    assert q.cluster_size == 4 and q.cta_warps == 5 and p.cluster_size == 0 and q.max_sifts == p.max_sifts
    pe = M.make_params(dtype=np.float64, exact=True)
    assert M.tuned(pe, [48000], 100).cta_warps == 0      # exact mode keeps 4-warp CTAs
    p2 = M.make_params(dtype=np.float32, config=M.EngineConfig(cluster_size=3))
    assert M.tuned(p2, [48000], 100).cluster_size == 3
    monkeypatch.setattr(A, "_table", lambda dtype: None)
    assert M.tuned(p, [48000], 100).cluster_size == 0


def test_committed_tables_are_well_formed():
    for dt in ("f32", "f64"):
        path = A.table_path(dt)
        if not path.exists():
            continue
        A._table.cache_clear()
        tab = A._table(dt)
        assert tab and all(1 <= c <= 16 and n >= 1024 and t >= 1 and w in (4, 5) for n, t, c, w in tab)
        assert L.EEMD_F32 == 1
