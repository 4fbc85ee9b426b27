"""EEMD stage adapter on the B200 engine (mirror of audio_eemd/eemd_stage.py:1-92).

run_eemd() calls decompose(), times it, applies the partition-of-unity gate
(recon_error <= 1e-6 * max|x|) and maps failures to typed EEMDError codes:
  eemd.bad_input   ValueError from decompose (bad shape, N < 8, method='cpu', ...)
  eemd.backend     any other failure of the engine
  eemd.recon_fail  partition of unity violated
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import emd_par as M


class EEMDError(Exception):
    """EEMD backend failure or partition-of-unity violation."""

    def __init__(self, message: str, code: str = "eemd.failure"):
        super().__init__(message)
        self.code = code


@dataclass
class Decomp:
    """Result of one EEMD run."""

    x: np.ndarray          # input segment, float64 [N]
    imfs: np.ndarray       # ensemble-averaged IMFs, float64 [n_modes, N]
    residual: np.ndarray   # float64 [N]
    n_modes: int
    stats: dict            # verbatim from decompose (method, E, sifting, ...)
    recon: float           # max|x - (sum imfs + residual)|
    wall_s: float          # wall-clock of the decompose() call


def run_eemd(x: np.ndarray, method: str = "auto", E: int = 64, eps: float = 0.2,
             tau: float = 0.25, max_imf: int = -1, max_sifts: int = 50,
             seed: int = 0, batch: int | None = None, **engine_kw) -> Decomp:
    """Run EMD (E=1) or EEMD (E>1) of a 1-D float64 signal on the engine.

    batch: trials resident at once (None = from free device memory).
    engine_kw: decompose() extensions (noise=, rules=, exact=, dtype=).
    Raises EEMDError on bad input, engine failure, or a partition-of-unity
    violation beyond 1e-6 * max|x|."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    t0 = time.perf_counter()
    try:
        res = M.decompose(x, method=method, E=E, eps=eps, tau=tau, max_imf=max_imf,
                          max_sifts=max_sifts, seed=seed, batch=batch, **engine_kw)
    except ValueError as e:
        raise EEMDError(f"EEMD bad input: {e}", "eemd.bad_input") from e
    except Exception as e:
        raise EEMDError(f"EEMD backend failure: {e}", "eemd.backend") from e
    wall = time.perf_counter() - t0

    recon = float(res.recon_error())
    scale = float(np.abs(x).max())
    if recon > 1e-6 * max(scale, 1e-300):
        raise EEMDError(
            f"partition of unity violated: recon_error={recon:.3e} "
            f"(gate 1e-6*max|x| = {1e-6 * scale:.3e})", "eemd.recon_fail")

    imfs = np.asarray(res.imfs, dtype=np.float64)
    if res.n_modes == 0:
        imfs = np.empty((0, x.shape[0]))
    elif imfs.ndim == 1:
        imfs = imfs[None, :]
    return Decomp(x=x, imfs=imfs, residual=np.asarray(res.residual, dtype=np.float64),
                  n_modes=int(res.n_modes), stats=dict(res.stats), recon=recon, wall_s=wall)
