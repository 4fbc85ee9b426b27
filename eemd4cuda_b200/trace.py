"""Per-phase cycle counters of a -DEEMD_TRACE build (libeemd_b200_trace.so).

The persistent kernel's thread 0 of every CTA sums clock64() deltas per phase
(lane 0 of every warp for the sweep's sub-phases) and adds them to the
workspace header at exit; `phase_cycles(ws)` reads them back (the header sits
at offset 0 of the workspace).
"""
from __future__ import annotations

import numpy as np

PHASES = ("setup", "solve", "barrier_solve", "sweep", "barrier_sweep", "decide", "claim")
SWEEP_PHASES = ("tile_wait", "values", "extrema_scan", "writes", "solve_staging", "solve_slopes",
                "solve_windows")
_HEADER_INTS = 16  # int32 fields before phase_cycles


def phase_cycles(ws) -> dict:
    """Cycles per phase summed over CTAs, from a workspace tensor after a traced run."""
    raw = ws[: _HEADER_INTS * 4 + 16 * 8].cpu().numpy().view(np.uint8)
    cyc = raw[_HEADER_INTS * 4:].view(np.uint64)
    out = {name: int(cyc[i]) for i, name in enumerate(PHASES)}
    out.update({"sweep." + name: int(cyc[8 + i]) for i, name in enumerate(SWEEP_PHASES)})
    return out
