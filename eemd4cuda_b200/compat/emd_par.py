"""`emd_par` module name for callers that import it from sys.path.

audio_eemd/eemd_stage.py:27-33 inserts a directory into sys.path and runs
`import emd_par`; pointing that directory at eemd4cuda_b200/compat makes the
stage call the B200 engine without editing the caller.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

from eemd4cuda_b200.emd_par import *  # noqa: E402,F401,F403
from eemd4cuda_b200.emd_par import (EMDResult, decompose, gpu_eemd_full,  # noqa: E402,F401
                                    make_reference_sweep)

__all__ = ["decompose", "EMDResult", "make_reference_sweep", "gpu_eemd_full"]
