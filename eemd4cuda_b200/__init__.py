"""B200-native EEMD engine (drop-in for misureaudio/EEMD4CUDA's emd_par path).

    from eemd4cuda_b200 import decompose, EMDResult
    r = decompose(x, E=64, eps=0.2, tau=0.25)

The compute path is libeemd_b200.so (hand-written sm_100a CUDA, C ABI in
include/eemd_b200.h) bound through ctypes; PyTorch tensors are the device
buffers.  There is no CPU fallback.
"""
from .emd_par import EMDResult, EngineConfig, decompose, gpu_eemd_full, make_reference_sweep

__all__ = ["decompose", "EMDResult", "EngineConfig", "gpu_eemd_full", "make_reference_sweep"]
__version__ = "0.1.0"
