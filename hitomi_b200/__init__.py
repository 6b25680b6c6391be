"""B200-native (sm_100a) FFT clustering estimators with the capabilities of
hitomi_measurement: P_l(k), B_{l1 l2 L}(k1, k2) and zeta_{l1 l2 L}(r1, r2).

The compute path is the CUDA library hitomi_b200/libhitomi_b200.so behind the C ABI
in include/hitomi_gpu.h; `hitomi_b200.api.Context` is its Python host binding.
"""
from .api import Binning, Context, HitomiError  # noqa: F401

__all__ = ["Binning", "Context", "HitomiError"]
