"""B200-native Li–Stephens imputation engine (PBWT sweep, L-state selection,
fused FP32 forward-backward with posterior dosage and haplotype sampling).

The compute path is the CUDA library ``lib/libswiftimpute_b200.so`` behind the
C ABI in ``include/swiftimpute_b200.h``; this package is a thin Python handle on
it (``Engine``) plus the synthetic workload generator used by tests and bench.
"""
from ._native import NativeLibraryError, SIError, default_params  # noqa: F401

__all__ = ["Engine", "NativeLibraryError", "SIError", "default_params"]


def __getattr__(name):
    if name == "Engine":
        from .engine import Engine
        return Engine
    raise AttributeError(name)
