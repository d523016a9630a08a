"""B200-native (sm_100a, FP64) implementation of the UGKS2D kinetic hot path.

The compute lives in libugks_b200.so (hand-written CUDA, C ABI in include/ugks_b200.h);
this package holds the host-side mirror of the reference's operator interface.
"""
from .case import (CouetteCase, reference_case, baseline_explicit_case, load_velocity_half32,  # noqa: F401
                   velocity_table, batched_cases, refined_high_order_case)

__all__ = ["CouetteCase", "reference_case", "baseline_explicit_case", "load_velocity_half32", "velocity_table",
           "batched_cases", "refined_high_order_case", "Solver", "Batch"]


def __getattr__(name):
    if name == "Solver":
        from .solver import Solver
        return Solver
    if name == "Batch":
        from .batch import Batch
        return Batch
    raise AttributeError(name)
