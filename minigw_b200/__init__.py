"""minigw_b200 -- B200-native (sm_100a) backend for miniGW's per-frequency G0W0 screening and
self-energy path.

The numerical work lives in libgwb200.so (C ABI in include/gwb200.h); this package is the
host-side mirror of the reference's interface (see minigw_b200.gw) plus the synthetic
workload generator used by the tests and the benchmark.

The library is loaded when the first name below is used (any of them imports the binding,
which raises ImportError when libgwb200.so is missing; there is no CPU fallback).  The input
generator (minigw_b200.synthetic) and GwInput (minigw_b200.gw_input) do not load it, so a
process that only runs the reference's own CPU code can use them without mapping the library.
"""
from __future__ import annotations

import importlib

_LIB_NAMES = ("FP64", "MIXED", "MIXED_REFINED", "STATUS", "GwB200Error", "version")
_GW_NAMES = (
    "B200Backend", "B200Server", "GwInput", "GwResult", "GwSettings", "GwSlices", "GwTimings",
    "generate_transformed_legendre_grid", "output_final_energy_table", "output_self_energy_after_pade",
    "output_self_energy_before_pade", "plan_buckets", "read_gw_input_hdf5", "read_gw_input_slices", "run_g0w0",
    "run_g0w0_batch",
    "selected_states",
)

__all__ = list(_LIB_NAMES + _GW_NAMES)


def __getattr__(name: str):
    if name in _LIB_NAMES:
        return getattr(importlib.import_module("._lib", __name__), name)
    if name in _GW_NAMES:
        return getattr(importlib.import_module(".gw", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def __dir__():
    return sorted(list(globals()) + __all__)
