"""minigw_b200 -- B200-native (sm_100a) backend for miniGW's per-frequency G0W0 screening and
self-energy path.

The numerical work lives in libgwb200.so (C ABI in include/gwb200.h); this package is the
host-side mirror of the reference's interface (see minigw_b200.gw) plus the synthetic
workload generator used by the tests and the benchmark.
"""
from ._lib import FP64, MIXED, STATUS, GwB200Error, version
from .gw import (
    B200Backend,
    B200Server,
    GwInput,
    GwResult,
    GwSettings,
    GwTimings,
    generate_transformed_legendre_grid,
    output_final_energy_table,
    output_self_energy_after_pade,
    output_self_energy_before_pade,
    plan_buckets,
    read_gw_input_hdf5,
    run_g0w0,
    run_g0w0_batch,
    selected_states,
)

__all__ = [
    "FP64", "MIXED", "STATUS", "GwB200Error", "version", "B200Backend", "B200Server", "GwInput", "GwResult", "GwSettings",
    "GwTimings", "generate_transformed_legendre_grid", "output_final_energy_table", "output_self_energy_after_pade",
    "output_self_energy_before_pade", "plan_buckets", "read_gw_input_hdf5", "run_g0w0", "run_g0w0_batch",
    "selected_states",
]
