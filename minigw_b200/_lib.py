"""ctypes binding of libgwb200.so (include/gwb200.h).

The library is the product: there is no Python or CPU fallback.  Importing this module
fails loudly when the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libgwb200.so"

STATUS = {
    0: "GWB200_OK",
    1: "GWB200_BAD_SHAPE",
    2: "GWB200_ETA_NONZERO",
    3: "GWB200_NOT_SPD",
    4: "GWB200_OOM",
    5: "GWB200_DEVICE_TIMEOUT",
    6: "GWB200_CUDA_ERROR",
    7: "GWB200_BAD_ARGUMENT",
    8: "GWB200_NO_SYSTEM",
    9: "GWB200_IO_ERROR",
    10: "GWB200_NONPOSITIVE_GAP",
}
STATUS_CODE = {v: k for k, v in STATUS.items()}

FP64 = 0
MIXED = 1
MIXED_REFINED = 2

# Every symbol include/gwb200.h declares.
EXPORTS = (
    "gwb200_last_error", "gwb200_version", "gwb200_create", "gwb200_destroy", "gwb200_set_stream",
    "gwb200_set_memory_limit", "gwb200_server_create", "gwb200_server_submit", "gwb200_server_wait",
    "gwb200_server_destroy",
    "gwb200_load_system", "gwb200_load_system_states", "gwb200_run_g0w0", "gwb200_sigma_c_shard",
    "gwb200_sigma_c", "gwb200_screened_forms", "gwb200_screened_forms_complex", "gwb200_sigma_x_diag", "gwb200_qp", "gwb200_pade_sweep",
    "gwb200_grid", "gwb200_read_input_h5", "gwb200_screened_forms_noalloc", "gwb200_fp64_peak_tflops",
    "gwb200_update_kernel", "gwb200_run_g0w0_batch", "gwb200_plan_buckets", "gwb200_read_resident",
    "gwb200_kernel_profile", "gwb200_load_system_slices", "gwb200_server_submit_slices", "gwb200_server_set_merge",
    "gwb200_server_counters", "gwb200_sigma_c_matrix", "gwb200_read_input_h5_slices",
)


class GwB200Error(RuntimeError):
    """A non-zero gwb200_status, with the library's message (mirrors the reference's
    std::runtime_error with a status name attached)."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.status = STATUS.get(code, f"status {code}")
        super().__init__(f"{self.status}: {message}")


class Stats(C.Structure):
    _fields_ = [
        ("device_ms_total", C.c_double),
        ("device_ms_gather", C.c_double),
        ("device_ms_screening", C.c_double),
        ("device_ms_contract", C.c_double),
        ("flops_screening", C.c_double),
        ("frequency_chunks", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("info", C.c_int64),
        ("nph", C.c_int64),
        ("ncols", C.c_int64),
        ("device_ms_update", C.c_double),
        ("update_launches", C.c_int64),
        ("flops_update", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)
_vp = C.c_void_p


class Request(C.Structure):
    """gwb200_request (include/gwb200.h)."""
    _fields_ = [
        ("nmo", C.c_int64), ("nocc", C.c_int64), ("mo_energy", _dp), ("eri", _dp), ("vxc", _dp),
        ("fermi_energy", C.c_double), ("nfreq", C.c_int64), ("npade", C.c_int64), ("states", _ip),
        ("nstates", C.c_int64), ("eta", C.c_double), ("precision", C.c_int), ("omega_out", _dp),
        ("weight_out", _dp), ("sigma_out", _dp), ("sigma_x_out", _dp), ("qp_out", _dp),
    ]


class RequestSlices(C.Structure):
    """gwb200_request_slices (include/gwb200.h)."""
    _fields_ = [("vph", _dp), ("panel", _dp), ("xdiag", _dp), ("vxc_diag", _dp)]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m minigw_b200.build` "
            "(the B200 backend has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    lib.gwb200_last_error.restype = C.c_char_p
    lib.gwb200_version.restype = C.c_char_p
    lib.gwb200_create.argtypes = [C.c_int, C.POINTER(_vp)]
    lib.gwb200_destroy.argtypes = [_vp]
    lib.gwb200_set_stream.argtypes = [_vp, _vp]
    lib.gwb200_set_memory_limit.argtypes = [_vp, C.c_int64]
    lib.gwb200_server_create.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(_vp)]
    lib.gwb200_server_submit.argtypes = [_vp, C.POINTER(Request), C.POINTER(C.c_int64)]
    lib.gwb200_server_wait.argtypes = [_vp, C.c_int64, C.POINTER(C.c_int), _dp, _dp, _dp]
    lib.gwb200_server_destroy.argtypes = [_vp]
    lib.gwb200_load_system.argtypes = [_vp, C.c_int64, C.c_int64, _dp, _dp, _dp, C.c_double]
    lib.gwb200_load_system_states.argtypes = [_vp, C.c_int64, C.c_int64, _dp, _dp, _dp, C.c_double, _ip, C.c_int64]
    lib.gwb200_sigma_c.argtypes = [_vp, _dp, _dp, C.c_int64, _ip, C.c_int64, C.c_double, C.c_int, _dp,
                                   C.POINTER(Stats)]
    lib.gwb200_sigma_c_matrix.argtypes = [_vp, _dp, _dp, C.c_int64, _ip, C.c_int64, _dp, C.POINTER(Stats)]
    lib.gwb200_sigma_c_shard.argtypes = [_vp, _dp, _dp, C.c_int64, C.c_int64, C.c_int64, _ip, C.c_int64, C.c_double,
                                         C.c_int, _dp, C.POINTER(Stats)]
    lib.gwb200_run_g0w0.argtypes = [_vp, C.c_int64, C.c_int64, _ip, C.c_int64, C.c_double, C.c_int, _dp, _dp, _dp,
                                    _dp, _dp, C.POINTER(Stats)]
    lib.gwb200_screened_forms.argtypes = [_vp, _dp, C.c_int64, _ip, C.c_int64, C.c_double, C.c_int, _dp,
                                          C.POINTER(Stats)]
    lib.gwb200_screened_forms_complex.argtypes = [_vp, _dp, C.c_int64, _ip, C.c_int64, C.c_double, _dp,
                                                  C.POINTER(Stats)]
    lib.gwb200_sigma_x_diag.argtypes = [_vp, _dp]
    lib.gwb200_qp.argtypes = [_vp, _dp, C.c_int64, _dp, C.c_int64, _ip, C.c_int64, _dp]
    lib.gwb200_pade_sweep.argtypes = [_vp, _dp, C.c_int64, _dp, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                      C.c_double, _dp]
    lib.gwb200_grid.argtypes = [C.c_int64, _dp, _dp]
    lib.gwb200_read_input_h5.argtypes = [C.c_char_p, _ip, _ip, _dp, _dp, _dp, _dp]
    lib.gwb200_read_input_h5_slices.argtypes = [C.c_char_p, _ip, C.c_int64, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.gwb200_screened_forms_noalloc.argtypes = [C.c_int64, C.c_int64, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp]
    lib.gwb200_fp64_peak_tflops.argtypes = [_vp, _dp]
    lib.gwb200_update_kernel.argtypes = [_vp, _ip]
    lib.gwb200_read_resident.argtypes = [_vp, _ip, C.c_int64, _dp, _dp]
    lib.gwb200_kernel_profile.argtypes = [_vp, _dp, _dp, _ip]
    lib.gwb200_load_system_slices.argtypes = [_vp, C.c_int64, C.c_int64, _dp, _dp, _dp, _dp, _dp, C.c_double, _ip,
                                              C.c_int64]
    lib.gwb200_server_submit_slices.argtypes = [_vp, C.POINTER(Request), C.POINTER(RequestSlices),
                                                C.POINTER(C.c_int64)]
    lib.gwb200_server_set_merge.argtypes = [_vp, C.c_int]
    lib.gwb200_server_counters.argtypes = [_vp, _ip, _ip]
    lib.gwb200_run_g0w0_batch.argtypes = [C.POINTER(_vp), C.c_int64, _ip, _ip, C.POINTER(_ip), _ip,
                                          C.c_int, C.POINTER(_dp), C.POINTER(_dp), _ip, C.POINTER(Stats)]
    lib.gwb200_plan_buckets.argtypes = [C.c_int64, _ip, _ip, C.c_int64, C.c_int, C.c_int64, C.c_double, C.c_double,
                                        _ip, _ip]
    for name in EXPORTS:
        if name not in ("gwb200_last_error", "gwb200_version"):
            getattr(lib, name).restype = C.c_int
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc != 0:
        raise GwB200Error(rc, lib.gwb200_last_error().decode(errors="replace"))


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype in (np.float64, np.complex128) and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def version() -> str:
    return lib.gwb200_version().decode()
