"""gwb200_screened_forms_noalloc: the screened-forms solve for callers that cannot call cudaMalloc
(their device memory is owned by another allocator, or they cannot take cudaMalloc's device-wide
synchronisation, or they run under a fixed memory budget).  The caller brings device buffers for
inputs and outputs; every intermediate lives in the library's fixed 4 MiB device array.

Checked through the C ABI against the allocating entry point gwb200_screened_forms on the same
system, on two calls in a row (the second with a different frequency set, so a stale scratch
from the first call would show), within the tolerance the other screened-forms tests use.
This file is collected last so that a failure here never hides the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-11  # same bound as tests/test_gpu_parity.py::test_random_systems_against_oracle


def _device_inputs(inp, states):
    import torch

    nocc, nmo = inp.nocc, inp.nmo
    n = nocc * (nmo - nocc)
    e = inp.eri_mo
    v = np.ascontiguousarray(e[:nocc, nocc:, :nocc, nocc:].reshape(n, n))          # (jb|ia)
    xt = np.ascontiguousarray(e[np.array(states)][:, :, :nocc, nocc:].reshape(len(states) * nmo, n))
    delta = np.ascontiguousarray((inp.mo_energy[nocc:][None, :] - inp.mo_energy[:nocc][:, None]).reshape(n))
    dev = torch.device("cuda", 0)
    return {k: torch.from_numpy(a).to(dev) for k, a in (("v", v), ("xt", xt), ("delta", delta))}, n


def _call_noalloc(lib, n, m, d, omegas):
    import torch

    om = torch.from_numpy(np.ascontiguousarray(omegas)).to("cuda:0")
    out = torch.full((len(omegas), m), float("nan"), dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.gwb200_screened_forms_noalloc(n, m, C.c_void_p(d["v"].data_ptr()), C.c_void_p(d["xt"].data_ptr()),
                                           C.c_void_p(d["delta"].data_ptr()), C.c_void_p(om.data_ptr()), len(omegas),
                                           C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    return rc, out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200._lib import check, lib
    from minigw_b200.synthetic import make_input

    inp = make_input(24, 5, seed=0)
    states = [3, 4, 5]
    d, n = _device_inputs(inp, states)
    m = len(states) * inp.nmo
    with B200Backend(0) as be:
        be.load_system(inp)
        for nfreq in (40, 17):
            om, _ = generate_transformed_legendre_grid(nfreq)
            ref, _ = be.screened_forms(om, states)
            rc, got = _call_noalloc(lib, n, m, d, om)
            check(rc)
            got = got.reshape(nfreq, len(states), inp.nmo)
            scale = max(1.0, np.abs(ref).max())
            assert np.all(np.isfinite(got))
            assert np.abs(got - ref).max() <= REL_TOL * scale


def test_noalloc_rejects_oversize_and_host_pointers():
    from minigw_b200._lib import STATUS, lib

    # beyond the static scratch: refused before any device work
    rc = lib.gwb200_screened_forms_noalloc(600, 600, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), 4,
                                           C.c_void_p(1), None)
    assert STATUS[rc] == "GWB200_BAD_SHAPE"
    assert b"static scratch" in lib.gwb200_last_error()
    # host memory instead of device memory: refused, nothing launched
    host = np.zeros(64)
    p = C.c_void_p(host.ctypes.data)
    rc = lib.gwb200_screened_forms_noalloc(4, 4, p, p, p, p, 2, p, None)
    assert STATUS[rc] == "GWB200_BAD_ARGUMENT"


def test_noalloc_rejects_memory_of_another_device():
    import torch

    from minigw_b200._lib import STATUS, lib

    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU")
    other = torch.zeros(64, dtype=torch.float64, device="cuda:1")
    p = C.c_void_p(other.data_ptr())
    torch.cuda.set_device(0)
    rc = lib.gwb200_screened_forms_noalloc(4, 4, p, p, p, p, 2, p, None)
    assert STATUS[rc] == "GWB200_BAD_ARGUMENT"
    assert b"not of the current device" in lib.gwb200_last_error()
