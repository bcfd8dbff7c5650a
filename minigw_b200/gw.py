"""Host-side mirror of the reference's G0W0 interface, driving libgwb200.

Names, argument meaning and error behaviour follow the reference (scnlong/miniGW):

    GwInput / GwSettings / GwResult / GwTimings   include/gw/gw.hpp:17-69
    run_g0w0                                      src/gw/gw.cpp:125-191
    read_gw_input_hdf5                            src/hdf5_input.cpp:192-212
    generate_transformed_legendre_grid            src/gw/frequency_grids.cpp:62-93
    B200Backend (name "b200", device family)      include/linalg/linalg.hpp:23-63,
                                                  registered like src/linalg/backend_factory.cpp:22-66
    output_self_energy_before_pade / _after_pade  src/io.cpp:86-108
    output_final_energy_table                     src/io.cpp:110-126

Failures raise GwB200Error (a RuntimeError, as the reference throws std::runtime_error).
All numerical work runs in libgwb200 on the GPU.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import ctypes as C
import numpy as np

from ._lib import (FP64, MIXED, MIXED_REFINED, GwB200Error, Request, RequestSlices, Stats, _dp, _ip, check, dptr,
                   iptr, lib)
from .gw_input import GwInput, GwSlices

HARTREE_TO_EV = 27.211386245988  # include/types.hpp:12


@dataclass
class GwSettings:
    """include/gw/gw.hpp:25-43.  `states` extends the reference's single selected state /
    all states: when given, it is the explicit 0-based state list (the driver loop of
    src/gw/sigma_c_driver.cpp:142 accepts any list)."""
    num_freq_points_total: int = 200
    num_pade_params: int = 16
    selected_state_0based: Optional[int] = 4
    eta: float = 0.0
    states: Optional[Sequence[int]] = None
    precision: str = "fp64"
    device: int = 0


@dataclass
class GwTimings:
    """include/gw/gw.hpp:45-56, plus the device-event split of the screening."""
    total_wall_seconds: float = 0.0
    exchange_seconds: float = 0.0
    screening_setup_seconds: float = 0.0
    sigma_c_wall_seconds: float = 0.0
    pade_seconds: float = 0.0
    device: dict = field(default_factory=dict)


@dataclass
class GwResult:
    """include/gw/gw.hpp:58-65 (sigma_x is returned as its diagonal)."""
    sigma_x_diag: np.ndarray
    sigma_c_im_points: np.ndarray
    qp_energy: np.ndarray
    omegas: np.ndarray
    weights: np.ndarray
    timings: GwTimings


def generate_transformed_legendre_grid(num_freq_points: int) -> tuple[np.ndarray, np.ndarray]:
    """Transformed Gauss-Legendre grid (src/gw/frequency_grids.cpp:62-93)."""
    if num_freq_points <= 0:
        raise GwB200Error(1, "generate_transformed_legendre_grid: num_freq_points must be positive")
    om = np.zeros(num_freq_points)
    w = np.zeros(num_freq_points)
    check(lib.gwb200_grid(num_freq_points, dptr(om), dptr(w)))
    return om, w


def read_gw_input_hdf5(path: str) -> GwInput:
    """Read gw_input.h5 (src/hdf5_input.cpp:192-212) with libgwb200's minimal HDF5 reader."""
    nmo = C.c_int64()
    nocc = C.c_int64()
    fermi = C.c_double()
    check(lib.gwb200_read_input_h5(path.encode(), C.byref(nmo), C.byref(nocc), C.byref(fermi), None, None, None))
    n = nmo.value
    mo = np.zeros(n)
    eri = np.zeros((n, n, n, n))
    vxc = np.zeros((n, n))
    check(lib.gwb200_read_input_h5(path.encode(), C.byref(nmo), C.byref(nocc), C.byref(fermi),
                                   dptr(mo), dptr(eri), dptr(vxc)))
    return GwInput(eri_mo=eri, mo_energy=mo, vxc_mo=vxc, nocc=nocc.value, fermi_energy=fermi.value)


def read_gw_input_slices(path: str, states) -> GwSlices:
    """Read from gw_input.h5 only what the screening path needs for `states` (V_ph, the states'
    panel rows, the exchange and vxc diagonals, mo_energy), never the nmo^4 ERI tensor
    (gwb200_read_input_h5_slices; the reference reads the whole tensor, src/hdf5_input.cpp:192-212).
    The result equals gw_input.slices_from_input(read_gw_input_hdf5(path), states) bit for bit."""
    st = np.ascontiguousarray(states, dtype=np.int64)
    nmo, nocc, fermi = C.c_int64(), C.c_int64(), C.c_double()
    check(lib.gwb200_read_input_h5_slices(path.encode(), None, 0, C.byref(nmo), C.byref(nocc), C.byref(fermi),
                                          None, None, None, None, None))
    m, o = nmo.value, nocc.value
    n = o * (m - o)
    mo, vph = np.zeros(m), np.zeros((n, n))
    panel, xdiag, vxc_diag = np.zeros((st.shape[0] * m, n)), np.zeros((m, o)), np.zeros(m)
    check(lib.gwb200_read_input_h5_slices(path.encode(), st.ctypes.data_as(_ip), st.shape[0], C.byref(nmo),
                                          C.byref(nocc), C.byref(fermi), dptr(mo), dptr(vph), dptr(panel),
                                          dptr(xdiag), dptr(vxc_diag)))
    return GwSlices(mo_energy=mo, nocc=o, fermi_energy=fermi.value, states=st, vph=vph, panel=panel, xdiag=xdiag,
                    vxc_diag=vxc_diag)


def _precision_code(p: str | int) -> int:
    if p in ("fp64", FP64):
        return FP64
    if p in ("mixed", MIXED):
        return MIXED
    if p in ("mixed-refined", MIXED_REFINED):
        return MIXED_REFINED
    raise GwB200Error(7, f"unknown precision {p!r}")


class B200Backend:
    """The `b200` linear-algebra backend: one device handle holding a resident system.

    capabilities() mirrors gw::linalg::BackendCapabilities for a device backend
    (include/linalg/linalg.hpp:23-41): not thread-safe, uses device memory, so the
    reference's validate_backend_for_execution rejects OpenMP frequency mode with it
    (src/linalg/backend_factory.cpp:68-99).
    """

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.gwb200_create(device, C.byref(h)))
        self._h = h
        self.nmo = 0
        self.nocc = 0
        self.fermi = 0.0

    @staticmethod
    def name() -> str:
        return "b200"

    @staticmethod
    def capabilities() -> dict:
        return {"family": "Device", "thread_safe": False, "uses_internal_threads": False,
                "distributed_mpi": False, "uses_device_memory": True}

    def close(self) -> None:
        if self._h:
            lib.gwb200_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_memory_limit(self, nbytes: int) -> None:
        """Cap the device memory this handle holds (0 = no cap)."""
        check(lib.gwb200_set_memory_limit(self._h, int(nbytes)))

    def set_stream(self, stream_ptr: int | None) -> None:
        """Issue all work on a caller's CUDA stream (e.g. torch.cuda.Stream().cuda_stream)."""
        check(lib.gwb200_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def load_system(self, inp: GwInput, states=None) -> None:
        """Upload a system.  With `states`, only V_ph and those states' panel rows are uploaded
        (gwb200_load_system_states) and later calls must use the same state list."""
        eri = np.ascontiguousarray(inp.eri_mo, dtype=np.float64)
        mo = np.ascontiguousarray(inp.mo_energy, dtype=np.float64)
        vxc = np.ascontiguousarray(inp.vxc_mo, dtype=np.float64)
        nmo = mo.shape[0]
        if eri.size != nmo ** 4 or vxc.size != nmo ** 2:
            raise GwB200Error(1, "MolecularIntegrals: ERI tensor must have shape [nmo,nmo,nmo,nmo]")
        if states is None:
            check(lib.gwb200_load_system(self._h, nmo, int(inp.nocc), dptr(mo), dptr(eri), dptr(vxc),
                                         float(inp.fermi_energy)))
        else:
            st = np.ascontiguousarray(states, dtype=np.int64)
            check(lib.gwb200_load_system_states(self._h, nmo, int(inp.nocc), dptr(mo), dptr(eri), dptr(vxc),
                                                float(inp.fermi_energy), iptr(st), st.shape[0]))
        self.nmo, self.nocc, self.fermi = nmo, int(inp.nocc), float(inp.fermi_energy)

    def load_slices(self, sl: GwSlices) -> None:
        """Upload a system from pre-cut slices (gwb200_load_system_slices); later calls must use
        sl.states."""
        st = np.ascontiguousarray(sl.states, dtype=np.int64)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (sl.mo_energy, sl.vph, sl.panel, sl.xdiag,
                                                                    sl.vxc_diag)]
        check(lib.gwb200_load_system_slices(self._h, sl.nmo, int(sl.nocc), *[dptr(a) for a in arrs],
                                            float(sl.fermi_energy), iptr(st), st.shape[0]))
        self.nmo, self.nocc, self.fermi = sl.nmo, int(sl.nocc), float(sl.fermi_energy)

    def sigma_c(self, omegas, weights, states, eta: float = 0.0, precision="fp64"):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros((self.nmo, om.shape[0]), dtype=np.complex128)
        stats = Stats()
        check(lib.gwb200_sigma_c(self._h, dptr(om), dptr(w), om.shape[0], iptr(st), st.shape[0], float(eta),
                                 _precision_code(precision), dptr(out), C.byref(stats)))
        return out, stats.as_dict()

    def sigma_c_matrix(self, omegas, weights, states):
        """Sigma_c(p_s, p_t; i w_n) between the requested states (plain FP64 form, eta = 0, at most
        64 states): a complex array [nstates, nstates, nfreq], symmetric in (s, t), whose diagonal
        is sigma_c's rows of the states to rounding (gwb200_sigma_c_matrix; the reference computes
        the diagonal only)."""
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros((st.shape[0], st.shape[0], om.shape[0]), dtype=np.complex128)
        stats = Stats()
        check(lib.gwb200_sigma_c_matrix(self._h, dptr(om), dptr(w), om.shape[0], iptr(st), st.shape[0], dptr(out),
                                        C.byref(stats)))
        return out, stats.as_dict()

    def sigma_c_shard(self, omegas, weights, f_begin: int, f_end: int, states, eta: float = 0.0, precision="fp64"):
        """Partial Sigma_c from the integration frequencies [f_begin, f_end) onto the whole grid."""
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros((self.nmo, om.shape[0]), dtype=np.complex128)
        stats = Stats()
        check(lib.gwb200_sigma_c_shard(self._h, dptr(om), dptr(w), om.shape[0], int(f_begin), int(f_end), iptr(st),
                                       st.shape[0], float(eta), _precision_code(precision), dptr(out),
                                       C.byref(stats)))
        return out, stats.as_dict()

    def run_g0w0(self, nfreq: int, npade: int, states, eta: float = 0.0, precision="fp64"):
        """Grid, Sigma_c(iw), Sigma_x diagonal and QP energies in one device call."""
        st = np.ascontiguousarray(states, dtype=np.int64)
        om, w = np.zeros(nfreq), np.zeros(nfreq)
        sig = np.zeros((self.nmo, nfreq), dtype=np.complex128)
        sx, qp = np.zeros(self.nmo), np.zeros(self.nmo)
        stats = Stats()
        check(lib.gwb200_run_g0w0(self._h, int(nfreq), int(npade), iptr(st), st.shape[0], float(eta),
                                  _precision_code(precision), dptr(om), dptr(w), dptr(sig), dptr(sx), dptr(qp),
                                  C.byref(stats)))
        return {"omegas": om, "weights": w, "sigma": sig, "sigma_x_diag": sx, "qp": qp, "stats": stats.as_dict()}

    def screened_forms(self, omegas, states, eta: float = 0.0, precision="fp64"):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros((om.shape[0], st.shape[0], self.nmo))
        stats = Stats()
        check(lib.gwb200_screened_forms(self._h, dptr(om), om.shape[0], iptr(st), st.shape[0], float(eta),
                                        _precision_code(precision), dptr(out), C.byref(stats)))
        return out, stats.as_dict()

    def screened_forms_complex(self, omegas, states, eta: float = 0.0):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros((om.shape[0], st.shape[0], self.nmo), dtype=np.complex128)
        stats = Stats()
        check(lib.gwb200_screened_forms_complex(self._h, dptr(om), om.shape[0], iptr(st), st.shape[0], float(eta),
                                                dptr(out), C.byref(stats)))
        return out, stats.as_dict()

    def sigma_x_diag(self) -> np.ndarray:
        out = np.zeros(self.nmo)
        check(lib.gwb200_sigma_x_diag(self._h, dptr(out)))
        return out

    def qp(self, omegas, sigma, npade, states) -> np.ndarray:
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        sg = np.ascontiguousarray(sigma, dtype=np.complex128)
        st = np.ascontiguousarray(states, dtype=np.int64)
        out = np.zeros(self.nmo)
        check(lib.gwb200_qp(self._h, dptr(om), om.shape[0], dptr(sg), int(npade), iptr(st), st.shape[0], dptr(out)))
        return out

    def pade_sweep(self, omegas, sigma_row, npade, npts=19836, fermi=None, x_start=-6.5, interval=0.00065):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        row = np.ascontiguousarray(sigma_row, dtype=np.complex128)
        out = np.zeros((npts, 3))
        f = self.fermi if fermi is None else fermi
        check(lib.gwb200_pade_sweep(self._h, dptr(om), om.shape[0], dptr(row), int(npade), int(npts), float(f),
                                    float(x_start), float(interval), dptr(out)))
        return out

    def read_resident(self, states=None, vph: bool = True):
        """(V_ph n x n, panel rows nstates*nmo x n) as resident on the device (gwb200_read_resident);
        either is None when not asked for (vph=False / states=None)."""
        n = self.nocc * (self.nmo - self.nocc)
        v = np.zeros((n, n)) if vph else None
        panel, st = None, None
        if states is not None:
            st = np.ascontiguousarray(states, dtype=np.int64)
            panel = np.zeros((st.shape[0] * self.nmo, n))
        check(lib.gwb200_read_resident(self._h, iptr(st) if st is not None else None,
                                       st.shape[0] if st is not None else 0, dptr(v), dptr(panel)))
        return v, panel

    def fp64_peak_tflops(self) -> float:
        v = C.c_double()
        check(lib.gwb200_fp64_peak_tflops(self._h, C.byref(v)))
        return v.value

    KERNEL_PROFILE_KINDS = ("k_gather_vph", "k_gather_panel", "k_build_tall", "k_sigma_contract")

    def kernel_profile(self) -> dict:
        """Event time, algorithmic bytes and launches of the memory-bound kernels since the last
        read, recorded while GWB200_PROFILE=1 (gwb200_kernel_profile)."""
        ms, by = np.zeros(4), np.zeros(4)
        n = np.zeros(4, dtype=np.int64)
        check(lib.gwb200_kernel_profile(self._h, dptr(ms), dptr(by), iptr(n)))
        return {k: {"ms": float(ms[i]), "bytes": float(by[i]), "launches": int(n[i])}
                for i, k in enumerate(self.KERNEL_PROFILE_KINDS)}

    def update_kernel(self) -> int:
        """Trailing-update kernel of the last screening call (gwb200_update_kernel codes)."""
        v = C.c_int64()
        check(lib.gwb200_update_kernel(self._h, C.byref(v)))
        return v.value


def run_g0w0_batch(backends: list[B200Backend], nfreq, npade, states: list, precision="mixed"):
    """Solve every loaded backend's molecule (eta = 0) through shared launches (gwb200_run_g0w0_batch).

    `nfreq` and `npade` are one count for all molecules or one per molecule.  Work runs on
    backends[0]'s stream and workspaces.  Returns per-molecule Sigma_c(iw) and QP energies, the
    number of buckets the molecules were grouped into, and the call's stats."""
    n = len(backends)
    nf = np.ascontiguousarray(np.broadcast_to(np.asarray(nfreq, dtype=np.int64), (n,)))
    npd = np.ascontiguousarray(np.broadcast_to(np.asarray(npade, dtype=np.int64), (n,)))
    hs = (C.c_void_p * n)(*[b._h for b in backends])
    st_arrays = [np.ascontiguousarray(s, dtype=np.int64) for s in states]
    if len(st_arrays) != n:
        raise GwB200Error(7, "one state list per molecule is required")
    st_ptrs = (_ip * n)(*[iptr(a) for a in st_arrays])
    nst = np.array([a.shape[0] for a in st_arrays], dtype=np.int64)
    sig = [np.zeros((b.nmo, int(f)), dtype=np.complex128) for b, f in zip(backends, nf)]
    qp = [np.zeros(b.nmo) for b in backends]
    sig_ptrs = (_dp * n)(*[dptr(a) for a in sig])
    qp_ptrs = (_dp * n)(*[dptr(a) for a in qp])
    nb = C.c_int64()
    stats = Stats()
    check(lib.gwb200_run_g0w0_batch(hs, n, iptr(nf), iptr(npd), st_ptrs, iptr(nst), _precision_code(precision),
                                    sig_ptrs, qp_ptrs, C.byref(nb), C.byref(stats)))
    return {"sigma": sig, "qp": qp, "buckets": nb.value, "stats": stats.as_dict()}


def plan_buckets(nph, ncols, nfreq: int, precision="mixed", budget_bytes: int = 64 << 30, step_us: float = 0.0,
                 tflops: float = 0.0) -> tuple[np.ndarray, int]:
    """Bucket index of every molecule under the batch cost model (host only)."""
    n = np.ascontiguousarray(nph, dtype=np.int64)
    m = np.ascontiguousarray(ncols, dtype=np.int64)
    out = np.zeros(n.shape[0], dtype=np.int64)
    nb = C.c_int64()
    check(lib.gwb200_plan_buckets(n.shape[0], iptr(n), iptr(m), int(nfreq), _precision_code(precision),
                                  int(budget_bytes), float(step_us), float(tflops), iptr(out), C.byref(nb)))
    return out, nb.value


def selected_states(nmo: int, settings: GwSettings) -> list[int]:
    """src/gw/gw.cpp:28-40 (plus the explicit list extension)."""
    if settings.states is not None:
        return [int(s) for s in settings.states]
    if settings.selected_state_0based is not None:
        if settings.selected_state_0based >= nmo:
            raise GwB200Error(1, "Selected state is out of range")
        return [int(settings.selected_state_0based)]
    return list(range(nmo))


def run_g0w0(inp: GwInput, settings: GwSettings, backend: B200Backend | None = None) -> GwResult:
    """src/gw/gw.cpp:125-191 on the b200 backend: grid, exchange, Sigma_c(iw), QP."""
    t0 = time.perf_counter()
    own = backend is None
    be = backend or B200Backend(settings.device)
    try:
        t = time.perf_counter()
        be.load_system(inp)
        setup = time.perf_counter() - t
        states = selected_states(inp.nmo, settings)
        t = time.perf_counter()
        r = be.run_g0w0(settings.num_freq_points_total, settings.num_pade_params, states, settings.eta,
                        settings.precision)
        wall = time.perf_counter() - t
    finally:
        if own:
            be.close()
    timings = GwTimings(total_wall_seconds=time.perf_counter() - t0, screening_setup_seconds=setup,
                        sigma_c_wall_seconds=wall, device=r["stats"])
    return GwResult(sigma_x_diag=r["sigma_x_diag"], sigma_c_im_points=r["sigma"], qp_energy=r["qp"],
                    omegas=r["omegas"], weights=r["weights"], timings=timings)


def _g17(x: float) -> str:
    return format(float(x), ".17g")


def output_self_energy_before_pade(path: str, sigma_c: np.ndarray, state_0based: int) -> None:
    """E_c_before_Pade.out: one '(re,im)' line per frequency at precision 17 (src/io.cpp:86-92)."""
    with open(path, "w") as f:
        for z in sigma_c[state_0based]:
            f.write(f"({_g17(z.real)},{_g17(z.imag)})\n")


def output_self_energy_after_pade(path: str, sweep: np.ndarray) -> None:
    """E_c.out: 'E[eV] Re Im' lines at precision 17 (src/io.cpp:94-108); `sweep` from pade_sweep."""
    with open(path, "w") as f:
        for e, re, im in sweep:
            f.write(f"{_g17(e)} {_g17(re)} {_g17(im)}\n")


def _cpp_default(x: float) -> str:
    # std::ostream default formatting (precision 6, %g-like).
    return format(float(x), ".6g")


def output_final_energy_table(mo_energy, sigma_x_diag, vxc, qp_energy, states) -> str:
    """The summary table of gw.out (src/io.cpp:110-126), returned as text."""
    lines = ["{:<10}{:<15}{:<15}{:<15}{:<15}{:<15}".format("Orbital", "KS Energy", "Sigma_x", "Sigma_c", "Vxc",
                                                           "QP Energy"),
             "{:<10}{:<15}{:<15}{:<15}{:<15}{:<15}".format("-------", "---------", "-------", "-------", "-------",
                                                           "---------")]
    for idx in states:
        sc = qp_energy[idx] + vxc[idx, idx] - mo_energy[idx] - sigma_x_diag[idx]
        vals = [mo_energy[idx], sigma_x_diag[idx], sc, vxc[idx, idx], qp_energy[idx]]
        lines.append("{:<10}".format(idx + 1) + "".join("{:<15}".format(_cpp_default(v * HARTREE_TO_EV)) for v in vals))
    return "\n".join(lines) + "\n"


class B200Server:
    """Continuous-batching request loop (gwb200_server_*): `slots` workers, each with its own
    handle and stream and a device-memory cap of hbm_budget/slots; requests are admitted FIFO as
    workers free up and run concurrently on the GPU."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: int = 64 << 30, merge: int | None = None):
        srv = C.c_void_p()
        check(lib.gwb200_server_create(device, slots, int(hbm_budget_bytes), C.byref(srv)))
        self._s = srv
        self._live = {}
        if merge is not None:
            check(lib.gwb200_server_set_merge(self._s, int(merge)))

    def submit(self, inp: GwInput | GwSlices, nfreq: int, npade: int, states, eta: float = 0.0,
               precision="fp64") -> int:
        """Queue one solve; `inp` is a full system (its ERI is read at load) or GwSlices (whose state
        list must be `states`)."""
        nmo = inp.nmo
        sliced = isinstance(inp, GwSlices)
        keep = {
            "mo": np.ascontiguousarray(inp.mo_energy, dtype=np.float64),
            "states": np.ascontiguousarray(states, dtype=np.int64),
            "omegas": np.zeros(nfreq), "weights": np.zeros(nfreq),
            "sigma": np.zeros((nmo, nfreq), dtype=np.complex128), "sigma_x_diag": np.zeros(nmo), "qp": np.zeros(nmo),
        }
        if sliced:
            if not np.array_equal(np.asarray(inp.states), keep["states"]):
                raise GwB200Error(7, "the state list must be the one the slices were cut for")
            for k in ("vph", "panel", "xdiag", "vxc_diag"):
                keep[k] = np.ascontiguousarray(getattr(inp, k), dtype=np.float64)
        else:
            keep["eri"] = np.ascontiguousarray(inp.eri_mo, dtype=np.float64)
            keep["vxc"] = np.ascontiguousarray(inp.vxc_mo, dtype=np.float64)
        req = Request(nmo, int(inp.nocc), dptr(keep["mo"]), dptr(keep.get("eri")), dptr(keep.get("vxc")),
                      float(inp.fermi_energy), int(nfreq), int(npade), iptr(keep["states"]), len(keep["states"]),
                      float(eta), _precision_code(precision), dptr(keep["omegas"]), dptr(keep["weights"]),
                      dptr(keep["sigma"]), dptr(keep["sigma_x_diag"]), dptr(keep["qp"]))
        keep["req"] = req
        ticket = C.c_int64()
        if sliced:
            sl = RequestSlices(dptr(keep["vph"]), dptr(keep["panel"]), dptr(keep["xdiag"]), dptr(keep["vxc_diag"]))
            keep["slices"] = sl
            check(lib.gwb200_server_submit_slices(self._s, C.byref(req), C.byref(sl), C.byref(ticket)))
        else:
            check(lib.gwb200_server_submit(self._s, C.byref(req), C.byref(ticket)))
        self._live[ticket.value] = keep
        return ticket.value

    def counters(self) -> dict:
        """Batches of two or more requests merged so far, and the requests in them."""
        b, r = C.c_int64(), C.c_int64()
        check(lib.gwb200_server_counters(self._s, C.byref(b), C.byref(r)))
        return {"merged_batches": b.value, "merged_requests": r.value}

    def wait(self, ticket: int) -> dict:
        st = C.c_int()
        q, sv, dv = C.c_double(), C.c_double(), C.c_double()
        rc = lib.gwb200_server_wait(self._s, int(ticket), C.byref(st), C.byref(q), C.byref(sv), C.byref(dv))
        keep = self._live.pop(int(ticket))
        check(rc)
        return {"omegas": keep["omegas"], "weights": keep["weights"], "sigma": keep["sigma"],
                "sigma_x_diag": keep["sigma_x_diag"], "qp": keep["qp"], "queue_ms": q.value,
                "service_ms": sv.value, "device_ms": dv.value}

    def close(self) -> None:
        if self._s:
            lib.gwb200_server_destroy(self._s)
            self._s = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
