"""CPU oracle for the G0W0 screening / self-energy path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and --impl reference)
may import this package.  The product (minigw_b200, libgwb200.so) never does.

  Oracle  -- ctypes binding of libgworacle.so, the plain-C restatement of the reference
             algorithm (oracle/gw_oracle.c), pinned against the reference's golden vectors.
  Ref     -- ctypes binding of _ref/libgwref.so: the reference's own sources compiled where
             they lie (oracle/Makefile) plus a C-ABI harness (oracle/ref_harness.cpp).
             Optional: present only where the reference tree was available at build time
             (it travels prebuilt).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libgworacle.so"
REF_SO = HERE / "_ref" / "libgwref.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)
i64 = C.c_int64


def build(ref_root: str | None = None) -> None:
    """make -C oracle (restatement always; _ref when the reference tree exists).  The tree is
    `ref_root`, else the MINIGW_REF_ROOT environment variable; without either only the
    restatement is built."""
    ref_root = ref_root or os.environ.get("MINIGW_REF_ROOT", "")
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF_ROOT={ref_root}", "all"], check=True)


def _d(a):
    return None if a is None else np.ascontiguousarray(a).ctypes.data_as(_dp)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64).ctypes.data_as(_ip)


class Oracle:
    """The C restatement (oracle/gw_oracle.c)."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        lib = C.CDLL(str(ORACLE_SO))
        lib.gwo_ph_map.argtypes = [i64, i64, _dp, _ip, _ip, _dp]
        lib.gwo_vph.argtypes = [i64, i64, _dp, _dp]
        lib.gwo_exchange.argtypes = [i64, i64, _dp, _dp]
        lib.gwo_pi0.argtypes = [C.c_double, C.c_double, i64, _dp, C.c_double, _dp]
        lib.gwo_inverse.argtypes = [i64, _dp, _dp]
        lib.gwo_w_c.argtypes = [i64, _dp, _dp, _dp]
        lib.gwo_panel.argtypes = [i64, i64, _dp, i64, i64, i64, _dp]
        lib.gwo_qforms.argtypes = [i64, _dp, _dp, i64, _dp]
        lib.gwo_screened_forms.argtypes = [i64, i64, _dp, _dp, i64, _dp, _ip, i64, C.c_double, i64, _dp]
        lib.gwo_sigma_from_forms.argtypes = [i64, _dp, C.c_double, i64, _dp, _dp, _ip, i64, i64, _dp, _dp]
        lib.gwo_sigma_c.argtypes = [i64, i64, _dp, _dp, C.c_double, i64, _dp, _dp, _ip, i64, C.c_double, i64, _dp]
        lib.gwo_grid.argtypes = [i64, _dp, _dp]
        lib.gwo_pade_coeffs.argtypes = [i64, _dp, _dp, i64, _dp, _dp]
        lib.gwo_pade_coeffs.restype = i64
        lib.gwo_pade_eval.argtypes = [i64, _dp, C.c_double, _dp, _dp]
        lib.gwo_qp.argtypes = [i64, _dp, C.c_double, _dp, _dp, i64, _dp, _dp, _ip, i64, i64, _dp]
        lib.gwo_ec_sweep.argtypes = [i64, _dp, _dp, i64, i64, C.c_double, C.c_double, C.c_double, _dp]
        self.lib = lib

    def grid(self, n):
        om, w = np.zeros(n), np.zeros(n)
        assert self.lib.gwo_grid(n, _d(om), _d(w)) == 0
        return om, w

    def ph_map(self, nmo, nocc, mo):
        n = nocc * (nmo - nocc)
        io, am, de = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n)
        self.lib.gwo_ph_map(nmo, nocc, _d(mo), io.ctypes.data_as(_ip), am.ctypes.data_as(_ip), _d(de))
        return io, am, de

    def vph(self, inp):
        n = inp.nocc * (inp.nmo - inp.nocc)
        v = np.zeros((n, n))
        self.lib.gwo_vph(inp.nmo, inp.nocc, _d(inp.eri_mo), _d(v))
        return v

    def exchange(self, inp):
        sx = np.zeros((inp.nmo, inp.nmo))
        self.lib.gwo_exchange(inp.nmo, inp.nocc, _d(inp.eri_mo), _d(sx))
        return sx

    def screened_forms(self, inp, omegas, states, eta=0.0, panel=32):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        q = np.zeros((om.shape[0], len(states), inp.nmo), dtype=np.complex128)
        rc = self.lib.gwo_screened_forms(inp.nmo, inp.nocc, _d(inp.mo_energy), _d(inp.eri_mo), om.shape[0], _d(om),
                                         _i(states), len(states), eta, panel, _d(q))
        if rc:
            raise RuntimeError(f"oracle screened_forms failed ({rc})")
        return q

    def sigma_from_forms(self, inp, omegas, weights, states, q, panel=32):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        sig = np.zeros((inp.nmo, om.shape[0]), dtype=np.complex128)
        qc = np.ascontiguousarray(q, dtype=np.complex128)
        self.lib.gwo_sigma_from_forms(inp.nmo, _d(inp.mo_energy), inp.fermi_energy, om.shape[0], _d(om),
                                      _d(np.ascontiguousarray(weights, dtype=np.float64)), _i(states), len(states),
                                      panel, _d(qc), _d(sig))
        return sig

    def sigma_c(self, inp, omegas, weights, states, eta=0.0, panel=32):
        q = self.screened_forms(inp, omegas, states, eta, panel)
        return self.sigma_from_forms(inp, omegas, weights, states, q, panel), q

    def sigma_c_matrix(self, inp, omegas, weights, states, eta=0.0):
        """Sigma_c(p_s, p_t; i w_n) between the states, complex [nstates, nstates, nfreq]: an
        extension beside the reference, which computes the diagonal only (docs/formulation.md:186).
        Per frequency W_c is gwo_w_c's (src/workspace/screening_workspace.cpp:21-66) and the panels
        gwo_panel's (src/workspace/pq_ph_panel.cpp:25-47); the cross forms are
        q[f, k, s, t] = x_{p_s k}^T W_c x_{p_t k}, and the accumulation is gwo_sigma_from_forms's
        (src/gw/sigma_c_driver.cpp:119-169) with q[f, s, k] replaced by q[f, k, s, t].  Its diagonal
        is sigma_c's rows of the states."""
        nmo, nocc = inp.nmo, inp.nocc
        n = nocc * (nmo - nocc)
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        wts = np.ascontiguousarray(weights, dtype=np.float64)
        _, _, delta = self.ph_map(nmo, nocc, inp.mo_energy)
        v = self.vph(inp)
        ns, nf = len(states), om.shape[0]
        xs = np.zeros((ns, n, nmo))  # xs[s] = the panel of state p_s over all k
        for s, p in enumerate(states):
            self.lib.gwo_panel(nmo, nocc, _d(inp.eri_mo), int(p), 0, nmo, _d(xs[s]))
        q = np.zeros((nf, nmo, ns, ns), dtype=np.complex128)
        for f in range(nf):
            pi0 = np.zeros(n, dtype=np.complex128)
            self.lib.gwo_pi0(0.0, float(om[f]), n, _d(delta), eta, _d(pi0))
            wc = np.zeros((n, n), dtype=np.complex128)
            if self.lib.gwo_w_c(n, _d(v), _d(pi0), _d(wc)):
                raise RuntimeError("oracle W_c: near-singular pivot")
            wx = wc @ xs  # [s, i, k]
            q[f] = xs.transpose(2, 0, 1) @ wx.transpose(2, 1, 0)  # [k, s, t]
        mo = np.asarray(inp.mo_energy, dtype=np.float64)
        sig = np.zeros((ns, ns, nf), dtype=np.complex128)
        for fn in range(nf):
            den = 1j * om[fn] + inp.fermi_energy - mo
            g0 = den[None, :] / (den[None, :] ** 2 + om[:, None] ** 2)  # (i w_p)^2 = -w_p^2
            sig[:, :, fn] = -np.einsum("fk,f,fkst->st", g0, wts, q) / np.pi
        return sig

    def pade_coeffs(self, x, y, npar):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.ascontiguousarray(y, dtype=np.complex128)
        c = np.zeros(len(x), dtype=np.complex128)
        xs = np.zeros(len(x), dtype=np.complex128)
        na = self.lib.gwo_pade_coeffs(len(x), _d(x), _d(y), npar, _d(c), _d(xs))
        return c[:na], xs[:na]

    def pade_eval(self, coeffs, z, xs):
        out = np.zeros(1, dtype=np.complex128)
        self.lib.gwo_pade_eval(len(coeffs), _d(np.ascontiguousarray(coeffs)), z, _d(np.ascontiguousarray(xs)),
                               _d(out))
        return out[0]

    def qp(self, inp, sigma_x_diag, omegas, sigma, states, npar):
        out = np.zeros(inp.nmo)
        vd = np.ascontiguousarray(np.diag(inp.vxc_mo))
        self.lib.gwo_qp(inp.nmo, _d(inp.mo_energy), inp.fermi_energy, _d(np.ascontiguousarray(sigma_x_diag)),
                        _d(vd), len(omegas), _d(np.ascontiguousarray(omegas, dtype=np.float64)),
                        _d(np.ascontiguousarray(sigma, dtype=np.complex128)), _i(states), len(states), npar, _d(out))
        return out

    def ec_sweep(self, omegas, sigma_row, npar, npts, fermi, x_start=-6.5, interval=0.00065):
        out = np.zeros((npts, 3))
        self.lib.gwo_ec_sweep(len(omegas), _d(np.ascontiguousarray(omegas, dtype=np.float64)),
                              _d(np.ascontiguousarray(sigma_row, dtype=np.complex128)), npar, npts, fermi, x_start,
                              interval, _d(out))
        return out

    def g0w0(self, inp, nfreq, npade, states):
        """Full oracle run: grid, Sigma_x, Sigma_c(iw), QP (src/gw/gw.cpp:125-191 order)."""
        om, w = self.grid(nfreq)
        sx = self.exchange(inp)
        sig, q = self.sigma_c(inp, om, w, states)
        qp = self.qp(inp, np.diag(sx).copy(), om, sig, states, npade)
        return {"omegas": om, "weights": w, "sigma_x": sx, "sigma": sig, "forms": q, "qp": qp}


class Ref:
    """The reference's own code (oracle/_ref/libgwref.so)."""

    available = REF_SO.exists()

    def __init__(self, blas_threads: int | None = None):
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} was not built (the reference tree was absent at build time)")
        lib = C.CDLL(str(REF_SO))
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_g0w0.argtypes = [i64, i64, C.c_double, _dp, _dp, _dp, i64, i64, _ip, i64, C.c_double, C.c_int,
                                 C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.ref_run_g0w0.argtypes = [i64, i64, C.c_double, _dp, _dp, _dp, i64, i64, i64, C.c_int, _dp, _dp, _dp]
        lib.ref_forms.argtypes = [i64, i64, C.c_double, _dp, _dp, _dp, i64, _dp, _ip, i64, C.c_double, C.c_int, i64,
                                  _dp]
        lib.ref_pair_seconds.argtypes = [i64, i64, C.c_double, _dp, _dp, _dp, i64, _dp, C.c_double, _dp, _ip, i64,
                                         C.c_int, C.c_int, _dp, _dp]
        lib.ref_resident.argtypes = [i64, i64, C.c_double, _dp, _dp, _dp, _ip, i64, _dp, _dp]
        lib.ref_grid.argtypes = [i64, _dp, _dp]
        lib.ref_pade_coeffs.argtypes = [i64, _dp, _dp, i64, _dp, _dp]
        lib.ref_pade_coeffs.restype = i64
        lib.ref_pade_eval.argtypes = [i64, _dp, C.c_double, _dp, _dp]
        lib.ref_write_ec.argtypes = [C.c_char_p, i64, _dp, _dp, i64, i64, C.c_double]
        lib.ref_blas_set_threads.argtypes = [C.c_int]
        lib.ref_blas_get_threads.restype = C.c_int
        if blas_threads is not None:
            lib.ref_blas_set_threads(int(blas_threads))
        self.lib = lib

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError("reference: " + self.lib.ref_last_error().decode())

    def set_blas_threads(self, n: int) -> None:
        self.lib.ref_blas_set_threads(int(n))

    def g0w0(self, inp, nfreq, npade, states, backend="reference", openmp=False, eta=0.0):
        nmo = inp.nmo
        sig = np.zeros((nmo, nfreq), dtype=np.complex128)
        qp, sx = np.zeros(nmo), np.zeros((nmo, nmo))
        om, w = np.zeros(nfreq), np.zeros(nfreq)
        wall = C.c_double()
        self._chk(self.lib.ref_g0w0(nmo, inp.nocc, inp.fermi_energy, _d(inp.mo_energy), _d(inp.eri_mo),
                                    _d(inp.vxc_mo), nfreq, npade, _i(states), len(states), eta,
                                    1 if backend == "blas-lapack" else 0, 1 if openmp else 0, _d(sig), _d(qp),
                                    _d(sx), _d(om), _d(w), C.byref(wall)))
        return {"omegas": om, "weights": w, "sigma_x": sx, "sigma": sig, "qp": qp, "wall_seconds": wall.value}

    def run_g0w0(self, inp, nfreq, npade, state0, backend="reference"):
        nmo = inp.nmo
        sig = np.zeros((nmo, nfreq), dtype=np.complex128)
        qp, sx = np.zeros(nmo), np.zeros((nmo, nmo))
        self._chk(self.lib.ref_run_g0w0(nmo, inp.nocc, inp.fermi_energy, _d(inp.mo_energy), _d(inp.eri_mo),
                                        _d(inp.vxc_mo), nfreq, npade, state0, 1 if backend == "blas-lapack" else 0,
                                        _d(sig), _d(qp), _d(sx)))
        return {"sigma": sig, "qp": qp, "sigma_x": sx}

    def forms(self, inp, omegas, states, backend="blas-lapack", eta=0.0, panel=32):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        q = np.zeros((om.shape[0], len(states), inp.nmo), dtype=np.complex128)
        self._chk(self.lib.ref_forms(inp.nmo, inp.nocc, inp.fermi_energy, _d(inp.mo_energy), _d(inp.eri_mo),
                                     _d(inp.vxc_mo), om.shape[0], _d(om), _i(states), len(states), eta,
                                     1 if backend == "blas-lapack" else 0, panel, _d(q)))
        return q

    def resident(self, inp, states=None, vph=True):
        """The reference's V_ph (n x n) and the panel columns of `states` as rows (nstates*nmo x n)."""
        n = inp.nocc * (inp.nmo - inp.nocc)
        v = np.zeros((n, n)) if vph else None
        panel = np.zeros((len(states) * inp.nmo, n)) if states is not None else None
        st = np.ascontiguousarray(states if states is not None else [0], dtype=np.int64)
        self._chk(self.lib.ref_resident(inp.nmo, inp.nocc, inp.fermi_energy, _d(inp.mo_energy), _d(inp.eri_mo),
                                        _d(inp.vxc_mo), st.ctypes.data_as(_ip), len(states) if states is not None
                                        else 0, _d(v), _d(panel)))
        return v, panel

    def pair_seconds(self, inp, omegas_fp, weights_fp, omega_n, states, backend="blas-lapack", threads=1):
        sec = C.c_double()
        chk = np.zeros(2)
        om = np.ascontiguousarray(omegas_fp, dtype=np.float64)
        self._chk(self.lib.ref_pair_seconds(inp.nmo, inp.nocc, inp.fermi_energy, _d(inp.mo_energy), _d(inp.eri_mo),
                                            _d(inp.vxc_mo), om.shape[0], _d(om), float(omega_n),
                                            _d(np.ascontiguousarray(weights_fp, dtype=np.float64)), _i(states),
                                            len(states), 1 if backend == "blas-lapack" else 0, int(threads),
                                            C.byref(sec), _d(chk)))
        return sec.value, complex(chk[0], chk[1])

    def grid(self, n):
        om, w = np.zeros(n), np.zeros(n)
        self._chk(self.lib.ref_grid(n, _d(om), _d(w)))
        return om, w

    def pade_coeffs(self, x, y, npar):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.ascontiguousarray(y, dtype=np.complex128)
        c = np.zeros(len(x), dtype=np.complex128)
        xs = np.zeros(len(x), dtype=np.complex128)
        na = self.lib.ref_pade_coeffs(len(x), _d(x), _d(y), npar, _d(c), _d(xs))
        return c[:na], xs[:na]

    def pade_eval(self, coeffs, z, xs):
        out = np.zeros(2)
        self.lib.ref_pade_eval(len(coeffs), _d(np.ascontiguousarray(coeffs)), z, _d(np.ascontiguousarray(xs)),
                               _d(out))
        return complex(out[0], out[1])
