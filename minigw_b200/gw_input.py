"""GwInput, the host-side system description (include/gw/gw.hpp:17-23).

Kept apart from the library binding so that input generators and readers can be imported
without loading libgwb200.so.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class GwInput:
    """include/gw/gw.hpp:17-23 (eri_mo C-order [nmo]*4, mo_energy, vxc_mo, nocc, fermi_energy)."""
    eri_mo: np.ndarray
    mo_energy: np.ndarray
    vxc_mo: np.ndarray
    nocc: int
    fermi_energy: float

    @property
    def nmo(self) -> int:
        return int(self.mo_energy.shape[0])


@dataclass
class GwSlices:
    """The parts of a system the screening path reads, cut from the ERI for a known state list
    (gwb200_load_system_slices): vph n x n with V_ph[jb, ia] = (jb|ia); panel (nstates*nmo) x n with
    row t*nmo + k = (states[t] k|ia); xdiag nmo x nocc = (p i|p i); vxc_diag the diagonal of vxc_mo."""
    mo_energy: np.ndarray
    nocc: int
    fermi_energy: float
    states: np.ndarray
    vph: np.ndarray
    panel: np.ndarray
    xdiag: np.ndarray
    vxc_diag: np.ndarray

    @property
    def nmo(self) -> int:
        return int(self.mo_energy.shape[0])


def slices_from_input(inp: GwInput, states) -> GwSlices:
    """Cut a full system's slices (numpy indexing; the same values the library's own ingest reads)."""
    nmo, nocc = inp.nmo, int(inp.nocc)
    n = nocc * (nmo - nocc)
    st = np.ascontiguousarray(states, dtype=np.int64)
    e = inp.eri_mo
    vph = np.ascontiguousarray(e[:nocc, nocc:, :nocc, nocc:].reshape(n, n))
    panel = np.ascontiguousarray(e[st][:, :, :nocc, nocc:].reshape(st.shape[0] * nmo, n))
    p = np.arange(nmo)
    xdiag = np.ascontiguousarray(e[p[:, None], np.arange(nocc)[None, :], p[:, None], np.arange(nocc)[None, :]])
    return GwSlices(mo_energy=np.ascontiguousarray(inp.mo_energy, dtype=np.float64), nocc=nocc,
                    fermi_energy=float(inp.fermi_energy), states=st, vph=vph, panel=panel, xdiag=xdiag,
                    vxc_diag=np.ascontiguousarray(np.diag(inp.vxc_mo)))
