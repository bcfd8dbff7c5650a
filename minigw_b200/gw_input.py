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
