"""Shared fixtures.  Tests marked `gpu` need a B200; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


def read_complex_lines(path: Path) -> np.ndarray:
    """Parse '(re,im)' lines (E_c_before_Pade.out, src/io.cpp:86-92)."""
    vals = []
    for line in path.read_text().splitlines():
        line = line.strip()
        if not line:
            continue
        re_s, im_s = line.strip("()").split(",")
        vals.append(complex(float(re_s), float(im_s)))
    return np.array(vals)


def read_summary_row(path: Path, orbital: int) -> dict:
    """The orbital row of gw.out's final energy table (eV)."""
    lines = path.read_text().splitlines()
    for i, line in enumerate(lines):
        if line.startswith("Orbital") and "QP Energy" in line:
            for row in lines[i + 2:]:
                parts = row.split()
                if parts and parts[0] == str(orbital):
                    ks, sx, sc, vxc, qp = map(float, parts[1:6])
                    return {"KS Energy": ks, "Sigma_x": sx, "Sigma_c": sc, "Vxc": vxc, "QP Energy": qp}
    raise KeyError(f"orbital {orbital} not in {path}")


def components_close(out: np.ndarray, ref: np.ndarray, tol: float) -> bool:
    """scripts/compare_reference.py:93-98 'components' mode: math.isclose on real and imaginary
    parts separately with rel_tol = abs_tol = tol."""
    ok_r = np.abs(out.real - ref.real) <= np.maximum(tol * np.maximum(np.abs(out.real), np.abs(ref.real)), tol)
    ok_i = np.abs(out.imag - ref.imag) <= np.maximum(tol * np.maximum(np.abs(out.imag), np.abs(ref.imag)), tol)
    return bool(np.all(ok_r & ok_i))


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    return oracle.Oracle()


@pytest.fixture(scope="session")
def h2o_input():
    from minigw_b200 import read_gw_input_hdf5

    return read_gw_input_hdf5(str(GOLDEN / "h2o" / "gw_input.h5"))


@pytest.fixture(scope="session")
def h2o_golden_sigma():
    return read_complex_lines(GOLDEN / "h2o" / "E_c_before_Pade.out")


@pytest.fixture(scope="session")
def cfg1_input():
    from minigw_b200.synthetic import WORKLOADS, make_workload_input

    return make_workload_input(WORKLOADS["cfg1"], seed=0)


@pytest.fixture(scope="session")
def cfg1_reference():
    return dict(np.load(GOLDEN / "cfg1_reference.npz"))
