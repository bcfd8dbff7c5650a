"""gw_input.h5 read for a known state list (gwb200_read_input_h5_slices): V_ph, the states' panel
rows and the exchange / vxc diagonals read straight from the file's /eri_mo, never the nmo^4
tensor.  CPU: bit for bit the slices numpy cuts from the fully read tensor, and the errors.  GPU:
a solve from the file's slices is bit-identical to the solve from the full tensor."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

H2O = str(GOLDEN / "h2o" / "gw_input.h5")


@pytest.mark.parametrize("states", [[4], [0, 17], [5, 4, 3], list(range(18))])
def test_slices_bit_exact_against_full_read(states):
    from minigw_b200 import read_gw_input_hdf5, read_gw_input_slices
    from minigw_b200.gw_input import slices_from_input

    got = read_gw_input_slices(H2O, states)
    want = slices_from_input(read_gw_input_hdf5(H2O), states)
    assert got.nmo == 18 and got.nocc == want.nocc and got.fermi_energy == want.fermi_energy
    for name in ("mo_energy", "states", "vph", "panel", "xdiag", "vxc_diag"):
        a, b = getattr(got, name), getattr(want, name)
        assert a.shape == b.shape, name
        np.testing.assert_array_equal(a, b, err_msg=name)


def test_slices_reader_errors(tmp_path):
    import ctypes as C

    from minigw_b200 import GwB200Error, read_gw_input_slices
    from minigw_b200._lib import lib

    with pytest.raises(GwB200Error) as e:
        read_gw_input_slices(H2O, [18])
    assert e.value.status == "GWB200_BAD_SHAPE"
    with pytest.raises(GwB200Error) as e:
        read_gw_input_slices(H2O, [-1])
    assert e.value.status == "GWB200_BAD_SHAPE"
    with pytest.raises(GwB200Error) as e:
        read_gw_input_slices(str(tmp_path / "missing.h5"), [0])
    assert e.value.status == "GWB200_IO_ERROR"
    # a file cut inside /eri_mo: the ranged reads stop at the end of the file
    trunc = tmp_path / "trunc.h5"
    trunc.write_bytes((GOLDEN / "h2o" / "gw_input.h5").read_bytes()[:400_000])
    with pytest.raises(GwB200Error) as e:
        read_gw_input_slices(str(trunc), [4])
    assert e.value.status == "GWB200_IO_ERROR"
    # some but not all output arrays: refused before anything is read
    nmo, nocc, fermi = C.c_int64(), C.c_int64(), C.c_double()
    mo = np.zeros(18)
    rc = lib.gwb200_read_input_h5_slices(H2O.encode(), None, 0, C.byref(nmo), C.byref(nocc), C.byref(fermi),
                                         mo.ctypes.data_as(C.POINTER(C.c_double)), None, None, None, None)
    assert rc != 0 and nmo.value == 18


@pytest.mark.gpu
def test_solve_from_file_slices_is_bit_identical():
    from minigw_b200 import B200Backend, read_gw_input_hdf5, read_gw_input_slices

    states = [3, 4, 5]
    full = read_gw_input_hdf5(H2O)
    with B200Backend(0) as a, B200Backend(0) as b:
        a.load_system(full, states)
        b.load_slices(read_gw_input_slices(H2O, states))
        ra = a.run_g0w0(64, 16, states)
        rb = b.run_g0w0(64, 16, states)
    np.testing.assert_array_equal(ra["sigma"], rb["sigma"])
    np.testing.assert_array_equal(ra["sigma_x_diag"], rb["sigma_x_diag"])
    np.testing.assert_array_equal(ra["qp"][states], rb["qp"][states])
