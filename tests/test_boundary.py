"""CPU tests of the drop-in boundary: the C-ABI library loads and exports every symbol the
header declares, its host-side pieces (grid, HDF5 reader, status codes, host mirror and
output formats) behave like the reference's, and it fails loudly without a GPU."""
from __future__ import annotations

import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, read_complex_lines


def _header_symbols() -> set[str]:
    text = (ROOT / "include" / "gwb200.h").read_text()
    return set(re.findall(r"^\s*(?:int|const char\*)\s+(gwb200_\w+)\s*\(", text, re.M))


def test_library_exports_every_declared_symbol():
    import ctypes

    from minigw_b200 import _lib

    declared = _header_symbols()
    assert declared == set(_lib.EXPORTS)
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for name in declared:
        assert hasattr(lib, name), name


def test_version_names_the_target():
    from minigw_b200 import version

    assert "sm_100a" in version()


def test_grid_bit_exact_against_oracle(oracle_lib):
    from minigw_b200 import generate_transformed_legendre_grid

    for n in (1, 2, 3, 7, 32, 64, 128, 200, 256):
        a = generate_transformed_legendre_grid(n)
        b = oracle_lib.grid(n)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_grid_matches_reference_fixture(cfg1_reference):
    from minigw_b200 import generate_transformed_legendre_grid

    om, w = generate_transformed_legendre_grid(200)
    np.testing.assert_array_equal(om, cfg1_reference["omegas"])
    np.testing.assert_array_equal(w, cfg1_reference["weights"])


def test_grid_rejects_nonpositive():
    from minigw_b200 import GwB200Error, generate_transformed_legendre_grid

    with pytest.raises(GwB200Error):
        generate_transformed_legendre_grid(0)


def test_h5_reader_reads_reference_input(h2o_input):
    inp = h2o_input
    assert inp.nmo == 18 and inp.nocc == 5
    assert abs(inp.fermi_energy * 27.211386245988 - (-2.93264)) < 1e-5  # gw.out:5
    assert inp.eri_mo.shape == (18, 18, 18, 18)
    # chemist-order ERI of a real molecule: (pq|rs) = (rs|pq)
    e = inp.eri_mo
    assert np.allclose(e, e.transpose(2, 3, 0, 1), atol=1e-12)
    assert np.allclose(inp.vxc_mo, inp.vxc_mo.T, atol=1e-12)
    assert np.all(np.diff(inp.mo_energy) >= 0)


def test_h5_reader_errors(tmp_path):
    from minigw_b200 import GwB200Error, read_gw_input_hdf5

    with pytest.raises(GwB200Error) as e:
        read_gw_input_hdf5(str(tmp_path / "missing.h5"))
    assert e.value.status == "GWB200_IO_ERROR"
    bad = tmp_path / "not_hdf5.h5"
    bad.write_bytes(b"plain text, not HDF5" * 10)
    with pytest.raises(GwB200Error) as e:
        read_gw_input_hdf5(str(bad))
    assert e.value.status == "GWB200_IO_ERROR"
    trunc = tmp_path / "trunc.h5"
    trunc.write_bytes((GOLDEN / "h2o" / "gw_input.h5").read_bytes()[:4000])
    with pytest.raises(GwB200Error) as e:
        read_gw_input_hdf5(str(trunc))
    assert e.value.status == "GWB200_IO_ERROR"


def test_create_fails_loudly_without_gpu():
    import torch

    from minigw_b200 import B200Backend, GwB200Error

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(GwB200Error) as e:
        B200Backend(0)
    assert e.value.status == "GWB200_CUDA_ERROR"


def test_selected_states_mirrors_reference():
    from minigw_b200 import GwB200Error, GwSettings, selected_states

    assert selected_states(18, GwSettings()) == [4]
    assert selected_states(6, GwSettings(selected_state_0based=None)) == list(range(6))
    assert selected_states(18, GwSettings(states=[3, 5])) == [3, 5]
    with pytest.raises(GwB200Error):
        selected_states(4, GwSettings(selected_state_0based=4))


def test_backend_capabilities_are_device_family():
    from minigw_b200 import B200Backend

    caps = B200Backend.capabilities()
    assert B200Backend.name() == "b200"
    assert caps["uses_device_memory"] and not caps["thread_safe"] and caps["family"] == "Device"


def test_sigma_file_format_round_trips_golden(tmp_path):
    from minigw_b200 import output_self_energy_before_pade

    gold_path = GOLDEN / "h2o" / "E_c_before_Pade.out"
    vals = read_complex_lines(gold_path)
    sig = np.zeros((18, len(vals)), dtype=np.complex128)
    sig[4] = vals
    out = tmp_path / "E_c_before_Pade.out"
    output_self_energy_before_pade(str(out), sig, 4)
    assert out.read_text() == gold_path.read_text()


def test_energy_table_format_matches_gw_out(h2o_input):
    from minigw_b200 import output_final_energy_table

    # feed the golden table's own numbers back (in Ha) and compare the text
    gold = (GOLDEN / "h2o" / "gw.out").read_text().splitlines()
    i = next(k for k, l in enumerate(gold) if l.startswith("Orbital"))
    row = gold[i + 2].split()
    ks, sx, sc, vxc, qp = (float(v) / 27.211386245988 for v in row[1:6])
    mo = np.zeros(18)
    mo[4] = ks
    sxd = np.zeros(18)
    sxd[4] = sx
    vx = np.zeros((18, 18))
    vx[4, 4] = vxc
    qpa = np.full(18, np.nan)
    qpa[4] = qp
    text = output_final_energy_table(mo, sxd, vx, qpa, [4]).splitlines()
    assert text[0].rstrip() == gold[i].rstrip()
    assert text[1].rstrip() == gold[i + 1].rstrip()
    got = text[2].split()
    assert got[0] == "5"
    # KS, Sigma_x, Vxc, QP round-trip through the 6-digit text exactly; Sigma_c is derived from
    # the rounded inputs (qp + vxc - e - sigma_x), so it only agrees to the inputs' rounding.
    for col in (1, 2, 4, 5):
        assert got[col] == row[col]
    assert abs(float(got[3]) - float(row[3])) < 5e-4


def test_cli_rejects_unknown_flags_and_backends():
    gw = ROOT / "minigw_b200" / "bin" / "gw"
    if not gw.exists():
        pytest.skip("gw CLI not built")
    r = subprocess.run([str(gw), "--bogus"], capture_output=True, text=True)
    assert r.returncode != 0 and "Unknown option: --bogus" in r.stderr
    r = subprocess.run([str(gw), "--linalg-backend", "blas-lapack", "--output-dir", "/tmp/gwb200_cli_test"],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "Unknown --linalg-backend value" in r.stderr
    r = subprocess.run([str(gw), "--frequency-parallel", "openmp", "--output-dir", "/tmp/gwb200_cli_test"],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "OpenMP frequency parallelism" in r.stderr
    r = subprocess.run([str(gw), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--linalg-backend" in r.stderr
    shutil.rmtree("/tmp/gwb200_cli_test", ignore_errors=True)


def test_synthetic_generator_contract():
    from minigw_b200.synthetic import WORKLOADS, make_input

    inp = make_input(12, 3, seed=1)
    again = make_input(12, 3, seed=1)
    np.testing.assert_array_equal(inp.eri_mo, again.eri_mo)
    e = inp.eri_mo
    np.testing.assert_array_equal(e, e.transpose(2, 3, 0, 1))  # (pq|rs) = (rs|pq) bit for bit
    assert np.allclose(e, e.transpose(1, 0, 2, 3), atol=1e-14)
    occ, vir = inp.mo_energy[:3], inp.mo_energy[3:]
    assert np.all((occ >= -1.2) & (occ <= -0.3)) and np.all((vir >= 0.05) & (vir <= 3.0))
    assert inp.fermi_energy == 0.5 * (occ[-1] + vir[0])
    nvir = 9
    v = e[:3, 3:, :3, 3:].reshape(3 * nvir, 3 * nvir)
    assert np.linalg.eigvalsh(v).min() > -1e-12  # PSD (ov|ov) block
    assert WORKLOADS["cfg3"].nph == 5100 and WORKLOADS["cfg3"].ncols == 2000
    assert WORKLOADS["cfg2"].nph == 2000 and WORKLOADS["cfg2"].ncols == 720
    assert WORKLOADS["cfg1"].nph == 95 and WORKLOADS["cfg1"].ncols == 24


def test_reference_executable_with_b200_fails_loudly_without_gpu(tmp_path):
    import torch

    exe = ROOT / "oracle" / "_ref" / "gw_ref_b200"
    if not exe.exists():
        pytest.skip("the reference executable with the b200 backend was not built")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([str(exe), "--linalg-backend", "b200", "--input-dir", str(GOLDEN / "h2o"), "--output-dir",
                        str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "CUDA" in r.stderr
