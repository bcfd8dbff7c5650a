"""GPU parity of the b200 path against the pinned CPU oracle and the reference's goldens.

Tolerances (plain FP64 form):
  * Sigma_c(iw), screened forms q: |GPU - oracle| <= 1e-10 Ha absolute (the stated parity bar),
    plus the reference's own regression tier (components, rtol = atol = 1e-8) against the
    committed H2O golden.
  * gathers, Sigma_x, grid, Pade coefficients, QP update and the E_c sweep: bit-exact on
    identical inputs.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, components_close, read_complex_lines, read_summary_row

pytestmark = pytest.mark.gpu

HA_EV = 27.211386245988
SIGMA_ATOL = 1e-10


@pytest.fixture(scope="module")
def backend():
    from minigw_b200 import B200Backend

    with B200Backend(0) as be:
        yield be


def _oracle_run(oracle_lib, inp, nfreq, npade, states):
    return oracle_lib.g0w0(inp, nfreq, npade, list(states))


def test_h2o_end_to_end_against_golden_and_oracle(backend, h2o_input, h2o_golden_sigma, oracle_lib):
    from minigw_b200 import GwSettings, run_g0w0

    res = run_g0w0(h2o_input, GwSettings(), backend=backend)
    sig = res.sigma_c_im_points
    assert sig.shape == (18, 200)
    assert np.all(sig[np.arange(18) != 4] == 0)
    # the reference's own regression check (scripts/compare_reference.py, reference tier)
    assert components_close(sig[4], h2o_golden_sigma, 1e-8)
    o = _oracle_run(oracle_lib, h2o_input, 200, 16, [4])
    assert np.abs(sig[4] - o["sigma"][4]).max() <= SIGMA_ATOL
    np.testing.assert_array_equal(res.sigma_x_diag, np.diag(o["sigma_x"]))
    row = read_summary_row(GOLDEN / "h2o" / "gw.out", 5)
    assert abs(res.qp_energy[4] * HA_EV - row["QP Energy"]) <= 1e-5 * abs(row["QP Energy"]) + 1e-4
    assert abs(res.qp_energy[4] - o["qp"][4]) < 1e-8  # well-conditioned Pade on H2O
    assert np.all(np.isnan(res.qp_energy[np.arange(18) != 4]))


def test_cfg1_sigma_and_forms_against_oracle(backend, cfg1_input, cfg1_reference, oracle_lib):
    from minigw_b200 import generate_transformed_legendre_grid

    om, w = generate_transformed_legendre_grid(200)
    backend.load_system(cfg1_input)
    sig, stats = backend.sigma_c(om, w, [4])
    np.testing.assert_array_equal(sig[np.arange(24) != 4], 0)
    # the reference itself (committed fixture from oracle/_ref)
    assert np.abs(sig[4] - cfg1_reference["sigma_row"]).max() <= SIGMA_ATOL
    q, _ = backend.screened_forms(om[cfg1_reference["forms_freq_index"]], [4])
    ref_q = cfg1_reference["forms"].real
    assert np.abs(q[:, 0, :] - ref_q).max() <= 1e-10 * max(1.0, np.abs(ref_q).max())
    assert stats["nph"] == 95 and stats["ncols"] == 24
    assert stats["kernel_launches"] > 0


def test_qp_update_bit_exact_on_oracle_sigma(backend, cfg1_input, cfg1_reference, oracle_lib):
    """QP code parity on bit-identical Sigma_c input (the Pade continuation on this
    generator amplifies 1e-15 Sigma differences, so QP parity is gated on identical input)."""
    om = cfg1_reference["omegas"]
    sig = np.zeros((24, 200), dtype=np.complex128)
    sig[4] = cfg1_reference["sigma_row"]
    backend.load_system(cfg1_input)
    qp = backend.qp(om, sig, 16, [4])
    assert qp[4] == cfg1_reference["qp"]
    sx = backend.sigma_x_diag()
    np.testing.assert_array_equal(sx, cfg1_reference["sigma_x_diag"])


def test_pade_sweep_bit_exact_on_oracle_sigma(backend, oracle_lib, h2o_golden_sigma, h2o_input):
    om, _ = oracle_lib.grid(200)
    backend.load_system(h2o_input)
    dev = backend.pade_sweep(om, h2o_golden_sigma, 16, npts=19836, fermi=h2o_input.fermi_energy)
    host = oracle_lib.ec_sweep(om, h2o_golden_sigma, 16, 19836, h2o_input.fermi_energy)
    np.testing.assert_array_equal(dev, host)
    gold = np.loadtxt(GOLDEN / "h2o" / "E_c_every20.out")
    np.testing.assert_array_equal(dev[::20, 0], gold[:, 0])
    assert np.abs(dev[::20, 1:] - gold[:, 1:]).max() < 1e-4


@pytest.mark.parametrize("npade", [1, 2, 5, 16, 33])
def test_pade_coefficients_edge_sizes(backend, oracle_lib, cfg1_input, npade):
    rng = np.random.default_rng(npade)
    om, _ = oracle_lib.grid(33)
    sig = np.zeros((24, 33), dtype=np.complex128)
    sig[[2, 4, 9]] = rng.standard_normal((3, 33)) * 0.05 + 1j * rng.standard_normal((3, 33)) * 0.01
    backend.load_system(cfg1_input)
    qp = backend.qp(om, sig, npade, [2, 4, 9])
    vd = np.diag(cfg1_input.vxc_mo).copy()
    sx = backend.sigma_x_diag()
    ref = oracle_lib.qp(cfg1_input, sx, om, sig, [2, 4, 9], npade)
    np.testing.assert_array_equal(qp[[2, 4, 9]], ref[[2, 4, 9]])
    assert np.all(np.isnan(np.delete(qp, [2, 4, 9])))
    del vd


@pytest.mark.parametrize("nmo,nocc,states,nfreq", [
    (7, 2, [0, 1, 2, 6], 9),        # tiny: n = 10, one 64-block
    (14, 4, list(range(14)), 17),   # all states, n = 40
    (30, 7, [5, 6, 7, 8], 24),      # n = 161: three Cholesky blocks, ragged edges
    (40, 12, [11, 12], 12),         # n = 336: six blocks
])
def test_random_systems_against_oracle(backend, oracle_lib, nmo, nocc, states, nfreq):
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=nmo)
    om, w = oracle_lib.grid(nfreq)
    backend.load_system(inp)
    sig, _ = backend.sigma_c(om, w, states)
    o = oracle_lib.sigma_c(inp, om, w, states)
    osig, oq = o
    assert np.abs(sig - osig).max() <= SIGMA_ATOL
    q, _ = backend.screened_forms(om, states)
    assert np.abs(oq.imag).max() == 0.0
    scale = max(1.0, np.abs(oq.real).max())
    assert np.abs(q - oq.real).max() <= 1e-11 * scale


def test_frequency_chunking_is_bit_identical(backend, cfg1_input, monkeypatch):
    from minigw_b200 import generate_transformed_legendre_grid

    om, w = generate_transformed_legendre_grid(40)
    backend.load_system(cfg1_input)
    full, s1 = backend.sigma_c(om, w, [3, 4, 5])
    monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", "7")
    part, s2 = backend.sigma_c(om, w, [3, 4, 5])
    assert s1["frequency_chunks"] == 1 and s2["frequency_chunks"] == 6
    np.testing.assert_array_equal(full, part)


def test_repeated_calls_are_deterministic(backend, cfg1_input):
    from minigw_b200 import generate_transformed_legendre_grid

    om, w = generate_transformed_legendre_grid(64)
    backend.load_system(cfg1_input)
    a, _ = backend.sigma_c(om, w, [4])
    b, _ = backend.sigma_c(om, w, [4])
    np.testing.assert_array_equal(a, b)


def test_error_statuses(backend, cfg1_input):
    from minigw_b200 import B200Backend, GwB200Error, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    om, w = generate_transformed_legendre_grid(8)
    with B200Backend(0) as fresh:
        with pytest.raises(GwB200Error) as e:
            fresh.sigma_c(om, w, [0])
        assert e.value.status == "GWB200_NO_SYSTEM"
    backend.load_system(cfg1_input)
    for bad_states in ([24], [-1], [3, 3], []):
        with pytest.raises(GwB200Error) as e:
            backend.sigma_c(om, w, bad_states)
        assert e.value.status == "GWB200_BAD_SHAPE"
    with pytest.raises(GwB200Error) as e:
        backend.screened_forms(om, [4], eta=1e-3)  # real forms exist only at eta == 0
    assert e.value.status == "GWB200_ETA_NONZERO"
    # a virtual level below an occupied one: chi0 is not negative definite
    inp = make_input(10, 3, seed=2)
    inp.mo_energy[4] = inp.mo_energy[0] - 0.1
    backend.load_system(inp)
    with pytest.raises(GwB200Error) as e:
        backend.sigma_c(om, w, [1])
    assert e.value.status == "GWB200_NONPOSITIVE_GAP"
    # a (ov|ov) block that is not PSD makes eps(iw) indefinite at small w: NOT_SPD, no trap
    inp = make_input(10, 3, seed=3)
    nv = 7
    for i in range(3):
        for a in range(3, 10):
            inp.eri_mo[i, a, i, a] = -50.0
    backend.load_system(inp)
    with pytest.raises(GwB200Error) as e:
        backend.sigma_c(om, w, [1])
    assert e.value.status == "GWB200_NOT_SPD"
    del nv
    # the handle stays usable after every error
    backend.load_system(cfg1_input)
    sig, _ = backend.sigma_c(om, w, [4])
    assert np.all(np.isfinite(sig))


def test_cli_drop_in_h2o(tmp_path):
    gw = ROOT / "minigw_b200" / "bin" / "gw"
    out = tmp_path / "out"
    r = subprocess.run([str(gw), "--linalg-backend", "b200", "--input-dir", str(GOLDEN / "h2o"), "--output-dir",
                        str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    sig = read_complex_lines(out / "E_c_before_Pade.out")
    gold = read_complex_lines(GOLDEN / "h2o" / "E_c_before_Pade.out")
    assert components_close(sig, gold, 1e-8)
    row = read_summary_row(out / "gw.out", 5)
    grow = read_summary_row(GOLDEN / "h2o" / "gw.out", 5)
    for key in grow:
        assert abs(row[key] - grow[key]) <= 1e-5 * abs(grow[key]) + 1e-4, key
    ec = np.loadtxt(out / "E_c.out")
    assert ec.shape == (19836, 3)
    gold_ec = np.loadtxt(GOLDEN / "h2o" / "E_c_every20.out")
    assert np.abs(ec[::20] - gold_ec).max() < 1e-4


def test_cfg2_sampled_frequencies_against_reference():
    """nmo=120, nph=2000, six states: the full Sigma_c is checked through size-independent
    properties; two frequencies of q are checked against the reference's own code (blas-lapack
    backend) where oracle/_ref is present."""
    import oracle
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import WORKLOADS, make_workload_input

    wl = WORKLOADS["cfg2"]
    inp = make_workload_input(wl, seed=0)
    om, w = generate_transformed_legendre_grid(wl.nfreq)
    with B200Backend(0) as be:
        be.load_system(inp)
        sig, stats = be.sigma_c(om, w, list(wl.states))
        q, _ = be.screened_forms(om, list(wl.states))
    assert stats["nph"] == 2000 and stats["ncols"] == 720
    assert np.all(np.isfinite(sig))
    # q = -b^T eps^{-1} b with eps >= I: 0 >= q >= -||D^1/2 x||^2
    assert np.all(q <= 0.0)
    nvir = wl.nmo - wl.nocc
    delta = (inp.mo_energy[wl.nocc:][None, :] - inp.mo_energy[:wl.nocc][:, None]).reshape(-1)
    x = inp.eri_mo[np.array(wl.states)][:, :, :wl.nocc, wl.nocc:].reshape(len(wl.states), wl.nmo, -1)
    for f in (0, 31, 63):
        d = 4 * delta / (om[f] ** 2 + delta ** 2)
        bound = -np.einsum("skn,n->sk", x * x, d)
        assert np.all(q[f] >= bound * (1 + 1e-12) - 1e-12)
    del nvir
    if oracle.Ref.available:
        ref = oracle.Ref(blas_threads=os.cpu_count())
        fsel = [0, 40]
        rq = ref.forms(inp, om[fsel], list(wl.states), backend="blas-lapack")
        assert np.abs(rq.imag).max() < 1e-9 * np.abs(rq.real).max()
        err = np.abs(q[fsel] - rq.real).max() / np.abs(rq.real).max()
        assert err < 1e-11, err


def test_run_g0w0_equals_separate_calls(backend, cfg1_input):
    from minigw_b200 import generate_transformed_legendre_grid

    backend.load_system(cfg1_input)
    states = [2, 4, 7]
    r = backend.run_g0w0(48, 12, states)
    om, w = generate_transformed_legendre_grid(48)
    np.testing.assert_array_equal(r["omegas"], om)
    np.testing.assert_array_equal(r["weights"], w)
    sig, _ = backend.sigma_c(om, w, states)
    np.testing.assert_array_equal(r["sigma"], sig)
    np.testing.assert_array_equal(r["sigma_x_diag"], backend.sigma_x_diag())
    qp = backend.qp(om, sig, 12, states)
    np.testing.assert_array_equal(r["qp"][states], qp[states])
    assert np.all(np.isnan(np.delete(r["qp"], states)))
    assert r["stats"]["kernel_launches"] > 0


REF_B200 = ROOT / "oracle" / "_ref" / "gw_ref_b200"


@pytest.mark.skipif(not REF_B200.exists(), reason="the reference executable with the b200 backend was not built")
def test_reference_executable_with_b200_backend(tmp_path):
    """The reference's own `gw` (its main, CLI, backend factory, run_g0w0 and writers) with the
    b200 backend registered (factory case + driver branch): `--linalg-backend b200` on the H2O input
    reproduces the reference's committed regression outputs."""
    out = tmp_path / "out"
    r = subprocess.run([str(REF_B200), "--linalg-backend", "b200", "--input-dir", str(GOLDEN / "h2o"), "--output-dir",
                        str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Using the b200 device backend" in (out / "gw.out").read_text()
    sig = read_complex_lines(out / "E_c_before_Pade.out")
    gold = read_complex_lines(GOLDEN / "h2o" / "E_c_before_Pade.out")
    assert components_close(sig, gold, 1e-8)
    row = read_summary_row(out / "gw.out", 5)
    grow = read_summary_row(GOLDEN / "h2o" / "gw.out", 5)
    for key in grow:
        assert abs(row[key] - grow[key]) <= 1e-5 * abs(grow[key]) + 1e-4, key


@pytest.mark.parametrize("eta", [1e-3, 0.05])
@pytest.mark.parametrize("nmo,nocc,states,nfreq", [
    (9, 3, [1, 2, 4], 10),       # one block
    (30, 7, [5, 6, 7, 8], 16),   # n = 161: three blocks, ragged
])
def test_eta_nonzero_against_oracle(backend, oracle_lib, eta, nmo, nocc, states, nfreq):
    """eta != 0: complex symmetric factorisation against the oracle's complex Gauss-Jordan path
    (pinned to the live reference on CPU, tests/test_oracle.py)."""
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=nmo + 1)
    om, w = oracle_lib.grid(nfreq)
    backend.load_system(inp)
    sig, _ = backend.sigma_c(om, w, states, eta=eta)
    osig, oq = oracle_lib.sigma_c(inp, om, w, states, eta=eta)
    assert np.abs(sig - osig).max() <= SIGMA_ATOL
    q, _ = backend.screened_forms_complex(om, states, eta=eta)
    assert np.abs(oq.imag).max() > 0  # genuinely complex
    assert np.abs(q - oq).max() <= 1e-11 * max(1.0, np.abs(oq).max())


def test_eta_nonzero_h2o_end_to_end(backend, oracle_lib, h2o_input):
    from minigw_b200 import GwSettings, run_g0w0

    res = run_g0w0(h2o_input, GwSettings(eta=0.01), backend=backend)
    om, w = oracle_lib.grid(200)
    osig, _ = oracle_lib.sigma_c(h2o_input, om, w, [4], eta=0.01)
    assert np.abs(res.sigma_c_im_points - osig).max() <= SIGMA_ATOL
    assert np.isfinite(res.qp_energy[4])


def test_complex_path_continuous_at_eta_zero(backend, cfg1_input):
    """The complex path at eta -> 0 meets the real SPD path (S = i D^1/2)."""
    from minigw_b200 import generate_transformed_legendre_grid

    om, w = generate_transformed_legendre_grid(24)
    backend.load_system(cfg1_input)
    real, _ = backend.sigma_c(om, w, [4])
    tiny, _ = backend.sigma_c(om, w, [4], eta=1e-13)
    assert np.abs(tiny - real).max() <= 1e-9 * np.abs(real).max()


@pytest.mark.parametrize("nmo,nocc,states,nfreq", [
    (14, 4, list(range(14)), 17),
    (40, 12, [11, 12], 24),      # n = 336: six blocks, outer blocks and look-left updates
])
def test_mixed_form_error_against_fp64(backend, nmo, nocc, states, nfreq):
    """The mixed form (FP32 tall matrices, 3xTF32 updates, no FP64 refinement) carries FP32-level
    error: screened forms and Sigma_c within 2e-5 relative of the FP64 form."""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=nmo + 2)
    om, w = generate_transformed_legendre_grid(nfreq)
    backend.load_system(inp)
    q64, _ = backend.screened_forms(om, states)
    q32, _ = backend.screened_forms(om, states, precision="mixed")
    assert np.abs(q32 - q64).max() <= 2e-5 * np.abs(q64).max()
    s64, _ = backend.sigma_c(om, w, states)
    s32, _ = backend.sigma_c(om, w, states, precision="mixed")
    assert np.abs(s32 - s64).max() <= 2e-5 * np.abs(s64).max()


def test_every_update_variant_agrees(backend, monkeypatch):
    """The autotuner picks among six FP64 trailing-update kernels (tile shape, K slice, pipeline
    depth); each one forced in turn gives the same screened forms up to FP64 rounding."""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(60, 14, seed=11)   # n = 644: trailing updates of several outer blocks
    om, _ = generate_transformed_legendre_grid(5)
    states = [12, 13, 14]
    backend.load_system(inp)
    q_auto, _ = backend.screened_forms(om, states)
    for v in range(6):
        monkeypatch.setenv("GWB200_UPDATE_VARIANT", str(v))
        q, _ = backend.screened_forms(om, states)
        assert np.abs(q - q_auto).max() <= 1e-12 * np.abs(q_auto).max(), v


@pytest.mark.parametrize("nmo,nocc,nst,nfreq,chunk", [
    (40, 10, 4, 6, None),     # n = 300: two outer trailing updates
    (80, 20, 6, 8, "3"),      # n = 1200, three frequency chunks
    (150, 30, 4, 16, None),   # n = 3600: 64-wide last column tiles, many work units per launch
])
def test_tcgen05_update_bit_identical_to_mma_sync(backend, monkeypatch, nmo, nocc, nst, nfreq, chunk):
    """The mixed form's trailing update on tcgen05 (kernels_tc.cu) performs the same 3xTF32
    products in the same order per element as the mma.sync update (kernels_f32.cu): the screened
    forms agree bit for bit."""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    if chunk:
        monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", chunk)
    inp = make_input(nmo, nocc, seed=nmo)
    om, _ = generate_transformed_legendre_grid(nfreq)
    states = list(range(nocc - nst // 2, nocc - nst // 2 + nst))
    backend.load_system(inp)
    monkeypatch.setenv("GWB200_MIXED_UPDATE", "mma")
    q_mma, st_mma = backend.screened_forms(om, states, precision="mixed")
    monkeypatch.delenv("GWB200_MIXED_UPDATE")
    q_tc, st_tc = backend.screened_forms(om, states, precision="mixed")
    assert st_tc["kernel_launches"] > st_mma["kernel_launches"]  # the tcgen05 path ran (two launches per update)
    np.testing.assert_array_equal(q_tc, q_mma)
    q64, _ = backend.screened_forms(om, states)
    assert np.abs(q_tc - q64).max() <= 2e-5 * np.abs(q64).max()


@pytest.mark.parametrize("nmo,nocc,nst,nfreq,chunk", [
    (40, 10, 4, 6, None),     # n = 300
    (80, 20, 6, 8, "3"),      # n = 1200, three frequency chunks
    (150, 30, 4, 16, None),   # n = 3600
])
def test_int8_emulated_fp64_update_matches_dmma(backend, monkeypatch, nmo, nocc, nst, nfreq, chunk):
    """The plain form's trailing update emulated on the int8 tensor cores (kernels_oz.cu, 7-digit
    row slices, exact int32 products) gives the screened forms of the FP64 DMMA update to 1e-12
    relative (measured ~8e-14), deterministically.  (Without GWB200_FP64_UPDATE the autotuner
    picks between the two per geometry.)"""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    if chunk:
        monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", chunk)
    inp = make_input(nmo, nocc, seed=nmo)
    om, _ = generate_transformed_legendre_grid(nfreq)
    states = list(range(nocc - nst // 2, nocc - nst // 2 + nst))
    backend.load_system(inp)
    monkeypatch.setenv("GWB200_FP64_UPDATE", "dmma")
    q64, st64 = backend.screened_forms(om, states)
    monkeypatch.setenv("GWB200_FP64_UPDATE", "ozaki")
    qo, sto = backend.screened_forms(om, states)
    qo2, _ = backend.screened_forms(om, states)
    assert sto["kernel_launches"] > st64["kernel_launches"]  # the int8 path ran (two launches per update)
    assert np.abs(qo - q64).max() <= 1e-12 * np.abs(q64).max()
    np.testing.assert_array_equal(qo, qo2)


def test_update_kernel_reports_the_choice(backend, monkeypatch):
    """gwb200_update_kernel names the trailing-update kernel of the last screening call: a DMMA
    variant (0-5), the int8 emulation (6), the mixed form's tcgen05 (7) or mma.sync (8) update, or
    -1 when there is no outer trailing update."""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    om, _ = generate_transformed_legendre_grid(4)
    backend.load_system(make_input(14, 4, seed=1))  # n = 40: one 64-block, no trailing update
    backend.screened_forms(om, [3, 4])
    assert backend.update_kernel() == -1
    backend.load_system(make_input(40, 10, seed=3))  # n = 300: trailing updates
    monkeypatch.setenv("GWB200_FP64_UPDATE", "dmma")
    backend.screened_forms(om, [9, 10])
    assert 0 <= backend.update_kernel() <= 5
    monkeypatch.setenv("GWB200_FP64_UPDATE", "ozaki")
    backend.screened_forms(om, [9, 10])
    assert backend.update_kernel() == 6
    backend.screened_forms(om, [9, 10], precision="mixed")
    assert backend.update_kernel() == 7
    monkeypatch.setenv("GWB200_MIXED_UPDATE", "mma")
    backend.screened_forms(om, [9, 10], precision="mixed")
    assert backend.update_kernel() == 8


def test_int8_emulated_update_expired_wait(backend, monkeypatch):
    """The int8 update's bounded waits: a withheld operand stage ends in GWB200_DEVICE_TIMEOUT and
    the context stays usable."""
    from minigw_b200 import GwB200Error, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    backend.load_system(make_input(40, 10, seed=3))
    om, _ = generate_transformed_legendre_grid(4)
    monkeypatch.setenv("GWB200_FP64_UPDATE", "ozaki")
    monkeypatch.setenv("GWB200_TEST_EXPIRE_WAIT", "1")
    with pytest.raises(GwB200Error) as e:
        backend.screened_forms(om, [9, 10])
    assert e.value.status == "GWB200_DEVICE_TIMEOUT"
    monkeypatch.delenv("GWB200_TEST_EXPIRE_WAIT")
    qo, _ = backend.screened_forms(om, [9, 10])
    monkeypatch.delenv("GWB200_FP64_UPDATE")
    q64, _ = backend.screened_forms(om, [9, 10])
    assert np.abs(qo - q64).max() <= 1e-12 * np.abs(q64).max()


def test_tcgen05_expired_wait_reports_device_timeout(backend, monkeypatch):
    """Every mbarrier wait of the tcgen05 update is bounded.  With one operand stage withheld
    (test hook), the wait for it expires after about two seconds: the call returns
    GWB200_DEVICE_TIMEOUT and the next call on the same context is correct."""
    from minigw_b200 import GwB200Error, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(40, 10, seed=3)
    om, _ = generate_transformed_legendre_grid(4)
    states = [9, 10]
    backend.load_system(inp)
    monkeypatch.setenv("GWB200_TEST_EXPIRE_WAIT", "1")
    with pytest.raises(GwB200Error) as e:
        backend.screened_forms(om, states, precision="mixed")
    assert e.value.status == "GWB200_DEVICE_TIMEOUT"
    monkeypatch.delenv("GWB200_TEST_EXPIRE_WAIT")
    q32, _ = backend.screened_forms(om, states, precision="mixed")
    q64, _ = backend.screened_forms(om, states)
    assert np.abs(q32 - q64).max() <= 2e-5 * np.abs(q64).max()


def test_mixed_form_h2o_qp(backend, h2o_input, oracle_lib):
    from minigw_b200 import GwB200Error

    backend.load_system(h2o_input)
    r64 = backend.run_g0w0(200, 16, [4])
    r32 = backend.run_g0w0(200, 16, [4], precision="mixed")
    rel = np.abs(r32["sigma"] - r64["sigma"]).max() / np.abs(r64["sigma"]).max()
    assert rel < 2e-5
    assert abs(r32["qp"][4] - r64["qp"][4]) * HA_EV < 0.01  # well-conditioned Pade on H2O: meV-level
    with pytest.raises(GwB200Error) as e:
        backend.run_g0w0(200, 16, [4], eta=0.01, precision="mixed")
    assert e.value.status == "GWB200_BAD_ARGUMENT"
