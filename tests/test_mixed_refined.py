"""The refined mixed form (GWB200_MIXED_REFINED): the FP32 factorisation of eps brought to FP64
accuracy by one energy-functional correction, q~ = -(2 x^T y - z^T z - y^T V y) with z the FP32
backward solve and y = D^1/2 z, evaluated in FP64 (kernels_refine.cu).

Checked against the oracle (the plain-C restatement of the reference, pinned to its goldens) and,
where it is present, the reference's own code:
  * screened forms within 1e-10 relative of the oracle (the unrefined mixed form: ~1e-7);
  * Sigma_c within 1e-10 Ha of the oracle;
  * QP on the H2O regression input within 1 meV of the oracle (and of the golden gw.out row);
  * the correction's paths: several frequency chunks, the mma.sync updates of memory-capped
    handles, a rank-deficient V (the generator's V has rank 2 nmo < n) and a full-rank V.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HA_EV = 27.211386245988
FORMS_RTOL = 1e-10
SIGMA_ATOL = 1e-10


@pytest.fixture(scope="module")
def backend():
    from minigw_b200 import B200Backend

    with B200Backend(0) as be:
        yield be


@pytest.mark.parametrize("nmo,nocc,states,nfreq", [
    (14, 4, list(range(14)), 17),  # n = 40: one block
    (24, 5, [4], 32),              # config-1 shape
    (40, 12, [11, 12], 24),        # n = 336: outer blocks and look-left updates
    (60, 10, [8, 9, 10, 11], 12),  # n = 500, m = 240
])
def test_refined_forms_and_sigma_against_oracle(backend, oracle_lib, nmo, nocc, states, nfreq):
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=nmo + 31)
    om, w = generate_transformed_legendre_grid(nfreq)
    backend.load_system(inp)
    ref_sig, ref_q = oracle_lib.sigma_c(inp, om, w, states)
    q, _ = backend.screened_forms(om, states, precision="mixed-refined")
    err = np.abs(q - ref_q.real).max() / np.abs(ref_q.real).max()
    assert err <= FORMS_RTOL, err
    q32, _ = backend.screened_forms(om, states, precision="mixed")
    err32 = np.abs(q32 - ref_q.real).max() / np.abs(ref_q.real).max()
    assert err < 1e-3 * err32 or err32 == 0.0  # the correction removes the FP32-level error
    sig, _ = backend.sigma_c(om, w, states, precision="mixed-refined")
    assert np.abs(sig - ref_sig).max() <= SIGMA_ATOL


def test_refined_h2o_qp_within_1_mev(backend, h2o_input, oracle_lib):
    from conftest import GOLDEN, read_summary_row

    backend.load_system(h2o_input)
    r = backend.run_g0w0(200, 16, [3, 4, 5], precision="mixed-refined")
    o = oracle_lib.g0w0(h2o_input, 200, 16, [3, 4, 5])
    assert np.abs(r["sigma"] - o["sigma"]).max() <= SIGMA_ATOL
    dqp = np.abs(r["qp"][[3, 4, 5]] - o["qp"][[3, 4, 5]]) * HA_EV * 1e3
    assert dqp.max() <= 1.0, dqp  # meV
    row = read_summary_row(GOLDEN / "h2o" / "gw.out", 5)
    assert abs(r["qp"][4] * HA_EV - row["QP Energy"]) <= 1e-5 * abs(row["QP Energy"]) + 1e-4


def test_refined_multi_chunk_and_capped_handle(backend, oracle_lib, monkeypatch):
    """Frequency chunks of 5 (the correction per chunk), and a memory-capped handle, whose mixed
    updates stay on mma.sync (the solve-only pass then runs the mma.sync right-hand-side tiles)."""
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(40, 12, seed=77)
    states = [10, 11, 12]
    om, w = generate_transformed_legendre_grid(23)
    _, ref_q = oracle_lib.sigma_c(inp, om, w, states)
    scale = np.abs(ref_q.real).max()
    backend.load_system(inp)
    whole, _ = backend.screened_forms(om, states, precision="mixed-refined")
    monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", "5")
    chunked, st = backend.screened_forms(om, states, precision="mixed-refined")
    assert st["frequency_chunks"] == 5
    np.testing.assert_array_equal(chunked, whole)
    monkeypatch.delenv("GWB200_MAX_FREQ_CHUNK")
    with B200Backend(0) as capped:
        capped.set_memory_limit(2 << 30)
        capped.load_system(inp)
        qc, _ = capped.screened_forms(om, states, precision="mixed-refined")
        assert capped.update_kernel() == 8  # mma.sync mixed update
    for q in (whole, qc):
        assert np.abs(q - ref_q.real).max() <= FORMS_RTOL * scale


def test_refined_full_rank_v(backend, h2o_input, oracle_lib):
    """The H2O regression input's V_ph comes from a real basis set (not the generator's rank-2 nmo
    construction): the pivoted Cholesky keeps as many columns as its numerical rank and the forms
    still match."""
    from minigw_b200 import generate_transformed_legendre_grid

    om, _ = generate_transformed_legendre_grid(40)
    backend.load_system(h2o_input)
    q, _ = backend.screened_forms(om, [2, 4, 7], precision="mixed-refined")
    ref = oracle_lib.screened_forms(h2o_input, om, [2, 4, 7])
    assert np.abs(q - ref.real).max() <= FORMS_RTOL * np.abs(ref.real).max()


def test_cfg2_refined_against_reference():
    """nmo=120, nph=2000, six states, 64 frequencies: the refined forms at two frequencies against
    the reference's own code (blas-lapack backend), and Sigma_c against the plain FP64 form."""
    import oracle
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import WORKLOADS, make_workload_input

    wl = WORKLOADS["cfg2"]
    inp = make_workload_input(wl, seed=0)
    om, w = generate_transformed_legendre_grid(wl.nfreq)
    states = list(wl.states)
    with B200Backend(0) as be:
        be.load_system(inp, states)
        q, _ = be.screened_forms(om, states, precision="mixed-refined")
        s64, _ = be.sigma_c(om, w, states)
        s, _ = be.sigma_c(om, w, states, precision="mixed-refined")
    assert np.abs(s - s64).max() <= SIGMA_ATOL
    if oracle.Ref.available:
        ref = oracle.Ref(blas_threads=os.cpu_count())
        fsel = [0, 40]
        rq = ref.forms(inp, om[fsel], states, backend="blas-lapack")
        err = np.abs(q[fsel] - rq.real).max() / np.abs(rq.real).max()
        assert err <= FORMS_RTOL, err


def test_cfg2_chain_against_reference_forms():
    """Config 2 (nmo=120, nph=2000, six states, 64 frequencies), whole chain: the reference's own
    screened forms at every frequency (oracle/_ref, blas-lapack backend), contracted, continued and
    solved by the oracle (Sigma_c(iw), the E_c Pade sweep, QP), against each form of this library.
    Sigma_c within 1e-10 Ha for the plain and the refined forms (the unrefined mixed form at the
    FP32 level); the E_c and QP differences are printed (QP on the synthetic generator is set by
    its Pade conditioning: tests/test_oracle.py::test_pade_qp_sensitivity_synthetic_vs_h2o)."""
    import oracle
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import WORKLOADS, make_workload_input

    if not oracle.Ref.available:
        pytest.skip("the reference's own code (oracle/_ref) is not built")
    wl = WORKLOADS["cfg2"]
    inp = make_workload_input(wl, seed=0)
    om, w = generate_transformed_legendre_grid(wl.nfreq)
    states = list(wl.states)
    rq = oracle.Ref(blas_threads=os.cpu_count()).forms(inp, om, states, backend="blas-lapack")
    o = oracle.Oracle()
    ref_sig = o.sigma_from_forms(inp, om, w, states, rq)
    ref_qp = o.qp(inp, np.diag(o.exchange(inp)).copy(), om, ref_sig, states, wl.npade)
    npts = 2000
    ref_ec = [o.ec_sweep(om, ref_sig[s], wl.npade, npts, inp.fermi_energy) for s in states]
    report = {}
    with B200Backend(0) as be:
        be.load_system(inp, states)
        for prec in ("fp64", "mixed-refined", "mixed"):
            r = be.run_g0w0(wl.nfreq, wl.npade, states, precision=prec)
            dsig = float(np.abs(r["sigma"][states] - ref_sig[states]).max())
            dec = max(float(np.abs(be.pade_sweep(om, r["sigma"][s], wl.npade, npts=npts) - e).max())
                      for s, e in zip(states, ref_ec))
            dqp = np.abs(r["qp"][states] - ref_qp[states]) * HA_EV * 1e3
            report[prec] = (dsig, dec, float(dqp.max()), float(np.median(dqp)))
    for prec, (dsig, dec, dqp, dqp_med) in report.items():
        print(f"cfg2 {prec}: |dSigma_c| {dsig:.2e} Ha, |dE_c sweep| {dec:.2e}, QP max {dqp:.3g} meV "
              f"(median {dqp_med:.3g})")
    assert report["fp64"][0] <= SIGMA_ATOL
    assert report["mixed-refined"][0] <= SIGMA_ATOL
    assert report["mixed"][0] > 100 * report["mixed-refined"][0]  # FP32 level without the correction


@pytest.mark.parametrize("nmo,nocc,states,nfreq", [
    (14, 4, [3, 4], 9), (40, 12, [11, 12], 24), (60, 10, [8, 9, 10, 11], 12)])
def test_refined_gram_int8_matches_dmma(backend, monkeypatch, nmo, nocc, states, nfreq):
    """The correction's y^T V y on the int8 tensor cores (digit slices, the default) against the FP64
    DMMA product (GWB200_REFINE_GRAM=dmma): the same forms to FP64 rounding."""
    from minigw_b200 import generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=nmo + 77)
    om, _ = generate_transformed_legendre_grid(nfreq)
    backend.load_system(inp)
    q8, _ = backend.screened_forms(om, states, precision="mixed-refined")
    monkeypatch.setenv("GWB200_REFINE_GRAM", "dmma")
    q64, _ = backend.screened_forms(om, states, precision="mixed-refined")
    assert np.abs(q8 - q64).max() <= 1e-12 * np.abs(q64).max()
