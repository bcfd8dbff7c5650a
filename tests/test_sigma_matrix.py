"""Sigma_c between states, Sigma_c(p_s, p_t; i w_n): gwb200_sigma_c_matrix against the oracle.

The reference computes the diagonal only; the matrix is an extension beside it.  The oracle's
restatement (Oracle.sigma_c_matrix) builds W_c per frequency from the same C functions as the
pinned diagonal path, so its diagonal is pinned here against Oracle.sigma_c first (CPU test).
The GPU tests then hold the whole matrix to the plain form's parity bar (1e-10 Ha absolute), its
symmetry in (s, t), and its diagonal to the device's own diagonal Sigma_c (same solved rows,
another summation order: 1e-12 relative).
"""
from __future__ import annotations

import numpy as np
import pytest

SIGMA_ATOL = 1e-10


def _grid(oracle_lib, nfreq):
    return oracle_lib.grid(nfreq)


def test_oracle_matrix_diagonal_is_the_pinned_sigma(oracle_lib, h2o_input):
    om, w = _grid(oracle_lib, 24)
    states = [0, 3, 4, 5, 9, 17]
    mat = oracle_lib.sigma_c_matrix(h2o_input, om, w, states)
    diag, _ = oracle_lib.sigma_c(h2o_input, om, w, states)
    assert mat.shape == (6, 6, 24)
    for s, p in enumerate(states):
        np.testing.assert_allclose(mat[s, s], diag[p], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(mat, mat.transpose(1, 0, 2), rtol=1e-12, atol=1e-14)
    # states of different irreducible representations of the molecule's point group couple to zero;
    # the others carry weight of their own
    off = np.abs(mat).max(axis=2)[~np.eye(6, dtype=bool)]
    assert off.max() > 1e-4 and off.min() < 1e-14


def test_oracle_matrix_against_numpy_restatement(oracle_lib):
    """The off-diagonal has no reference counterpart, so the oracle's matrix is checked against a
    second, independent restatement: W_c = (I - diag(Pi0) V)^-1 diag(Pi0) by numpy's LU solve (the
    oracle uses its Gauss-Jordan inverse, src/linalg/linalg.cpp:44-91), panels from the ERI tensor
    by fancy indexing (eri[p, k, i, a], src/workspace/pq_ph_panel.cpp:25-47), and the G0 sum written
    out per (n, f', k) as in src/gw/sigma_c_driver.cpp:154-168."""
    from minigw_b200.synthetic import make_input

    nmo, nocc = 18, 5
    inp = make_input(nmo, nocc, seed=21)
    om, w = _grid(oracle_lib, 6)
    states = [2, 4, 5, 9]
    mat = oracle_lib.sigma_c_matrix(inp, om, w, states)

    nvir = nmo - nocc
    eri = np.asarray(inp.eri_mo).reshape(nmo, nmo, nmo, nmo)
    mo = np.asarray(inp.mo_energy)
    io = np.repeat(np.arange(nocc), nvir)
    av = nocc + np.tile(np.arange(nvir), nocc)
    delta = mo[av] - mo[io]
    v = eri[io[:, None], av[:, None], io[None, :], av[None, :]]  # V[ia, jb] = (ia|jb)
    x = {p: eri[p][:, io, av].T for p in states}  # x_p[ia, k] = (p k|i a)
    ref = np.zeros_like(mat)
    for fp, wp in enumerate(om):
        pi0 = 2.0 * (1.0 / (1j * wp - delta) - 1.0 / (1j * wp + delta))
        wc = np.linalg.solve(np.eye(len(delta)) - pi0[:, None] * v, np.diag(pi0))
        for s, ps in enumerate(states):
            for t, pt in enumerate(states):
                q = np.einsum("ik,ij,jk->k", x[ps], wc, x[pt])
                for fn, wn in enumerate(om):
                    den = 1j * wn + inp.fermi_energy - mo
                    g0 = den / (den * den - (1j * wp) ** 2)
                    ref[s, t, fn] -= np.sum(g0 * q) * w[fp] / np.pi
    assert np.abs(mat - ref).max() <= 1e-12 * np.abs(ref).max()


def test_cross_forms_are_dot_products_of_the_solved_rows(oracle_lib):
    """The identity the device path rests on: with eps = I + D^1/2 V D^1/2 = L L^T (D = -Pi0),
    x_s^T W_c x_t = -(L^-1 D^1/2 x_s) . (L^-1 D^1/2 x_t) for the reference's W_c
    (src/workspace/screening_workspace.cpp:21-66), so one factorisation and its solved rows give
    every cross form; checked against the oracle's W_c at three frequencies."""
    import ctypes as C

    from minigw_b200.synthetic import make_input

    def dp(a):
        return a.ctypes.data_as(C.POINTER(C.c_double))

    nmo, nocc = 20, 6
    inp = make_input(nmo, nocc, seed=4)
    eri = np.ascontiguousarray(inp.eri_mo)
    _, _, delta = oracle_lib.ph_map(nmo, nocc, inp.mo_energy)
    v = oracle_lib.vph(inp)
    n = v.shape[0]
    xs = np.zeros((2, n, nmo))
    for s, p in enumerate((5, 8)):
        oracle_lib.lib.gwo_panel(nmo, nocc, dp(eri), p, 0, nmo, dp(xs[s]))
    for omega in (0.1, 1.0, 10.0):
        pi0 = np.zeros(n, dtype=np.complex128)
        oracle_lib.lib.gwo_pi0(0.0, omega, n, dp(delta), 0.0, dp(pi0))
        wc = np.zeros((n, n), dtype=np.complex128)
        assert oracle_lib.lib.gwo_w_c(n, dp(v), dp(pi0), dp(wc)) == 0
        q_ref = np.einsum("ik,ij,jk->k", xs[0], wc, xs[1])
        dh = np.sqrt(-pi0.real)
        chol = np.linalg.cholesky(np.eye(n) + dh[:, None] * v * dh[None, :])
        w0 = np.linalg.solve(chol, dh[:, None] * xs[0])
        w1 = np.linalg.solve(chol, dh[:, None] * xs[1])
        q = -np.sum(w0 * w1, axis=0)
        assert np.abs(q_ref.imag).max() <= 1e-14 * np.abs(q_ref).max()
        np.testing.assert_allclose(q, q_ref.real, rtol=1e-11, atol=1e-14 * np.abs(q_ref).max())


def _check_against_oracle(be, oracle_lib, inp, nfreq, states):
    om, w = _grid(oracle_lib, nfreq)
    be.load_system(inp)
    mat, stats = be.sigma_c_matrix(om, w, states)
    ns = len(states)
    assert mat.shape == (ns, ns, nfreq)
    np.testing.assert_array_equal(mat, mat.transpose(1, 0, 2))  # both triangles from one sum
    ref = oracle_lib.sigma_c_matrix(inp, om, w, states)
    err = np.abs(mat - ref).max()
    assert err <= SIGMA_ATOL, err
    diag, _ = be.sigma_c(om, w, states)
    for s, p in enumerate(states):
        np.testing.assert_allclose(mat[s, s], diag[p], rtol=1e-12, atol=1e-15)
    assert stats["kernel_launches"] > 0
    return mat


@pytest.mark.gpu
def test_h2o_all_states(oracle_lib, h2o_input):
    from minigw_b200 import B200Backend

    with B200Backend(0) as be:
        _check_against_oracle(be, oracle_lib, h2o_input, 32, list(range(18)))


@pytest.mark.gpu
def test_synthetic_subset_and_one_state(oracle_lib):
    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import make_input

    inp = make_input(40, 12, seed=3)
    with B200Backend(0) as be:
        mat = _check_against_oracle(be, oracle_lib, inp, 20, [0, 5, 11, 12, 20, 39])
        one = _check_against_oracle(be, oracle_lib, inp, 20, [11])
        np.testing.assert_allclose(one[0, 0], mat[2, 2], rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_several_frequency_chunks(oracle_lib, monkeypatch):
    """The cross forms are taken per frequency chunk, after that chunk's factorisation: with
    chunks of 3 frequencies the matrix is the one-chunk matrix to rounding, and the oracle's."""
    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import make_input

    inp = make_input(36, 9, seed=11)
    states = [6, 8, 9, 12]
    om, w = _grid(oracle_lib, 11)
    with B200Backend(0) as be:
        be.load_system(inp)
        whole, st1 = be.sigma_c_matrix(om, w, states)
        monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", "3")
        chunked, st3 = be.sigma_c_matrix(om, w, states)
    assert st1["frequency_chunks"] == 1 and st3["frequency_chunks"] == 4
    np.testing.assert_allclose(chunked, whole, rtol=1e-13, atol=1e-16)
    assert np.abs(chunked - oracle_lib.sigma_c_matrix(inp, om, w, states)).max() <= SIGMA_ATOL


@pytest.mark.gpu
def test_sixty_four_states_several_row_chunks(oracle_lib):
    """64 states (the cap): the cross-form kernel stages the rows in 32-column chunks, so n = 384
    spans twelve of them; several frequency chunks are not needed for the kernel's correctness
    but 10 frequencies exercise the per-chunk hook's offsets."""
    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import make_input

    inp = make_input(70, 6, seed=5)
    states = list(range(3, 67))
    with B200Backend(0) as be:
        _check_against_oracle(be, oracle_lib, inp, 10, states)


@pytest.mark.gpu
def test_bad_state_lists():
    from minigw_b200 import B200Backend, GwB200Error
    from minigw_b200.synthetic import make_input

    inp = make_input(70, 6, seed=5)
    om = np.linspace(0.1, 2.0, 4)
    w = np.full(4, 0.1)
    with B200Backend(0) as be:
        be.load_system(inp)
        with pytest.raises(GwB200Error) as e:
            be.sigma_c_matrix(om, w, list(range(65)))
        assert e.value.status == "GWB200_BAD_SHAPE"
        with pytest.raises(GwB200Error):
            be.sigma_c_matrix(om, w, [])
        with pytest.raises(GwB200Error):
            be.sigma_c_matrix(om, w, [0, 70])
        # the handle stays usable after the refusals
        mat, _ = be.sigma_c_matrix(om, w, [0, 1])
        assert np.isfinite(mat).all()
