"""gwb200_load_system_states (V_ph and the states' panel rows copied straight from the host ERI)
against gwb200_load_system (the (pq|o.) block resident, gathered on the device): identical bits."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(14, 3, [2, 3]), (24, 5, [4]), (30, 4, list(range(30))), (40, 7, [5, 6, 7, 8])]


@pytest.mark.parametrize("nmo,nocc,states", CASES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_state_bound_load_is_bit_identical(nmo, nocc, states, precision):
    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=700 + nmo)
    with B200Backend(0) as full, B200Backend(0) as bound:
        full.load_system(inp)
        bound.load_system(inp, states)
        a = full.run_g0w0(24, 12, states, precision=precision)
        b = bound.run_g0w0(24, 12, states, precision=precision)
        np.testing.assert_array_equal(a["sigma"], b["sigma"])
        np.testing.assert_array_equal(a["sigma_x_diag"], b["sigma_x_diag"])
        np.testing.assert_array_equal(a["qp"][states], b["qp"][states])


@pytest.mark.parametrize("nmo,nocc,states", CASES[:2] + [(120, 20, [17, 18, 19, 20, 21, 22])])
def test_gathers_bit_exact_against_reference(nmo, nocc, states, oracle_lib):
    """Both ingest paths' resident V_ph and panel rows, bit for bit against the reference's
    calculate_v_ph_matrix (src/gw/sigma.cpp:56-71) and PqPhPanelView::make_panel
    (src/workspace/pq_ph_panel.cpp:18-47), and the oracle's gwo_vph."""
    import oracle
    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import make_input

    inp = make_input(nmo, nocc, seed=900 + nmo)
    with B200Backend(0) as full, B200Backend(0) as bound:
        full.load_system(inp)  # V_ph and panels gathered on the device from the (pq|o.) block
        bound.load_system(inp, states)  # copied from the host ERI by 3D copies
        va, pa = full.read_resident(states)
        vb, pb = bound.read_resident(states)
    np.testing.assert_array_equal(va, vb)
    np.testing.assert_array_equal(pa, pb)
    np.testing.assert_array_equal(va, oracle_lib.vph(inp))
    if oracle.Ref.available:
        rv, rp = oracle.Ref().resident(inp, states)
        np.testing.assert_array_equal(va, rv)
        np.testing.assert_array_equal(pa, rp)


def test_kernel_profile_of_memory_bound_kernels(monkeypatch):
    """gwb200_kernel_profile: with GWB200_PROFILE=1 the gathers, the build and the contraction are
    timed with events and credited with their algorithmic bytes; reading resets the sums."""
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    nmo, nocc, states = 30, 6, [5, 6]
    inp = make_input(nmo, nocc, seed=3)
    n, m = nocc * (nmo - nocc), len(states) * nmo
    om, w = generate_transformed_legendre_grid(10)
    monkeypatch.setenv("GWB200_PROFILE", "1")
    with B200Backend(0) as be:
        be.load_system(inp)
        be.sigma_c(om, w, states)
        kp = be.kernel_profile()
        assert kp["k_gather_vph"]["launches"] == 1 and kp["k_gather_vph"]["bytes"] == 16.0 * n * n
        assert kp["k_gather_panel"]["launches"] == 1 and kp["k_gather_panel"]["bytes"] == 16.0 * n * m
        n64, m64 = -(-n // 64) * 64, -(-m // 64) * 64
        assert kp["k_build_tall"]["bytes"] == 8.0 * (n * n + n * m) + 8.0 * 10 * (n64 * (n64 + 1) / 2 + m64 * n64)
        assert kp["k_sigma_contract"]["launches"] == 1
        assert all(v["ms"] > 0 for v in kp.values())
        again = be.kernel_profile()
        assert all(v["launches"] == 0 and v["ms"] == 0 for v in again.values())


def test_state_bound_load_complex_forms_and_shards():
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.synthetic import make_input

    inp = make_input(22, 4, seed=11)
    states = [3, 4, 9]
    om, w = generate_transformed_legendre_grid(16)
    with B200Backend(0) as full, B200Backend(0) as bound:
        full.load_system(inp)
        bound.load_system(inp, states)
        qa, _ = full.screened_forms_complex(om, states, eta=1e-3)
        qb, _ = bound.screened_forms_complex(om, states, eta=1e-3)
        np.testing.assert_array_equal(qa, qb)
        pa, _ = full.sigma_c_shard(om, w, 3, 11, states)
        pb, _ = bound.sigma_c_shard(om, w, 3, 11, states)
        np.testing.assert_array_equal(pa, pb)


def test_state_bound_load_rejects_another_state_list():
    from minigw_b200 import B200Backend, GwB200Error
    from minigw_b200.synthetic import make_input

    inp = make_input(16, 3, seed=5)
    with B200Backend(0) as be:
        be.load_system(inp, [2, 3])
        with pytest.raises(GwB200Error) as e:
            be.run_g0w0(8, 4, [3, 2])
        assert e.value.status == "GWB200_BAD_ARGUMENT"
        with pytest.raises(GwB200Error) as e:
            be.load_system(inp, [2, 2])
        assert e.value.status == "GWB200_BAD_SHAPE"
        be.load_system(inp)  # the full block again: any state list
        r = be.run_g0w0(8, 4, [3, 2])
        assert np.isfinite(r["sigma"][2]).all()


def test_batch_of_state_bound_members():
    from minigw_b200 import B200Backend, run_g0w0_batch
    from minigw_b200.synthetic import make_input

    specs = [(12, 2), (26, 4), (20, 3)]
    inputs = [make_input(nmo, nocc, seed=800 + i) for i, (nmo, nocc) in enumerate(specs)]
    states = [[inp.nocc - 1, inp.nocc] for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp, st in zip(bes, inputs, states):
            be.load_system(inp, st)
        alone = [be.run_g0w0(16, 8, st, precision="mixed") for be, st in zip(bes, states)]
        got = run_g0w0_batch(bes, 16, 8, states)
        for a, s in zip(alone, got["sigma"]):
            np.testing.assert_array_equal(s, a["sigma"])
    finally:
        for be in bes:
            be.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed-refined"])
def test_sliced_load_is_bit_identical(precision):
    """gwb200_load_system_slices (the caller cuts V_ph, the panel rows and the exchange diagonal)
    against gwb200_load_system_states on the full ERI: same resident data, same results."""
    from minigw_b200 import B200Backend
    from minigw_b200.gw_input import slices_from_input
    from minigw_b200.synthetic import make_input

    inp = make_input(34, 6, seed=41)
    states = [4, 5, 6, 7]
    sl = slices_from_input(inp, states)
    with B200Backend(0) as full, B200Backend(0) as cut:
        full.load_system(inp, states)
        cut.load_slices(sl)
        va, pa = full.read_resident(states)
        vb, pb = cut.read_resident(states)
        np.testing.assert_array_equal(va, vb)
        np.testing.assert_array_equal(pa, pb)
        a = full.run_g0w0(20, 10, states, precision=precision)
        b = cut.run_g0w0(20, 10, states, precision=precision)
    np.testing.assert_array_equal(a["sigma"], b["sigma"])
    np.testing.assert_array_equal(a["sigma_x_diag"], b["sigma_x_diag"])
    np.testing.assert_array_equal(a["qp"][states], b["qp"][states])


def test_slice_generator_matches_full_generator():
    """make_slices_on_device (from the factors, no nmo^4 ERI) against slices of make_input's ERI:
    the same recipe and draws, equal up to the rounding of the sums over K."""
    from minigw_b200.gw_input import slices_from_input
    from minigw_b200.synthetic import make_input, make_slices_on_device

    states = [5, 6, 7]
    a = slices_from_input(make_input(30, 6, seed=9), states)
    b = make_slices_on_device(30, 6, states, seed=9)
    np.testing.assert_array_equal(a.mo_energy, b.mo_energy)
    np.testing.assert_array_equal(a.vxc_diag, b.vxc_diag)
    assert a.fermi_energy == b.fermi_energy
    for k in ("vph", "panel", "xdiag"):
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= 1e-13 * np.abs(x).max(), k
    np.testing.assert_array_equal(b.vph, b.vph.T)
