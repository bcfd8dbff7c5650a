"""The serving loop (gwb200_server_*): continuous admission, concurrent slots, and results that
are identical whether a request runs alone or in a mix of concurrent requests."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from minigw_b200.synthetic import make_input

    specs = [(12, 2, [1, 2], 24), (24, 5, [4], 40), (30, 5, [3, 4, 5, 6], 32), (18, 3, [2, 3], 17),
             (40, 7, [6, 7], 48), (16, 3, list(range(16)), 20)]
    return [(make_input(nmo, nocc, seed=100 + i), nf, states) for i, (nmo, nocc, states, nf) in enumerate(specs)]


def test_results_identical_alone_and_in_mix():
    from minigw_b200 import B200Server

    reqs = _requests()
    with B200Server(0, slots=1, hbm_budget_bytes=8 << 30) as alone:
        ref = [alone.wait(alone.submit(inp, nf, 12, st)) for inp, nf, st in reqs]
    with B200Server(0, slots=3, hbm_budget_bytes=12 << 30) as mix:
        tickets = [mix.submit(inp, nf, 12, st) for inp, nf, st in reqs]
        got = [mix.wait(t) for t in tickets]
    for a, b, (inp, nf, st) in zip(ref, got, reqs):
        np.testing.assert_array_equal(a["sigma"], b["sigma"])
        np.testing.assert_array_equal(a["qp"][st], b["qp"][st])
        np.testing.assert_array_equal(a["sigma_x_diag"], b["sigma_x_diag"])
        assert b["service_ms"] > 0 and b["queue_ms"] >= 0


def test_server_matches_backend_and_rejects_oversize():
    from minigw_b200 import B200Backend, B200Server, GwB200Error
    from minigw_b200.synthetic import make_input

    inp = make_input(20, 4, seed=3)
    with B200Backend(0) as be:
        be.load_system(inp)
        ref = be.run_g0w0(32, 12, [3, 4])
    with B200Server(0, slots=2, hbm_budget_bytes=2 << 30) as srv:
        r = srv.wait(srv.submit(inp, 32, 12, [3, 4]))
        np.testing.assert_array_equal(r["sigma"], ref["sigma"])
        big = make_input(60, 10, seed=4)  # V_ph alone is 2 MB > the 1 MB slot below
        with B200Server(0, slots=1, hbm_budget_bytes=1 << 20) as tiny:
            with pytest.raises(GwB200Error) as e:
                tiny.submit(big, 16, 8, [9])
            assert e.value.status == "GWB200_OOM"


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed-refined"])
def test_merged_requests_identical_to_alone(precision):
    """Requests that wait while the worker is busy are merged into one gwb200_run_g0w0_batch; each
    result is bit-identical to the same request solved alone (merging off), and a request that
    cannot share launches (eta != 0, the complex symmetric path) runs alone in between."""
    from minigw_b200 import B200Server

    reqs = _requests()
    with B200Server(0, slots=1, hbm_budget_bytes=8 << 30, merge=1) as alone:
        ref = [alone.wait(alone.submit(inp, nf, 12, st, precision=precision)) for inp, nf, st in reqs]
        odd = reqs[2]
        ref_odd = alone.wait(alone.submit(odd[0], odd[1], 12, odd[2], eta=0.01))
        assert alone.counters()["merged_requests"] == 0
    with B200Server(0, slots=1, hbm_budget_bytes=8 << 30, merge=8) as srv:
        tickets = [srv.submit(inp, nf, 12, st, precision=precision) for inp, nf, st in reqs[:3]]
        t_odd = srv.submit(odd[0], odd[1], 12, odd[2], eta=0.01)
        tickets += [srv.submit(inp, nf, 12, st, precision=precision) for inp, nf, st in reqs[3:]]
        got = [srv.wait(t) for t in tickets]
        got_odd = srv.wait(t_odd)
        counters = srv.counters()
    assert counters["merged_batches"] >= 1 and counters["merged_requests"] >= 2, counters
    for a, b, (inp, nf, st) in zip(ref, got, reqs):
        np.testing.assert_array_equal(a["sigma"], b["sigma"])
        np.testing.assert_array_equal(a["qp"][st], b["qp"][st])
        np.testing.assert_array_equal(a["sigma_x_diag"], b["sigma_x_diag"])
        np.testing.assert_array_equal(a["omegas"], b["omegas"])
        np.testing.assert_array_equal(a["weights"], b["weights"])
    np.testing.assert_array_equal(ref_odd["sigma"], got_odd["sigma"])


def test_sliced_requests():
    """A request whose system arrives as slices (no ERI) gives the backend's own result."""
    from minigw_b200 import B200Backend, B200Server
    from minigw_b200.gw_input import slices_from_input
    from minigw_b200.synthetic import make_input

    inp = make_input(26, 4, seed=12)
    states = [3, 4, 5]
    sl = slices_from_input(inp, states)
    with B200Backend(0) as be:
        be.load_system(inp, states)
        ref = be.run_g0w0(30, 12, states)
    with B200Server(0, slots=2, hbm_budget_bytes=4 << 30) as srv:
        ts = [srv.submit(sl, 30, 12, states), srv.submit(inp, 30, 12, states), srv.submit(sl, 30, 12, states)]
        out = [srv.wait(t) for t in ts]
    for r in out:
        np.testing.assert_array_equal(r["sigma"], ref["sigma"])
        np.testing.assert_array_equal(r["qp"][states], ref["qp"][states])
        np.testing.assert_array_equal(r["sigma_x_diag"], ref["sigma_x_diag"])
