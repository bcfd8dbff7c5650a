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
