"""Batched solves of molecules of uneven size (gwb200_run_g0w0_batch): the bucket planner on the
CPU, and on the GPU each molecule's result against its own gwb200_run_g0w0."""
from __future__ import annotations

import itertools

import numpy as np
import pytest


def _model_cost(sizes, n_sorted, m_sorted, nfreq, step_us, tflops):
    """The planner's cost model with every bucket in one chunk (budget large)."""
    cost, pos = 0.0, 0
    for b in sizes:
        n = max(n_sorted[pos:pos + b])
        m = max(m_sorted[pos:pos + b])
        N = (n + 63) // 64 * 64
        M = (m + 63) // 64 * 64
        cost += (N // 64) * step_us * 1e-6 + b * nfreq * (N ** 3 / 3 + N * N * M) / (tflops * 1e12)
        pos += b
    return cost


def _sizes_from(bucket_of, order):
    seq = [int(bucket_of[i]) for i in order]
    return [len(list(g)) for _, g in itertools.groupby(seq)]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_planner_matches_exhaustive_search(seed):
    from minigw_b200 import plan_buckets

    rng = np.random.default_rng(seed)
    k, nfreq, step_us, tflops = 8, 64, 60.0, 90.0
    nmo = rng.integers(20, 161, size=k)
    nocc = np.rint(nmo / 6).astype(np.int64)
    nph = nocc * (nmo - nocc)
    ncols = 2 * nmo
    bucket_of, nb = plan_buckets(nph, ncols, nfreq, "mixed", 1 << 50, step_us, tflops)
    order = sorted(range(k), key=lambda i: (nph[i], ncols[i], i))
    # buckets are contiguous runs of the size order, numbered in ascending size
    seq = [int(bucket_of[i]) for i in order]
    assert seq == sorted(seq) and seq[0] == 0 and seq[-1] == nb - 1
    n_sorted = [int(nph[i]) for i in order]
    m_sorted = [int(ncols[i]) for i in order]
    got = _model_cost(_sizes_from(bucket_of, order), n_sorted, m_sorted, nfreq, step_us, tflops)
    best = min(
        _model_cost([b - a for a, b in zip((0,) + cuts, cuts + (k,))], n_sorted, m_sorted, nfreq, step_us, tflops)
        for r in range(k) for cuts in itertools.combinations(range(1, k), r))
    assert got == pytest.approx(best, rel=1e-12)


def test_planner_extremes():
    from minigw_b200 import plan_buckets

    nph = np.array([50, 300, 700, 1500, 3500])
    ncols = np.array([40, 80, 120, 200, 320])
    # launch latency dominant: one bucket; padding dominant: one bucket per padded geometry
    _, nb = plan_buckets(nph, ncols, 64, "mixed", 1 << 50, 1e9, 90.0)
    assert nb == 1
    b, nb = plan_buckets(nph, ncols, 64, "mixed", 1 << 50, 1e-9, 90.0)
    assert nb == 5 and sorted(b.tolist()) == [0, 1, 2, 3, 4]


def test_planner_rejects_bad_input():
    from minigw_b200 import GwB200Error, plan_buckets

    with pytest.raises(GwB200Error):
        plan_buckets([10, 0], [4, 4], 16)
    with pytest.raises(GwB200Error):
        plan_buckets([10], [4], 0)


# ---- GPU ----

_SPECS = [(12, 2), (18, 3), (24, 4), (30, 5), (40, 7), (48, 8), (20, 3)]


def _systems(specs=_SPECS, seed0=300):
    from minigw_b200.synthetic import make_input

    return [make_input(nmo, nocc, seed=seed0 + i) for i, (nmo, nocc) in enumerate(specs)]


def _states(inp):
    return [inp.nocc - 1, inp.nocc]  # HOMO and LUMO


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_matches_each_molecule_alone(precision, monkeypatch):
    from minigw_b200 import B200Backend, run_g0w0_batch

    if precision == "fp64":  # the same update kernel for every geometry, so the bits can match
        monkeypatch.setenv("GWB200_FP64_UPDATE", "dmma")
        monkeypatch.setenv("GWB200_UPDATE_VARIANT", "0")
    inputs = _systems()
    nfreq, npade = 24, 12
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp in zip(bes, inputs):
            be.load_system(inp)
        alone = [be.run_g0w0(nfreq, npade, _states(inp), precision=precision) for be, inp in zip(bes, inputs)]
        got = run_g0w0_batch(bes, nfreq, npade, [_states(inp) for inp in inputs], precision=precision)
        assert 1 <= got["buckets"] <= len(inputs)
        for a, s, q, inp in zip(alone, got["sigma"], got["qp"], inputs):
            st = _states(inp)
            np.testing.assert_array_equal(s, a["sigma"])
            np.testing.assert_array_equal(q[st], a["qp"][st])
            assert np.isnan(np.delete(q, st)).all()
        # the cached plan on a second call gives the same numbers
        again = run_g0w0_batch(bes, nfreq, npade, [_states(inp) for inp in inputs], precision=precision)
        for s0, s1 in zip(got["sigma"], again["sigma"]):
            np.testing.assert_array_equal(s0, s1)
        assert again["stats"]["flops_screening"] == got["stats"]["flops_screening"] > 0
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
@pytest.mark.parametrize("plan", ["each", "single", "model", "model-3-streams", "each-4-streams-unshared"])
def test_every_bucket_plan_gives_the_same_bits(plan, monkeypatch):
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems(seed0=400)
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp in zip(bes, inputs):
            be.load_system(inp)
        states = [_states(inp) for inp in inputs]
        monkeypatch.setenv("GWB200_BATCH_PLAN", "each")
        ref = run_g0w0_batch(bes, 16, 8, states)
        assert ref["buckets"] == len(inputs)
        if "streams" in plan:  # buckets on concurrent streams with their own workspaces
            monkeypatch.setenv("GWB200_BATCH_STREAMS", plan.split("-")[1])
            monkeypatch.setenv("GWB200_BATCH_SHARE_SMS", "0" if plan.endswith("unshared") else "1")
        monkeypatch.setenv("GWB200_BATCH_PLAN", plan.split("-")[0])
        got = run_g0w0_batch(bes, 16, 8, states)
        if plan == "single":
            assert got["buckets"] == 1
        for a, b in zip(ref["sigma"], got["sigma"]):
            np.testing.assert_array_equal(a, b)
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
def test_batch_multi_chunk_and_states(monkeypatch):
    """Many states per molecule and frequencies split across chunks of one bucket."""
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems([(16, 3), (22, 4), (26, 4)], seed0=500)
    states = [list(range(inputs[0].nmo)), [1, 4, 5], [3]]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp in zip(bes, inputs):
            be.load_system(inp)
        alone = [be.run_g0w0(20, 10, st, precision="mixed") for be, st in zip(bes, states)]
        monkeypatch.setenv("GWB200_BATCH_PLAN", "single")
        monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", "7")  # 60 matrices in 9 launch sequences
        got = run_g0w0_batch(bes, 20, 10, states)
        assert got["stats"]["frequency_chunks"] == 9
        for a, s in zip(alone, got["sigma"]):
            np.testing.assert_array_equal(s, a["sigma"])
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
def test_batch_rejects_bad_members():
    from minigw_b200 import B200Backend, GwB200Error, run_g0w0_batch
    from minigw_b200.synthetic import make_input

    a, b, c = B200Backend(0), B200Backend(0), B200Backend(0)
    try:
        a.load_system(make_input(12, 2, seed=1))
        b.load_system(make_input(14, 3, seed=2))
        with pytest.raises(GwB200Error) as e:
            run_g0w0_batch([a, b, a], 8, 4, [[1], [2], [1]])
        assert e.value.status == "GWB200_BAD_ARGUMENT"
        with pytest.raises(GwB200Error) as e:
            run_g0w0_batch([a, c], 8, 4, [[1], [2]])
        assert e.value.status == "GWB200_NO_SYSTEM"
        with pytest.raises(GwB200Error) as e:
            run_g0w0_batch([a, b], 8, 4, [[1], [14]])
        assert e.value.status == "GWB200_BAD_SHAPE"
        # the handles stay usable
        r = run_g0w0_batch([a, b], 8, 4, [[1], [2]])
        assert np.isfinite(r["sigma"][0][1]).all()
    finally:
        for x in (a, b, c):
            x.close()


@pytest.mark.gpu
def test_graph_replay_matches_eager_and_follows_reloads(monkeypatch):
    """A repeated batch runs as one CUDA graph launch; replays give the eager launches' bits and
    pick up a member reloaded with another system of the same size."""
    from minigw_b200 import B200Backend, run_g0w0_batch
    from minigw_b200.synthetic import make_input

    inputs = _systems([(18, 3), (30, 5), (24, 4)], seed0=900)
    states = [_states(inp) for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp, st in zip(bes, inputs, states):
            be.load_system(inp, st)
        monkeypatch.setenv("GWB200_BATCH_PLAN", "model")
        monkeypatch.setenv("GWB200_BATCH_GRAPH", "0")
        eager = run_g0w0_batch(bes, 20, 10, states)
        monkeypatch.setenv("GWB200_BATCH_GRAPH", "1")
        for _ in range(3):  # capture, then replays
            got = run_g0w0_batch(bes, 20, 10, states)
            for a, b, qa, qb, st in zip(eager["sigma"], got["sigma"], eager["qp"], got["qp"], states):
                np.testing.assert_array_equal(a, b)
                np.testing.assert_array_equal(qa[st], qb[st])
        other = make_input(30, 5, seed=977)  # same shape as member 1, other values
        bes[1].load_system(other, states[1])
        replay = run_g0w0_batch(bes, 20, 10, states)
        monkeypatch.setenv("GWB200_BATCH_GRAPH", "0")
        fresh = run_g0w0_batch(bes, 20, 10, states)
        for a, b in zip(fresh["sigma"], replay["sigma"]):
            np.testing.assert_array_equal(a, b)
        assert not np.array_equal(fresh["sigma"][1], eager["sigma"][1])
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
def test_graph_recaptured_when_chunk_boundaries_move(monkeypatch):
    """The same plan cut into the same number of launch sequences with other boundaries (chunk cap
    20 -> 25 on 60 matrices: 20/20/20 -> 25/25/10) must not replay the old graph."""
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems([(16, 3), (22, 4), (26, 4)], seed0=1200)
    states = [_states(inp) for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp, st in zip(bes, inputs, states):
            be.load_system(inp, st)
        alone = [be.run_g0w0(20, 10, st, precision="mixed") for be, st in zip(bes, states)]
        monkeypatch.setenv("GWB200_BATCH_PLAN", "single")
        monkeypatch.setenv("GWB200_BATCH_GRAPH", "1")
        for cap in ("20", "20", "25", "25", "20"):
            monkeypatch.setenv("GWB200_MAX_FREQ_CHUNK", cap)
            got = run_g0w0_batch(bes, 20, 10, states)
            assert got["stats"]["frequency_chunks"] == 3
            for a, s, q, st in zip(alone, got["sigma"], got["qp"], states):
                np.testing.assert_array_equal(s, a["sigma"])
                np.testing.assert_array_equal(q[st], a["qp"][st])
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
def test_batch_with_per_molecule_frequency_and_pade_counts():
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems([(16, 3), (28, 5), (22, 4)], seed0=950)
    states = [_states(inp) for inp in inputs]
    nfreq, npade = [16, 24, 20], [8, 12, 10]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp in zip(bes, inputs):
            be.load_system(inp)
        alone = [be.run_g0w0(nf, npd, st, precision="mixed") for be, nf, npd, st in zip(bes, nfreq, npade, states)]
        for _ in range(2):  # eager (plan timed), then the graph
            got = run_g0w0_batch(bes, nfreq, npade, states)
            for a, s, q, st, nf in zip(alone, got["sigma"], got["qp"], states, nfreq):
                assert s.shape[1] == nf
                np.testing.assert_array_equal(s, a["sigma"])
                np.testing.assert_array_equal(q[st], a["qp"][st])
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
@pytest.mark.parametrize("plan", ["single", "each", "model"])
def test_refined_batch_bit_identical_to_alone(monkeypatch, plan):
    """The refined mixed form in a batch (each molecule's factor reversed within its own n_pad, one
    backward solve of the bucket, each molecule's FP64 correction with its own pivoted Cholesky factor
    of V): bit-identical to each molecule's own refined solve, whatever the bucketing (a single bucket
    pads the smallest molecule by three 64-blocks)."""
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems([(16, 3), (22, 4), (26, 4), (40, 7)], seed0=1300)
    states = [_states(inp) for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp, st in zip(bes, inputs, states):
            be.load_system(inp, st)
        alone = [be.run_g0w0(20, 10, st, precision="mixed-refined") for be, st in zip(bes, states)]
        monkeypatch.setenv("GWB200_BATCH_PLAN", plan)
        for _ in range(2):  # eager, then the graph replay
            got = run_g0w0_batch(bes, 20, 10, states, precision="mixed-refined")
            for a, s, q, st in zip(alone, got["sigma"], got["qp"], states):
                np.testing.assert_array_equal(s, a["sigma"])
                np.testing.assert_array_equal(q[st], a["qp"][st])
    finally:
        for be in bes:
            be.close()


@pytest.mark.gpu
def test_refined_batch_against_oracle(oracle_lib):
    """Batched refined mixed forms feed Sigma_c within 1e-10 Ha of the oracle for every molecule."""
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid, run_g0w0_batch

    inputs = _systems([(18, 3), (30, 5), (24, 4)], seed0=1400)
    states = [_states(inp) for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp in zip(bes, inputs):
            be.load_system(inp)
        got = run_g0w0_batch(bes, 24, 12, states, precision="mixed-refined")
    finally:
        for be in bes:
            be.close()
    om, w = generate_transformed_legendre_grid(24)
    for inp, st, s in zip(inputs, states, got["sigma"]):
        ref, _ = oracle_lib.sigma_c(inp, om, w, st)
        assert np.abs(s - ref).max() <= 1e-10


@pytest.mark.gpu
def test_batches_of_different_forms_on_the_same_handles():
    """Refined, plain and mixed batches in turn on the same member handles: the lead handle's lane
    workspaces are re-planned for each form (buffers one form does not use are freed before the
    next form's are allocated), and each batch stays bit-identical to the molecules' own solves."""
    from minigw_b200 import B200Backend, run_g0w0_batch

    inputs = _systems([(16, 3), (26, 4), (40, 7)], seed0=1500)
    states = [_states(inp) for inp in inputs]
    bes = [B200Backend(0) for _ in inputs]
    try:
        for be, inp, st in zip(bes, inputs, states):
            be.load_system(inp, st)
        for prec in ("mixed-refined", "fp64", "mixed", "mixed-refined", "fp64"):
            alone = [be.run_g0w0(16, 8, st, precision=prec) for be, st in zip(bes, states)]
            got = run_g0w0_batch(bes, 16, 8, states, precision=prec)
            for a, s, q, st in zip(alone, got["sigma"], got["qp"], states):
                np.testing.assert_array_equal(s, a["sigma"])
                np.testing.assert_array_equal(q[st], a["qp"][st])
    finally:
        for be in bes:
            be.close()
