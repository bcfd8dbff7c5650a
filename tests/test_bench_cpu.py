"""bench.py's host-side pieces that run without a GPU: the reference CPU baseline of the
uneven-molecule batch (the reference's own code on a size-spread sample, interpolated)."""
from __future__ import annotations

import types

import numpy as np
import pytest


def test_reference_arm_runs_only_the_reference():
    """`bench.py --impl reference` maps the reference's compiled code and not libgwb200.so, takes the
    grid from the reference, and prints the config dict the b200 arm prints for the same command."""
    import json
    import subprocess
    import sys

    import oracle
    from conftest import ROOT

    if not oracle.Ref.available:
        pytest.skip("oracle/_ref was not built (reference tree absent)")
    code = ("import sys; sys.argv=['bench.py','--impl','reference','--workload','cfg1','--steps','1','--warmup','1',"
            "'--cpu-pairs','4']; import bench; bench.main(); maps=open('/proc/self/maps').read(); "
            "print('MAPS', 'libgwb200' in maps, 'libgwref' in maps)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "MAPS False True"
    out = json.loads(lines[-2])
    import bench
    from minigw_b200.synthetic import WORKLOADS

    args = types.SimpleNamespace(precision="fp64", split_frequencies=False)
    assert out["impl"] == "reference" and out["config"] == bench.workload_config(args, WORKLOADS["cfg1"], 1)
    assert out["cpu_baseline"]["kind"] == "reference" and out["cpu_baseline"]["cpu_model"]
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["value"] > 0


def test_batch_cpu_baseline_samples_and_interpolates(monkeypatch):
    import bench
    import minigw_b200.synthetic as syn
    import oracle

    if not oracle.Ref.available:
        pytest.skip("oracle/_ref was not built (reference tree absent)")
    # host generator in place of the GPU one (same recipe and draws)
    monkeypatch.setattr(syn, "make_input_on_device",
                        lambda nmo, nocc, seed=0, device=0, pin=True: syn.make_input(nmo, nocc, seed))
    calls = []
    real = bench.cpu_reference_sample

    def spy(inp, wl, om, w, pairs, threads):
        out = real(inp, wl, om, w, pairs, threads)
        calls.append((wl.nph, out["seconds_per_pair"]))
        return out

    monkeypatch.setattr(bench, "cpu_reference_sample", spy)
    nmos = [20, 26, 31, 38, 24, 44]
    cb = bench.batch_cpu_baseline(types.SimpleNamespace(seed=0), nmos, 16, 8, sample=3)
    nph = sorted(round(n / 6) * (n - round(n / 6)) for n in nmos)
    sampled = sorted(n for n, _ in calls)
    assert sampled[0] == nph[0] and sampled[-1] == nph[-1] and len(calls) == 3
    per_pair_max = max(t for _, t in calls)
    # 6 solves, each 16^2 pairs no longer than the slowest sampled pair
    assert cb["kind"] == "reference" and cb["unit"] == "GW solves/s"
    assert cb["value"] >= 6 / (6 * 16 ** 2 * per_pair_max) * (1 - 1e-9)
    assert np.isfinite(cb["value"]) and cb["cores"] >= 1
