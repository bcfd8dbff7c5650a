"""Multi-rank path: frequency sharding of one solve with an all-reduce of the partial Sigma_c.

CPU: world_size-2 gloo ranks (spawned processes) run minigw_b200.sharding with per-shard partial
sums computed from the oracle's screened forms; the reduced Sigma_c equals the oracle's full one.
GPU (one device): the shards' partial sums from gwb200_sigma_c_shard add up to gwb200_sigma_c.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def test_shard_bounds_partition():
    from minigw_b200.sharding import shard_bounds

    for nfreq in (1, 7, 64, 128, 200):
        for world in (1, 2, 3, 8):
            bounds = [shard_bounds(nfreq, world, r) for r in range(world)]
            assert bounds[0][0] == 0 and bounds[-1][1] == nfreq
            for (b0, e0), (b1, _) in zip(bounds, bounds[1:]):
                assert e0 == b1
            sizes = [e - b for b, e in bounds]
            assert max(sizes) - min(sizes) <= 1


def _partial_from_forms(q, inp, omegas, weights, states, b, e):
    """-(1/pi) sum over f' in [b, e) and k of w g q (src/gw/sigma_c_driver.cpp:154-168), all f_n."""
    nmo = inp.nmo
    out = np.zeros((nmo, len(omegas)), dtype=np.complex128)
    for s_i, p in enumerate(states):
        for fn, wn in enumerate(omegas):
            a = 1j * wn + inp.fermi_energy - inp.mo_energy
            acc = 0.0j
            for fp in range(b, e):
                g = a / (a * a + omegas[fp] ** 2)
                acc += np.sum(-weights[fp] * g * q[fp, s_i, :].real)
            out[p, fn] = acc / np.pi
    return out


def _rank_main(rank, world, port, result_path):
    import sys

    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import oracle
    from minigw_b200.sharding import sharded_sigma_c, torch_allreduce_sum
    from minigw_b200.synthetic import make_input

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = oracle.Oracle()
        inp = make_input(9, 3, seed=4)
        om, w = o.grid(11)
        states = [1, 2, 5]
        q = o.screened_forms(inp, om, states)
        full = sharded_sigma_c(lambda b, e: _partial_from_forms(q, inp, om, w, states, b, e), len(om), world, rank,
                               torch_allreduce_sum())
        if rank == 0:
            ref = o.sigma_from_forms(inp, om, w, states, q)
            np.save(result_path, np.array([np.abs(full - ref).max(), np.abs(ref).max()]))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_reduce_to_full_sigma(tmp_path):
    import torch.multiprocessing as mp

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = tmp_path / "res.npy"
    mp.start_processes(_rank_main, args=(2, port, str(out)), nprocs=2, start_method="spawn", join=True)
    err, scale = np.load(out)
    assert scale > 0 and err <= 1e-13 * max(1.0, scale)


@pytest.mark.gpu
def test_gpu_shards_add_up_to_full_sigma():
    from minigw_b200 import B200Backend, generate_transformed_legendre_grid
    from minigw_b200.sharding import shard_bounds
    from minigw_b200.synthetic import make_input

    inp = make_input(30, 7, seed=12)
    om, w = generate_transformed_legendre_grid(23)
    states = [5, 6, 7, 8]
    with B200Backend(0) as be:
        be.load_system(inp)
        full, _ = be.sigma_c(om, w, states)
        for world in (2, 3):
            total = np.zeros_like(full)
            for r in range(world):
                b, e = shard_bounds(len(om), world, r)
                part, _ = be.sigma_c_shard(om, w, b, e, states)
                total += part
            assert np.abs(total - full).max() <= 1e-14 * max(1.0, np.abs(full).max())
        empty, _ = be.sigma_c_shard(om, w, 5, 5, states)
        assert np.all(empty == 0)
