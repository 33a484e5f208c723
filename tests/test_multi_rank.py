"""Multi-rank logic on CPU (gloo, world size 2): source sharding covers every
source exactly once with balanced cost, and the detector all-reduce of the
per-rank weighted sums equals the single-process sum."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from rave_sim_b200.sharding import reduce_detector, shard_sources


def test_shard_covers_and_balances():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        costs = (2.0 ** rng.integers(20, 26, size=128)) * rng.integers(30, 110, size=128)
        shards = shard_sources(costs.tolist(), world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(128))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= costs.max()  # LPT bound
    assert shard_sources([1.0, 1.0], 4)[2:] == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fake_detector(energy, n_phase=3, n_pix=5):
    # stands in for one source's detector output: smooth in energy and pixel
    p = np.arange(n_phase)[:, None]
    j = np.arange(n_pix)[None, :]
    return np.cos(energy * 1e-4 + p) * (1 + j) / energy


def _worker(rank, world, port, energies, weights, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_sources([1.0] * len(energies), world)[rank]
        acc = torch.zeros((3, 5), dtype=torch.float64)
        for i in mine:
            acc += weights[i] * torch.from_numpy(fake_detector(energies[i]))
        reduce_detector(acc)
        q.put((rank, acc.numpy()))
    finally:
        dist.destroy_process_group()


def test_detector_allreduce_gloo_world2():
    energies = np.linspace(20000.0, 70000.0, 11)
    weights = np.linspace(1.0, 2.0, 11)
    ref = sum(w * fake_detector(e) for e, w in zip(energies, weights))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, energies, weights, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        np.testing.assert_allclose(res[r], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
