"""Multi-rank logic on CPU (gloo, world size 2): source sharding covers every
source exactly once with balanced cost, and the all-reduce of the per-rank
spectrum-weighted FP64 detector arrays ([phase][pix], one per source, from
the CPU oracle on fields of two lengths) equals the single-process sum."""

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


def _sources():
    """Energies on fields of two lengths (the batched-config shape, scaled
    down): per source its case, energy, spectrum weight and cost N * steps."""
    from rave_sim_b200 import workloads

    out = []
    for case, energies, weights in workloads.batched_energies(
            count=6, log_min=10, log_max=11, window=float(1 << 11) * 20e-9, nr_steps=2, phase_steps=3):
        for e, w in zip(energies, weights):
            out.append((case, float(e), float(w)))
    return out


def _detector(case, energy):
    """One source's FP64 detector array [phase][pix] from the CPU oracle."""
    from oracle import bigwave_np as bw
    from rave_sim_b200 import workloads

    return bw.run_simulation(dict(case, energy=energy, db=workloads.db_table(energy)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        src = _sources()
        costs = [float(c["sim_params"]["N"]) for c, _, _ in src]
        mine = shard_sources(costs, world)[rank]
        acc = None
        for i in mine:
            case, e, w = src[i]
            d = torch.from_numpy(w * _detector(case, e))
            acc = d if acc is None else acc + d
        if acc is None:
            acc = torch.zeros_like(torch.from_numpy(_detector(*src[0][:2])))
        reduce_detector(acc)
        q.put((rank, sorted(mine), acc.numpy()))
    finally:
        dist.destroy_process_group()


def test_detector_allreduce_gloo_world2():
    src = _sources()
    assert len({int(c["sim_params"]["N"]) for c, _, _ in src}) == 2
    ref = sum(w * _detector(c, e) for c, e, w in src)
    assert ref.ndim == 2 and ref.shape[0] == 3 and ref.max() > 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, mine, acc = q.get(timeout=300)
        res[r] = (mine, acc)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][0] + res[1][0]) == list(range(len(src)))  # every source once
    assert res[0][0] and res[1][0]
    for r in range(2):
        np.testing.assert_allclose(res[r][1], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
