"""Instance sharding across ranks (the multi-GPU path) on CPU: world-size-2
gloo process groups, with the oracle standing in for each rank's GPU engine.
The gathered atoms must equal a single-process decomposition of all epochs."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_decompose(variant, epochs, fs, eps, iterations, pct, smin, smax, fmax):
    from oracle import oracle as O

    out = []
    for e in epochs:
        r = O.decompose(variant, fs, e.T.astype(np.float64), eps, iterations, pct, smin, smax, fmax)
        out.append((r.atoms, r.natoms))
    return out


def make_epochs():
    from empi_b200 import synth

    rng = np.random.default_rng(3)
    shapes = [(300, 1), (700, 2), (450, 1), (520, 3), (256, 2)]
    return [np.stack([synth.smp_channel(rng, n, 128.0, 4, 10.0) for _ in range(c)], 1).astype(np.float32)
            for n, c in shapes]


def _worker(rank, world, port, variant, queue):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from empi_b200 import shard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        epochs = make_epochs()
        costs = [float(e.shape[0] * e.shape[1]) for e in epochs]
        res = shard.decompose_sharded(variant, epochs, 128.0, 0.02, 6, 99.0, group=None,
                                      decompose_fn=oracle_decompose, costs=costs)
        if rank == 0:
            queue.put([(a.tolist(), n.tolist()) for a, n in res])
    finally:
        dist.barrier()
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("variant", ["smp", "mmp3"])
def test_sharded_decomposition_matches_single_process(variant):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, variant, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = queue.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = oracle_decompose(variant, make_epochs(), 128.0, 0.02, 6, 99.0, 0.0, float("inf"), float("inf"))
    assert len(got) == len(want)
    for (ga, gn), (wa, wn) in zip(got, want):
        assert gn == wn.tolist()
        np.testing.assert_array_equal(np.array(ga), wa)


def test_partition_is_balanced_and_complete():
    from empi_b200.shard import partition

    costs = [5.0, 1.0, 4.0, 3.0, 3.0, 2.0, 8.0]
    parts = partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert partition([1.0], 4) == [[0], [], [], []]
