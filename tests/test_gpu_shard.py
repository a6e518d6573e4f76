"""Instance sharding with the real engine: decompose_sharded at world size 1
(a gloo process group in this process) on the GPU gives the atoms of one
batch of all epochs; the multi-rank partition and gather are covered on CPU
(tests/test_shard.py, world size 2)."""
import datetime
import socket

import numpy as np
import pytest

import empi_b200
from empi_b200 import shard

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_decompose_sharded_world_size_1_real_engine(engine):
    import torch.distributed as dist
    from test_shard import make_epochs

    epochs = make_epochs()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = shard.decompose_sharded("smp", epochs, 128.0, 0.01, 8, 99.0, engine=engine)
    finally:
        dist.destroy_process_group()
    ref = empi_b200.decompose_epochs("smp", epochs, 128.0, 0.01, 8, 99.0, engine=engine)
    assert len(got) == len(ref) == len(epochs)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g.counts, r.counts)
        np.testing.assert_array_equal(g.indices, r.indices)
        np.testing.assert_allclose(g.atoms, r.atoms, rtol=1e-12, atol=0)
