"""N>1 path (replicas): max-over-ranks time and summed work, world size 2
over gloo on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from pic3d_b200.replicas import combine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [10.0, 25.0][rank]
    parts = [1000.0, 3000.0][rank]
    out[rank] = combine(ms, parts, steps=5, dist=dist, device="cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    for r in range(2):
        ms, total, rate = out[r]
        assert ms == 25.0 and total == 4000.0
        assert rate == pytest.approx(4000.0 * 5 / 0.025)


def test_single_process():
    from pic3d_b200.replicas import combine
    assert combine(2.0, 100, 4) == (2.0, 100.0, 100 * 4 / 0.002)
