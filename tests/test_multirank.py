"""Host logic of the multi-GPU (replicas-only) bench on CPU ranks over gloo.

bench.py --gpus N runs one independent solve per rank and reports the max over
ranks; no collective touches the data path.  Here two gloo ranks check the
max-over-ranks reduction the bench uses.
"""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK="0")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    assert bench._dist() == (world, rank, 0)
    v = bench.max_over_ranks(10.0 + rank)
    out[rank] = v
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        assert dict(out) == {0: 11.0, 1: 11.0}


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
