"""The N>1 path of bench.py (independent replicas, no data-path collective):
two gloo ranks on the CPU agree on the barrier, the max-over-ranks step time
and the summed work, exactly as the NCCL ranks do on GPUs."""
import os
import socket
import sys

import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, pg = bench.dist_setup(world)
    dev = torch.device("cpu")
    bench.barrier(pg, dev)
    t = bench.max_over_ranks(pg, 10.0 + rank, dev)
    n = bench.sum_over_ranks(pg, 100.0 * (rank + 1), dev)
    out[rank] = (r, w, t, n)
    pg.destroy_process_group()


def test_two_replicas_reduce_over_gloo():
    if torch.cuda.is_available():
        return   # on a GPU box bench.py selects NCCL; this checks the CPU / gloo path
    world = 2
    mgr = mp.get_context("spawn").Manager()   # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == (0, 2, 11.0, 300.0)
    assert out[1] == (1, 2, 11.0, 300.0)
