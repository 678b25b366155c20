"""The N>1 path of bench.py (independent replicas, no data-path collective).

* Two gloo ranks on the CPU agree on the barrier, the max-over-ranks step time
  and the summed work, exactly as the NCCL ranks do on GPUs.
* `bench.py --gpus 2` started without a rank environment launches itself as
  two ranks (torch.distributed.run on 127.0.0.1) and rank 0 prints the reduced
  line: world size 2, the slower rank's time, the summed packets, and a
  distinct packet-source seed per rank.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
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
    r, w, local, pg = bench.dist_setup(world, backend="gloo")
    dev = torch.device("cpu")
    bench.barrier(pg, dev)
    t = bench.max_over_ranks(pg, 10.0 + rank, dev)
    n = bench.sum_over_ranks(pg, 100.0 * (rank + 1), dev)
    out[rank] = (r, w, t, n)
    pg.destroy_process_group()


def test_two_replicas_reduce_over_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()   # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == (0, 2, 11.0, 300.0)
    assert out[1] == (1, 2, 11.0, 300.0)


def test_bench_launches_two_ranks_itself():
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["OMP_NUM_THREADS"] = "1"
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--launcher-check"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    if p.returncode != 0:
        pytest.fail(f"launcher exited {p.returncode}:\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout                       # rank 0 alone prints
    line = lines[0]
    sys.path.insert(0, ROOT)
    import bench
    assert line["launcher_check"] and line["n_gpus"] == 2
    assert line["max_ms"] == 11.0                          # the slower rank's time
    assert line["packets"] == 300.0                        # work summed over ranks
    assert line["seed_sum"] == 2 * bench.SEED + 1          # seeds SEED, SEED + 1
