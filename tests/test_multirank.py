"""Multi-GPU form of the bench on CPU: world_size 2 with the gloo backend.  Each rank
builds its own replica workload (different instances), no data-path collective, and
the final reduction sums the solve counts and takes the max time over ranks."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    probs, pidx, ics = bench.make_workload(rank, 2, 3)
    first = int(np.abs(probs[0][0][:3]).sum())
    sums, tmax = bench.reduce_over_ranks(dist, [10 * (rank + 1), first], 1.5 + rank, "cpu")
    out[rank] = (sums.tolist(), tmax, first, len(pidx), ics.shape)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_reduce():
    port = _free_port()
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    r0, r1 = out[0], out[1]
    assert r0[0][0] == r1[0][0] == 30.0                  # summed solve counts
    assert r0[1] == r1[1] == 2.5                         # max time over ranks
    assert r0[2] != r1[2]                                # different instances per rank
    assert r0[3] == r1[3] == 6 and r0[4] == r1[4] == (6, 1000 + 4250)
