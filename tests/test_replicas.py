"""bench.py --gpus N renders N independent views (no data-path collective);
its whole-job figures come from combine_ranks: the slowest rank's device
times and the sum of the rays.  Checked here with world_size-2 gloo ranks on
the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [10.0, 12.5][rank]
    e2e = [11.0, 13.0][rank]
    rays = [1000, 3000][rank]
    q.put((rank, bench.combine_ranks(ms, e2e, rays, world, "cpu")))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_combine_to_slowest_time_and_total_rays():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r] == (12.5, 13.0, 4000.0)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_ranks(3.0, 4.0, 7, 1, None) == (3.0, 4.0, 7.0)
