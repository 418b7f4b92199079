"""The N > 1 path of bench.py: replicas on contiguous voltage blocks, max-over-ranks timing
and the sum of converged points, run as two gloo ranks on CPU (no GPU)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    block = bench.voltage_block(rank, world)
    # stand-in per-rank results: device seconds, wall seconds, converged points
    dev_s, wall, n_conv = 1.0 + rank, 2.0 + 3 * rank, len(block)
    res = bench.reduce_replicas(dev_s, wall, n_conv)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, block, res))


def test_two_gloo_replicas_partition_the_sweep_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    import bench
    blocks = [g[1] for g in got]
    assert blocks[0] + blocks[1] == bench.VOLTS  # contiguous, disjoint, complete
    for _, _, (dev_s, wall, n_conv) in got:
        assert dev_s == 2.0 and wall == 5.0 and n_conv == len(bench.VOLTS)
