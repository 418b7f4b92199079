"""The N > 1 path of bench.py: replicas on contiguous voltage blocks, max-over-ranks timing
and the sum of converged points, run as two gloo ranks on CPU (no GPU). Each rank solves
its own block of a small sweep with the CPU oracle (continuation inside the block, a fresh
start at its first voltage), as a GPU replica does with the B200 solver."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

SWEEP = [-0.4, -0.3, -0.2, -0.1, 0.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _solve_block(volts):
    """IV points of a 3 x 2 helix at `volts` with the oracle: (converged flags, currents)."""
    import time

    import oracle_py
    m = oracle_py.Helix(3, 2, 0.5, 0.7, 1.0, 0.0, 1.0, 0.05, 0.3, 0.6, 0.4, 0.5, 300.0, 0.1, -4.0, 0.05, 160)
    s = oracle_py.Solver(m, alpha_mix=0.5, nhist=8, tolf=1e-7, maxscf=400, single_history=0)
    conv, J, ok = [], [], False
    t0 = time.perf_counter()
    for k, V in enumerate(volts):
        r = s.solve_scf(V, k == 0 or not ok)
        ok = r["converged"]
        conv.append(ok)
        J.append(s.current(V))
    s.close()
    return conv, J, time.perf_counter() - t0


def _rank(rank, world, port, out):
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="1")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    block = bench.voltage_block(rank, world, SWEEP)
    conv, J, wall = _solve_block(block)
    res = bench.reduce_replicas(wall, wall, sum(conv))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, block, conv, J, wall, res))


def test_two_gloo_replicas_solve_their_blocks_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    blocks = [g[1] for g in got]
    assert blocks[0] + blocks[1] == SWEEP  # contiguous, disjoint, complete
    n_conv = sum(sum(g[2]) for g in got)
    assert n_conv == len(SWEEP)
    for _, _, _, _, _, (dev_s, wall, total) in got:
        assert total == n_conv  # converged points summed over ranks
        assert dev_s == max(g[4] for g in got)  # max over ranks
    # each replica's points are those of the same block solved alone (fresh at the block's
    # start): the same converged flags and, where converged, the same currents to the SCF
    # tolerance (thread counts differ, so the paths differ by rounding)
    for _, block, conv, J, _, _ in got:
        conv1, J1, _ = _solve_block(block)
        assert conv == conv1
        for c, a, b in zip(conv, J, J1):
            if c:
                assert np.allclose(a, b, rtol=1e-5, atol=1e-9)
