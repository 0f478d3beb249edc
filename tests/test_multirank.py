"""Multi-rank host logic of bench.py on CPU with the gloo backend (world size 2): each rank owns its
own cameras (weak scaling, no data-path collective), and the timing is the max over ranks."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from cuvslam_b200 import synthetic
    from oracle import oracle as O

    # each rank tracks its own small camera set (seed offset = rank)
    shapes = [(160, 120), (128, 96)]
    prevs, nexts = [], []
    for i, (w, h) in enumerate(shapes):
        p, n, _ = synthetic.frame_pair(i + 100 * rank, w, h)
        prevs.append(p)
        nexts.append(n)
    step, attempted = bench.cpu_reference_step_fn(shapes, [60, 60], prevs, nexts, 1)
    out = step()
    local_ms = 10.0 + rank  # stand-in elapsed times: the slowest rank (rank 1) must win
    ms = bench.reduce_max(local_ms, dist, "cpu")
    total = bench.reduce_sum(attempted, dist, "cpu")
    value = bench.throughput(total, 5, ms)
    checksum = float(sum(a.sum() for a in out[0]))
    q.put((rank, attempted, ms, value, checksum, int(prevs[0].sum()), total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, ms0, v0, c0, s0, t0), (r1, a1, ms1, v1, c1, s1, t1) = res
    assert ms0 == ms1 == 11.0  # max over ranks
    assert t0 == t1 == a0 + a1  # units of all ranks
    assert s0 != s1  # different cameras per rank
    assert v0 == v1 == (a0 + a1) * 5 / 0.011
    assert np.isfinite(c0) and np.isfinite(c1)
