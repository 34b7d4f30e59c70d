"""Multi-rank host logic of bench.py on CPU: two gloo ranks, the job time is the max over ranks and every rank
takes the same collective steps (barrier, all-reduce) in the same order."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ws, r, local = bench.dist_env()
    assert (ws, r, local) == (world, rank, rank)
    bench.barrier(ws)
    t = bench.reduce_max(1.0 + rank * 0.5, ws)
    bench.barrier(ws)
    out.put((rank, t))
    dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 1.5), (1, 1.5)]


def test_algorithmic_bytes_formula():
    import bench
    # 2D FP64: nb*(4 + 3*8 + 1) + N*64
    assert bench.algorithmic_bytes(81200, 2251924, 2, "fp64") == 2251924 * 29 + 81200 * 64
    assert bench.algorithmic_bytes(10, 100, 3, "mixed") == 100 * (4 + 24 + 1) + 10 * 96


def test_roofline_traffic_is_the_tuned_variants_capture():
    """roofline.traffic comes from the committed ncu summary line of the very variant the autotuner picked; a variant
    without a captured line reports none rather than another variant's bytes."""
    import bench
    assert bench.read_traffic("slab", "mixed", 8) == 1.477e9
    assert bench.read_traffic("slab", "fp64", 13) == 2.594e9
    assert bench.read_traffic("plate", "mixed", 5) == 43007000.0
    assert bench.read_traffic("slab", "mixed", 3) is None
    assert bench.read_traffic("slab", "fp64", 99) is None
