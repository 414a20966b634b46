"""The N-rank bench path on CPU: two gloo ranks (127.0.0.1) run the
aggregation the bench runs over NCCL — a barrier, the maximum of every
rank's timing scalars, the whole-job rate over the slowest rank — and the
replica sharding (each rank seeds its own frames)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oxideav-vp8_b200"))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        dist.barrier()
        # Rank r's timings: the device step, e2e, e2e per call.
        mine = [10.0 + 5 * rank, 12.0 - rank, 20.0 + rank]
        got = bench.max_over_ranks(mine, dist, torch.device("cpu"))
        rate = bench.whole_job_rate(bench.N_MB, 3, world, got[0])
        # Replica sharding: the rank's own seeded inputs (small frames).
        from vp8a import synth

        frames, _ = synth.make_sequence(64, 48, 3, bench.SEED + rank)
        out.put((rank, got, rate, synth.digest(frames)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_own_inputs():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, g0, rate0, d0), (r1, g1, rate1, d1) = res
    assert g0 == g1 == [15.0, 12.0, 21.0]
    assert rate0 == rate1 == pytest.approx(8160 * 3 * 2 / 0.015)
    assert d0 != d1
