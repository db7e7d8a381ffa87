"""The N > 1 host logic of bench.py on two CPU ranks (gloo, 127.0.0.1).

With several GPUs each rank evaluates its own frame: frames are independent,
so there is no data-path collective. The only cross-rank steps are the
barriers around the timed region and the max of the step times. These tests
run those steps as two gloo processes and check:
* every rank sees the slowest rank's time;
* whole-job throughput counts every rank's atoms;
* the ranks' frames differ but have the same size (weak scaling);
* the reference arm's rank 1 leaves without work.
"""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cpu")
        step_ms = [0.80, 0.95][rank]          # rank 1 is the slow one
        dist.barrier()
        ms = bench.max_over_ranks(step_ms, world, dev)
        e2e = bench.max_over_ranks(1.0 + rank, world, dev)
        value = bench.whole_job_us_per_atom(ms, 12288, world)
        dist.barrier()
        out.put((rank, ms, e2e, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, e2e, value in res:
        assert ms == pytest.approx(0.95)       # the slowest rank's step time
        assert e2e == pytest.approx(2.0)
        # 2 x 12,288 atoms per 0.95 ms step
        assert value == pytest.approx(0.95e3 / (12288 * 2))


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(1.25, 1, None) == 1.25
    assert bench.whole_job_us_per_atom(0.9, 12288, 1) == pytest.approx(0.9e3 / 12288)


def test_rank_frames_are_independent_and_equal_sized(dpb):
    import importlib

    sys.path.insert(0, ROOT)
    import bench

    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    c0, t0, b0 = wl.water_frame(4, seed=bench.frame_seed(0))
    c1, t1, b1 = wl.water_frame(4, seed=bench.frame_seed(1))
    assert c0.shape == c1.shape and (t0 == t1).all() and (b0 == b1).all()
    assert not (c0 == c1).all()


def test_reference_arm_other_ranks_exit_without_work():
    sys.path.insert(0, ROOT)
    import bench

    # rank 1 of the reference arm returns before touching the package or the
    # reference library (rank 0 alone times and prints the CPU reference)
    assert bench.run_reference(None, 1, 2) is None
