"""The N > 1 path of bench.py on the CPU: two gloo ranks (one per process, as torchrun launches them) take the
same collective steps, agree on the slowest rank's time, and report every rank's units over it; the reference
arm leaves ranks other than 0 without work.  No GPU involved (the GPU run uses the same helpers over NCCL)."""
import datetime
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        bench.barrier(world)
        ms = 100.0 + 50.0 * rank                       # this rank's device time for its 320 units
        rate, worst = bench.job_rate(320, ms, world)
        bench.barrier(world)

        class Args:
            steps, warmup, gpus = 1, 0, world
        ran = bench.run_reference(Args, world, rank) if rank != 0 else None   # rank 0 would time the port
        q.put((rank, rate, worst, ran))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_job_over_the_slowest_rank():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, rate, worst, ran in got:
        assert worst == 150.0                          # both ranks see the slowest rank's time
        assert abs(rate - 2 * 320 / 0.150) < 1e-6      # every rank's units over it
        assert ran is None
    assert [g[0] for g in got] == [0, 1]


def test_one_rank_is_its_own_job():
    import bench
    rate, worst = bench.job_rate(64 * 20, 227.5, 1)
    assert worst == 227.5 and abs(rate - 64 * 20 / 0.2275) < 1e-6
