"""The multi-GPU path is N independent replicas; its only cross-rank step is
the timing reduction (max time, summed work).  Two gloo ranks on the CPU
run it exactly as bench.py does under torchrun."""
import multiprocessing as mp
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist

    from sh_baker_b200.replicas import job_rate, rank_info
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, lr = rank_info()
        ms = 100.0 + 50.0 * r          # rank 1 is the slow one
        units = 1000 * (r + 1)
        q.put((r, (w, r, lr), job_rate(ms, units, dist)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(2):
        r, info, res = q.get(timeout=120)
        out[r] = (info, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        info, (ms, units, rate) = out[r]
        assert info == (2, r, r)
        assert ms == 150.0 and units == 3000
        assert rate == 3000 / 0.150


def test_single_process_passthrough():
    from sh_baker_b200.replicas import job_rate
    assert job_rate(200.0, 500) == (200.0, 500, 2500.0)
