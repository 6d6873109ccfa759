"""The multi-GPU bench path on CPU: world_size-2 gloo ranks (127.0.0.1)
run bench.py's rank aggregation — job throughput = all ranks' frames over
the slowest rank's time — exactly as the NCCL run does on GPUs."""
import multiprocessing as mp
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        frames = [16, 12][rank]          # frames each rank encoded
        ms = [400.0, 500.0][rank]        # each rank's device time
        q.put((rank, bench.max_over_ranks(ms, world), bench.sum_over_ranks(frames, world),
               bench.job_throughput(frames, ms, world)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_gpu_run():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, thr in res:
        assert mx == 500.0 and sm == 28.0
        assert abs(thr - 28.0 / 0.5) < 1e-9
