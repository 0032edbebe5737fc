"""bench.py's multi-process plumbing on CPU: two ranks over gloo on
127.0.0.1 take the timing maximum over ranks and pass the barriers; in the
reference arm only rank 0 works, the other returns at once without output.
(One geometry does not shard, so `bench.py --gpus N` runs N replicas with no
data-path collective; these are its only cross-rank steps.)"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    r, w, l = bench.dist_env()
    t = bench.max_over_ranks(1.5 + r, w)  # rank r "took" 1.5 + r seconds
    bench.barrier(w)

    class Args:
        config, steps, warmup = "c1", 1, 0
    if r != 0:
        bench.run_reference(Args(), r, w)  # must return without touching a GPU
    bench.barrier(w)
    dist.destroy_process_group()
    out.put((r, w, l, t))


@pytest.mark.timeout(120)
def test_two_ranks_max_and_barrier():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert all(x[3] == 2.5 for x in res)  # the maximum over both ranks
