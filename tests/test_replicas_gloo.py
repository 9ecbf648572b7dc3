"""The multi-GPU path of bench.py is replicas only: every rank advances its own
copy of the workload and the ranks meet only at the barriers around the timed
regions and in the max-over-ranks of the device time.  That host logic, run
here as two gloo ranks on the CPU."""
import multiprocessing as mp
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import sys
    from datetime import timedelta
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=timedelta(seconds=60))
    barrier, max_over_ranks = bench.rank_sync(ws, "cpu")
    barrier()
    ms = max_over_ranks(10.0 + 5.0 * rank)  # the slowest rank's time
    zones = 1000  # each replica's zone-updates
    value = ws * zones / (ms / 1e3)  # the whole job's throughput
    barrier()
    dist.destroy_process_group()
    q.put((rank, ms, value))


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    assert all(abs(o[2] - 2 * 1000 / 0.015) < 1e-6 for o in out)
