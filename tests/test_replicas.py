"""Multi-rank host logic of the benchmark (replicas only), on CPU with the gloo backend.

The step does not shard: N ranks run N independent replicas and the only collective is the
max-over-ranks reduction of the device time.  These tests run two gloo ranks as child processes:
 * the reduction returns the slowest rank's time on every rank;
 * a rank that leaves before the collective makes the other rank's collective end with an error
   within the process-group timeout instead of waiting for ever.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, world, port, timeout_s):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _put_and_flush(q, item):
    q.put(item)
    q.close()
    q.join_thread()


def _max_worker(rank, world, port, q):
    dist = _init(rank, world, port, 30)
    import bench
    q.put((rank, bench.max_over_ranks(1.5 + rank, "cpu")))
    dist.destroy_process_group()


def _leaver_worker(rank, world, port, q):
    dist = _init(rank, world, port, 5)
    import bench
    if rank == 1:
        _put_and_flush(q, (rank, "left"))
        os._exit(0)  # leaves between steps, with nothing in flight
    try:
        bench.max_over_ranks(1.0, "cpu")
    except Exception as e:  # noqa: BLE001 - any collective error is the expected outcome
        _put_and_flush(q, (rank, "error:" + type(e).__name__))
        os._exit(0)
    _put_and_flush(q, (rank, "no error"))
    os._exit(0)


def _run(fn, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, v = q.get(timeout=timeout)
        out[r] = v
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return out


def test_max_over_ranks_is_the_slowest_rank():
    out = _run(_max_worker)
    assert out == {0: 2.5, 1: 2.5}


def test_rank_that_leaves_ends_the_others_collective_with_an_error():
    out = _run(_leaver_worker)
    assert out[1] == "left"
    assert out[0].startswith("error:")


@pytest.mark.parametrize("world", [1])
def test_single_rank_needs_no_process_group(world):
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, "cpu") == 3.25
