"""The multi-rank path of bench.py on the CPU: two gloo ranks (127.0.0.1) agree on the slowest rank's times and
on the whole-job throughput; a rank that fails before the collective makes the other end with an error, not a
hang (short process-group timeout)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q, fail_rank):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    import bench
    try:
        if rank == fail_rank:
            raise RuntimeError('injected failure before the collective')
        ms = [10.0 + 5 * rank, 20.0 - rank, 1.0, 2.0 + rank, 3.0]
        agg = bench.max_over_ranks(ms, world)
        q.put((rank, agg, bench.job_throughput(65536, world, agg[0])))
    except Exception as e:  # the failing rank, or the survivor whose collective times out
        q.put((rank, 'error', type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
    alive = [p for p in ps if p.is_alive()]
    for p in alive:
        p.kill()
    out = {}
    while not q.empty():
        r, a, b = q.get()
        out[r] = (a, b)
    return out, alive


def test_two_gloo_ranks_take_the_max_and_weak_scale():
    out, alive = _run(2)
    assert not alive and sorted(out) == [0, 1]
    for r in (0, 1):
        agg, thr = out[r]
        assert agg == [15.0, 20.0, 1.0, 3.0, 3.0]
        assert thr == pytest.approx(2 * 65536 / 0.015)


def test_a_failing_rank_does_not_hang_the_other():
    out, alive = _run(2, fail_rank=1)
    assert not alive
    assert out[1][0] == 'error'
    assert out.get(0, ('error',))[0] == 'error'
