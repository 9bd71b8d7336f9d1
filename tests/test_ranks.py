"""Multi-process rank plumbing on CPU (gloo, world size 2): the collectives
bench.py uses around its timed region, the batch shards and the whole-job
rate, run as two real processes."""

import multiprocessing as mp
import os
import socket

import pytest

from fhelium_b200 import ranks


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, ws: int, port: int, times: list, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    try:
        got_ws, got_rank, _ = ranks.init("gloo", timeout_s=60)
        ranks.barrier(got_ws)
        worst = ranks.max_over_ranks(times[rank], got_ws)
        ranks.barrier(got_ws)
        start, end = ranks.shard(10, got_ws, got_rank)
        rate = ranks.job_rate(16, got_ws, worst)
        ranks.finish(got_ws)
        q.put((rank, got_ws, worst, start, end, rate))
    except Exception as exc:  # reported to the parent
        q.put((rank, "error", repr(exc)))


def test_two_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [12.5, 17.25]  # ms of each rank's timed region
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    assert all(r[1] == 2 for r in results), results
    for _, _, worst, _, _, rate in results:
        assert worst == 17.25
        assert rate == pytest.approx(2 * 16 / 0.01725)
    # shards of 10 items over 2 ranks
    assert [(r[3], r[4]) for r in results] == [(0, 5), (5, 10)]


@pytest.mark.parametrize("total,ws", [(10, 3), (7, 7), (3, 4), (0, 2), (1000, 8)])
def test_shards_cover_disjointly(total, ws):
    spans = [ranks.shard(total, ws, r) for r in range(ws)]
    assert spans[0][0] == 0 and spans[-1][1] == total
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_single_rank_needs_no_process_group():
    assert ranks.max_over_ranks(3.5, 1) == 3.5
    assert ranks.job_rate(32, 1, 32.0) == pytest.approx(1000.0)
    with pytest.raises(ValueError):
        ranks.shard(4, 2, 2)
