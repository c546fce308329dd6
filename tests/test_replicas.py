"""The multi-rank bookkeeping of pysurf_b200.replicas, run as two gloo ranks on CPU.

Independent cases shard over ranks with no data-path collective; the ranks only meet at the
barrier around a timed region, the maximum of their times and the gathering of results.  These
tests run that logic with world size 2 over gloo (127.0.0.1), and check that a rank that leaves
makes its peer fail fast instead of waiting.
"""
import multiprocessing as mp
import os
import socket
import time

import pytest

from pysurf_b200 import replicas


def freePort() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def environment(port: int) -> None:
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)


def bookkeeping(rank: int, port: int, queue) -> None:
    environment(port)
    ranks = replicas.Ranks(rank, 2, rank)
    replicas.initialize(ranks, 'gloo', timeoutSeconds=30.0)
    try:
        mine = replicas.shard(range(11), ranks)
        replicas.barrier(ranks)
        worst = replicas.maxOverRanks(1.5 + rank, ranks)
        total = replicas.sumOverRanks(len(mine), ranks)
        gathered = replicas.gatherResults([(rank, item) for item in mine], ranks)
        queue.put((rank, mine, worst, total, gathered))
    finally:
        replicas.finalize(ranks)


def leaver(rank: int, port: int, queue) -> None:
    environment(port)
    ranks = replicas.Ranks(rank, 2, rank)
    replicas.initialize(ranks, 'gloo', timeoutSeconds=5.0)
    if rank == 1:
        os._exit(0)             # leaves between steps, with nothing in flight
    start = time.monotonic()
    try:
        replicas.barrier(ranks)
        queue.put(('no error', time.monotonic() - start))
    except Exception as error:  # the peer is gone: the collective ends with an error
        queue.put((type(error).__name__, time.monotonic() - start))


def runRanks(target, timeout: float = 60.0):
    context = mp.get_context('spawn')
    queue = context.Queue()
    port = freePort()
    processes = [context.Process(target=target, args=(rank, port, queue)) for rank in range(2)]
    for p in processes:
        p.start()
    results = []
    deadline = time.monotonic() + timeout
    try:
        while len(results) < sum(1 for _ in processes) and time.monotonic() < deadline:
            try:
                results.append(queue.get(timeout=1.0))
            except Exception:
                if all(not p.is_alive() for p in processes):
                    break
    finally:
        for p in processes:
            p.join(timeout=max(1.0, deadline - time.monotonic()))
            if p.is_alive():
                p.kill()
                p.join()
    return results, [p.exitcode for p in processes]


def test_shard_splits_every_item_once_and_evenly():
    items = list(range(257))
    for world in (1, 2, 3, 8):
        shares = [replicas.shard(items, replicas.Ranks(r, world, r)) for r in range(world)]
        assert sorted(x for share in shares for x in share) == items
        assert max(map(len, shares)) - min(map(len, shares)) <= 1


def test_one_rank_needs_no_process_group():
    ranks = replicas.Ranks(0, 1, 0)
    replicas.initialize(ranks)
    assert replicas.maxOverRanks(3.0, ranks) == 3.0
    assert replicas.gatherResults([1, 2], ranks) == [1, 2]
    replicas.barrier(ranks)
    replicas.finalize(ranks)


def test_two_gloo_ranks_share_cases_and_meet_only_for_bookkeeping():
    results, codes = runRanks(bookkeeping)
    assert codes == [0, 0]
    byRank = {r[0]: r for r in results}
    assert set(byRank) == {0, 1}
    assert byRank[0][1] == [0, 2, 4, 6, 8, 10] and byRank[1][1] == [1, 3, 5, 7, 9]
    for rank in (0, 1):
        assert byRank[rank][2] == 2.5          # the slower rank's time
        assert byRank[rank][3] == 11.0
    assert byRank[0][4] == [(0, i) for i in (0, 2, 4, 6, 8, 10)] + [(1, i) for i in (1, 3, 5, 7, 9)]
    assert byRank[1][4] is None


def test_a_rank_that_leaves_ends_its_peers_collective_with_an_error():
    results, codes = runRanks(leaver, timeout=90.0)
    assert len(results) == 1
    outcome, waited = results[0]
    assert outcome != 'no error'
    assert waited < 60.0
