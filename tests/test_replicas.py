"""Replica bookkeeping of multi-GPU runs, on CPU with gloo and two ranks.

bench.py --gpus N runs one replica per GPU: the ranks share nothing but a barrier and the
maximum of their device times. These tests run the same Replicas code as two gloo ranks:
the maximum and the shards are right on every rank, and a rank that dies before a
collective makes the other rank's collective fail within the group timeout instead of
hanging."""
import multiprocessing as mp
import os
import socket

import pytest

from axon_b200.replicas import Replicas


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank: int, world: int, port: int, mode: str, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        rep = Replicas.from_env(world, backend="gloo", timeout_s=5.0)
        if mode == "die" and rank == 1:
            q.put((rank, "died"))
            q.close()
            q.join_thread()  # the message must leave before the process does
            os._exit(0)  # leaves between steps, with nothing in flight
        rep.barrier()
        m = rep.max(1.5 + rank)
        shard = list(rep.shard(25))
        rep.barrier()
        rep.close()
        q.put((rank, (m, shard)))
    except Exception as e:  # the surviving rank of the "die" case ends up here
        q.put((rank, f"error: {type(e).__name__}"))


def run(world: int, mode: str):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_max_and_shards_over_two_ranks():
    out = run(2, "ok")
    (m0, s0), (m1, s1) = out[0], out[1]
    assert m0 == m1 == 2.5
    assert s0 + s1 == list(range(25)) and abs(len(s0) - len(s1)) <= 1


def test_single_replica_needs_no_group():
    rep = Replicas.from_env(1)
    assert (rep.rank, rep.world) == (0, 1) and rep.max(3.0) == 3.0 and list(rep.shard(4)) == [0, 1, 2, 3]


def test_dead_rank_fails_the_collective_not_hangs():
    out = run(2, "die")
    assert out[1] == "died"
    assert isinstance(out[0], str) and out[0].startswith("error")
