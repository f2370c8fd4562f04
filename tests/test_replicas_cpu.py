"""Multi-rank replica plumbing of bench.py on CPU: two gloo ranks (127.0.0.1), each with its own
timing, agree on the barrier and on the MAX over ranks that the bench reports; the ensemble decks
of different ranks differ (seed + rank) while a rank's own decks are reproducible."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    from salec_b200 import decks
    r = bench.Ranks("gloo", timeout_s=60)
    r.barrier()
    mx = r.all_max(10.0 * (rank + 1))
    d = decks.ensemble_decks(3, seed=100 + rank)
    q.put((rank, mx, [(x.npx, x.npy) for x in d]))
    r.close()


def test_two_gloo_ranks_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [20.0, 20.0]
    assert out[0][2] != out[1][2]
