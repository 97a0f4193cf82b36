"""Multi-process host logic on CPU (gloo, world_size 2, 127.0.0.1): scenario
sharding (longest processing time first), barrier, max / sum over ranks and
gathering on rank 0 as bench.py uses them, and a rank that never joins ending
its peer's rendezvous with an error instead of a hang."""
import multiprocessing as mp
import os
import socket
import time

import numpy as np
import pytest

from hydroflux_b200.dist import lpt_shards


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_lpt_shards_partition_and_balance():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        w = (np.exp(rng.uniform(np.log(64), np.log(1024), 97)) ** 2).round()
        sh = lpt_shards(w, world)
        assert len(sh) == world
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(w)))
        loads = [w[s].sum() for s in sh]
        lower = max(w.max(), w.sum() / world)  # no schedule beats this
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
        assert lpt_shards(w, world) == sh  # deterministic
    assert lpt_shards([], 2) == [[], []]
    with pytest.raises(ValueError):
        lpt_shards([1.0], 0)


def _worker(rank, world, port, q, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    try:
        from hydroflux_b200.dist import Dist
        if mode == "absent" and rank == 1:
            q.put((rank, "left"))  # this rank never joins
            return
        t0 = time.time()
        try:
            d = Dist(use_gpu=False, timeout_s=8.0)
        except Exception as e:  # the peer never came: an error, not a hang
            q.put((rank, ("init-error", time.time() - t0, type(e).__name__)))
            return
        from hydroflux_b200.workloads import uniform
        sides = np.exp(uniform(0, 1, 40, np.log(64), np.log(1024))).round()
        weights = sides * sides
        mine = d.shard(weights)
        d.barrier()
        mx = d.max(float(rank + 1) * 1.5)
        sm = d.sum(float(len(mine)))
        got = d.gather({"rank": rank, "mine": mine, "load": float(weights[mine].sum())})
        d.close()
        q.put((rank, {"mine": mine, "max": mx, "sum": sm, "gather": got}))
    except Exception as e:  # report, never hang the test
        q.put((rank, ("error", repr(e))))


def run_ranks(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, v = q.get(timeout=120)
        out[r] = v
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_two_ranks_shard_reduce_gather():
    out = run_ranks("ok")
    for r in (0, 1):
        assert isinstance(out[r], dict), out[r]
    a, b = out[0]["mine"], out[1]["mine"]
    assert not set(a) & set(b) and sorted(a + b) == list(range(40))
    assert out[0]["max"] == out[1]["max"] == 3.0
    assert out[0]["sum"] == out[1]["sum"] == 40.0
    g = out[0]["gather"]
    assert [x["rank"] for x in g] == [0, 1] and g[1]["mine"] == b
    assert out[1]["gather"] is None
    loads = [x["load"] for x in g]
    assert max(loads) <= 4.0 / 3.0 * max(max(loads) - min(loads), sum(loads) / 2.0)


def test_absent_rank_ends_rendezvous_with_error():
    t0 = time.time()
    out = run_ranks("absent")
    assert out[1] == "left"
    assert isinstance(out[0], tuple) and out[0][0] == "init-error", out[0]
    assert time.time() - t0 < 110
