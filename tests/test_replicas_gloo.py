"""Sample-sharded replicas across ranks, exercised with the gloo backend on CPU
(world_size 2 and 3): sharding covers every sample once, results gather in sample order,
timings reduce to the max, and a rank that fails is seen by the others as an error."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import PKG_ROOT, REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_samples, q, fail_rank):
    import sys
    for p in (REPO, PKG_ROOT):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    from rlmb import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
        first, count = replicas.shard(n_samples, world, rank)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the collective")
        # stand-in per-sample results: a deterministic function of the sample index
        local = np.stack([np.arange(4) + 10.0 * (first + i) for i in range(count)]) if count else np.zeros((0, 4))
        full = replicas.gather_samples(local, n_samples, dist)
        t = replicas.max_over_ranks(0.5 + rank, dist)
        q.put((rank, first, count, full.tolist(), t))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:   # report to the parent instead of hanging
        q.put((rank, "error", repr(exc)))


def _run(world, n_samples, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_samples, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(res, key=lambda r: r[0])


def test_shard_covers_samples_once():
    from rlmb import replicas
    for n in (0, 1, 7, 64, 65):
        for w in (1, 2, 3, 8):
            seen = []
            for r in range(w):
                f, c = replicas.shard(n, w, r)
                seen.extend(range(f, f + c))
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


@pytest.mark.parametrize("world,n_samples", [(2, 64), (3, 7)])
def test_gather_and_max_over_gloo_ranks(world, n_samples):
    res = _run(world, n_samples)
    expect = np.stack([np.arange(4) + 10.0 * s for s in range(n_samples)])
    for rank, first, count, full, t in res:
        assert np.array_equal(np.array(full), expect)
        assert t == 0.5 + (world - 1)


def test_failing_rank_is_reported_not_hung():
    res = _run(2, 8, fail_rank=1)
    assert res[1][1] == "error"
    # the surviving rank's collective ends in an error (peer gone / timeout), not a hang
    assert res[0][1] == "error"
