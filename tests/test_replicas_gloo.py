"""Replica bookkeeping with two gloo ranks on the CPU: plan sharding, the
slowest-rank time, the whole-job work sum, and a rank that fails before a
collective is seen by its peer as an error, not a hang."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "dosecuda-jax_b200"))
    from dosecuda_b200 import replicas
    w, r, _ = replicas.init("gloo", timeout_s=10.0)
    assert (w, r) == (world, rank)
    mine = list(replicas.shard(11, r, w))
    t = replicas.max_over_ranks(1.5 + r, w)
    e = replicas.sum_over_ranks(len(mine), w)
    if fail_rank == r:
        os._exit(3)          # leaves between collectives, as a crashed rank would
    try:
        replicas.barrier(w)
        out.put((r, mine, t, e, "ok"))
    except Exception as exc:  # the peer learns of the failure from the collective
        out.put((r, mine, t, e, type(exc).__name__))
    finally:
        try:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()
        except Exception:
            pass


def _run(fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, fail_rank)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    results = []
    while not q.empty():
        results.append(q.get())
    for p in procs:
        if p.is_alive():
            p.kill()
    return sorted(results), [p.exitcode for p in procs]


def test_shard_covers_items_once():
    from dosecuda_b200 import replicas
    for n in (0, 1, 7, 32):
        for w in (1, 2, 3, 8):
            got = [i for r in range(w) for i in replicas.shard(n, r, w)]
            assert got == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_two_gloo_ranks_reduce():
    results, codes = _run(fail_rank=None)
    assert codes == [0, 0]
    assert [r[0] for r in results] == [0, 1]
    assert results[0][1] == list(range(0, 6)) and results[1][1] == list(range(6, 11))
    assert all(r[2] == 2.5 for r in results)          # max over ranks
    assert all(r[3] == 11 for r in results)           # sum over ranks
    assert all(r[4] == "ok" for r in results)


def test_failed_rank_surfaces_as_error_on_peer():
    results, codes = _run(fail_rank=1)
    assert codes[1] == 3
    assert len(results) == 1 and results[0][0] == 0
    assert results[0][4] != "ok"
