"""Multi-GPU replica plumbing on CPU: 2-rank gloo process groups (no GPU).

The barotropic path does not shard; N GPUs run independent integrations.
These tests cover what the ranks share -- max/sum reductions of the timing
figures, the barrier, the work-balanced assignment of ensemble members or
requests to ranks -- and that a rank that fails makes its peer's next
collective end with an error instead of waiting forever.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from licom4py_gpu_b200.ensemble import uneven_mix
from licom4py_gpu_b200.replicas import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, mode, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from licom4py_gpu_b200 import replicas
    try:
        replicas.setup("gloo", timeout_s=10.0)
        if mode == "fail" and rank == 1:
            raise SystemExit(3)  # this rank dies before the collective; its process group goes away
        mx = replicas.max_over_ranks(rank + 1.5)
        sm = replicas.sum_over_ranks(rank + 1.5)
        replicas.barrier()
        specs = uneven_mix()
        mine = shard(specs, world, rank, work=lambda s: s.n * s.n * s.nsub)
        import torch.distributed as dist
        allv = [None] * world
        dist.all_gather_object(allv, [specs.index(s) for s in mine])
        out.put((rank, "ok", mx, sm, allv))
    except SystemExit:
        raise
    except Exception as e:  # the peer's failure surfaces here as an error, not a hang
        out.put((rank, "error", type(e).__name__, str(e)[:200], None))
    finally:
        try:
            replicas.teardown()
        except Exception:
            pass


def _run(world, mode):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = []
    for p in procs:
        p.join(timeout=90)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
    while not out.empty():
        res.append(out.get())
    return {r[0]: r for r in res}, [p.exitcode for p in procs]


@pytest.mark.timeout(120)
def test_two_rank_reductions_barrier_and_sharding():
    res, codes = _run(2, "ok")
    assert codes == [0, 0]
    for rank in (0, 1):
        _, status, mx, sm, allv = res[rank]
        assert status == "ok" and mx == 2.5 and sm == 4.0
        a, b = allv
        assert not set(a) & set(b) and sorted(a + b) == list(range(64))


@pytest.mark.timeout(120)
def test_a_failed_rank_ends_the_peer_collective_with_an_error():
    res, codes = _run(2, "fail")
    assert codes[1] == 3
    assert res[0][1] == "error"  # rank 0 learned of it from its collective, within the timeout


def test_shard_is_balanced_disjoint_and_deterministic():
    specs = uneven_mix()
    work = lambda s: 6 * s.n * s.n * s.nsub  # noqa: E731
    for world in (1, 2, 3, 4, 8):
        parts = [shard(specs, world, r, work) for r in range(world)]
        assert sorted(x for p in parts for x in map(specs.index, p)) == list(range(len(specs)))
        loads = [sum(work(s) for s in p) for p in parts]
        assert max(loads) - min(loads) <= max(work(s) for s in specs)
        assert parts == [shard(specs, world, r, work) for r in range(world)]
    with pytest.raises(ValueError):
        shard(specs, 2, 2)
