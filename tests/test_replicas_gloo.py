"""CPU, world size 2 over gloo: the host logic of multi-GPU replica runs.

* the max-over-ranks timing every rank reports;
* root sharding (every root in exactly one share);
* a rank that fails before the collective: the other rank's collective ends
  with an error after the group's short timeout instead of waiting forever
  (failure detection on the host, no GPU involved).
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    from velographx_b200 import replicas

    try:
        replicas.init("gloo", timeout_s=5.0 if mode == "fail" else 60.0)
        if mode == "ok":
            t = replicas.max_over_ranks(1.5 + rank)
            mine = replicas.shard(list(range(11)), rank, world)
            q.put((rank, t, mine))
        else:
            if rank == 1:
                q.put((rank, "left", None))
                return  # leaves without joining the collective
            try:
                replicas.max_over_ranks(1.0)
                q.put((rank, "no-error", None))
            except Exception as e:  # the collective times out
                q.put((rank, "error", type(e).__name__))
    finally:
        if dist.is_initialized() and not (mode == "fail" and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda x: x[0])


def test_max_over_ranks_and_root_shards():
    out = _run("ok")
    assert [o[1] for o in out] == [2.5, 2.5]
    shares = [o[2] for o in out]
    assert sorted(shares[0] + shares[1]) == list(range(11))
    assert abs(len(shares[0]) - len(shares[1])) <= 1


def test_a_rank_that_leaves_ends_the_collective_with_an_error():
    out = _run("fail")
    assert out[1][1] == "left"
    assert out[0][1] == "error", out


def test_shard_rejects_bad_ranks():
    from velographx_b200 import replicas

    with pytest.raises(ValueError):
        replicas.shard([1, 2], 2, 2)
    assert replicas.max_over_ranks(3.25) == 3.25  # no group: the value itself
