"""The multi-GPU host path on the CPU: two gloo ranks each play their shard of the rank space (with the
oracle, since there is no GPU here) and combine with shard.allreduce_result; the combined result must
equal the whole range played at once.  Also the shard arithmetic itself."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, n, mode, flags, q):
    sys.path.insert(0, os.path.join(ROOT, "endless-games-of-war_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch.distributed as dist
    import oracle
    import shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    total = oracle.space_size(n, mode)
    lo, hi = shard.shard_range(0, total, rank, world)
    r = oracle.enumerate_job(oracle.make_job(n, mode, 0, flags, lo, hi, hbins=256, dbins=64), threads=2)
    red = shard.allreduce_result(shard.result_to_dict(r))
    q.put((rank, red))
    dist.destroy_process_group()


@pytest.mark.parametrize("n,mode,flags", [(9, 0, 0), (9, 1, 2)])
def test_two_gloo_ranks_equal_whole_range(oracle, n, mode, flags):
    sys.path.insert(0, os.path.join(ROOT, "endless-games-of-war_b200"))
    import shard
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, n, mode, flags, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = shard.result_to_dict(oracle.enumerate_job(oracle.make_job(n, mode, 0, flags, hbins=256, dbins=64)))
    for rank, red in got:
        assert red == whole, rank


def test_shard_range_partitions():
    sys.path.insert(0, os.path.join(ROOT, "endless-games-of-war_b200"))
    import shard
    for lo, hi in ((0, 6227020800), (5, 5), (17, 1000003)):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_range(lo, hi, r, world) for r in range(world)]
            assert parts[0][0] == lo and parts[-1][1] == hi
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert sum(b - a for a, b in parts) == hi - lo
    with pytest.raises(ValueError):
        shard.shard_range(0, 10, 2, 2)
