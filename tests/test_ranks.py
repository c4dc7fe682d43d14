"""The N > 1 path of bench.py on CPU: one process per rank over `gloo`
(world size 2), as torchrun starts them.  The path does not shard (each rank
runs an independent replica of the workload), so what the ranks share is the
timing protocol: a barrier on both sides of the timed region and the maximum
of the per-rank times, which every rank must see.  The reference arm runs on
rank 0 only; the other ranks return without work."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks()
    ranks.init("gloo")
    try:
        ranks.barrier()
        out[rank] = ranks.max(1.5 + rank)  # each rank's own "time"
        ranks.barrier()
        # the reference arm on a rank other than 0 returns at once, with no work
        out[world + rank] = bench.run_reference(None, ranks) is None if rank else True
    finally:
        ranks.close()


def test_two_gloo_ranks_share_the_max_time():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0]
        assert [out[r] for r in range(world)] == [2.5, 2.5]
        assert out[world + 1] is True


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks()
    if ranks.world != 1:
        pytest.skip("run under a launcher")
    ranks.init("gloo")
    assert ranks.dist is None
    assert ranks.max(3.25) == 3.25
    ranks.barrier()
    ranks.close()
