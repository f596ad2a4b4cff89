"""Multi-rank host logic of bench.py on CPU: two gloo ranks (world_size 2) check the
max-over-ranks timing rule, the per-rank batches (weak scaling: no data-path collective) and
that the reference arm runs on rank 0 only."""
import datetime
import os
import socket
import sys

import pytest

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, REPO)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        r, w, lr = bench.rank_info()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, w, device="cpu")
        rate = bench.aggregate_rate(1024 * 3, w, ms)
        seed = bench.shard_seed(r)

        class Args:
            batch, steps, warmup = 4, 1, 0

        ref = bench.reference_arm(Args()) if r != 0 else "rank0-skipped"
        dist.barrier()
        q.put((r, w, ms, rate, seed, ref))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_bench_host_logic():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, ms0, rate0, seed0, _), (r1, w1, ms1, rate1, seed1, ref1) = out
    assert (r0, r1) == (0, 1) and w0 == w1 == 2
    assert ms0 == ms1 == 15.0  # the slowest rank's time
    assert rate0 == rate1 == pytest.approx(2 * 1024 * 3 / 15e-3)
    assert seed0 != seed1  # each rank evaluates its own binaries
    assert ref1 is None  # the reference arm runs on rank 0 only
