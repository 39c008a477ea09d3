"""Multi-rank plumbing on CPU: two gloo ranks split a batch of worlds by cell count (every world on exactly one
rank, the loads balanced) and agree on the max-over-ranks timing; no GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from sandbox_reactions_b200.distributed import max_over_ranks, partition


def test_partition_covers_every_world_once_and_balances():
    cells = [2048 ** 2] * 5 + [1024 ** 2] * 11 + [512 ** 2] * 20 + [256 ** 2] * 28
    for world in (1, 2, 4, 8):
        share = partition(cells, world)
        flat = sorted(i for s in share for i in s)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in s) for s in share]
        assert max(loads) - min(loads) <= max(cells)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cells = [64 * 64, 128 * 128, 32 * 32, 256 * 256, 64 * 64]
    mine = partition(cells, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    slowest = max_over_ranks(dist, 10.0 + rank)
    out[rank] = (sorted(i for s in got for i in s), slowest)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_split_the_batch_and_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
            assert p.exitcode == 0
        for r in range(2):
            assert out[r][0] == [0, 1, 2, 3, 4]
            assert out[r][1] == 11.0
