"""The N > 1 path of bench.py on the CPU: two ranks over gloo, as
torch.distributed.run starts them.  Each rank runs its own replicate (its own
seed); the reported time is the slowest rank's; the whole-job rate counts
every rank's work; only rank 0 reports."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from lattice_microbes_b200.replicas import Ranks, aggregate_rate
    r = Ranks().init("gloo", timeout_s=60)
    my_ms = 100.0 + 50.0 * rank           # rank 1 is the slow one
    r.barrier()
    slowest = r.max(my_ms)
    rate = aggregate_rate(1000, slowest, r.world)
    out.put((r.rank, r.leader, r.seed(2024), slowest, rate))
    r.finish()


def test_two_ranks_over_gloo():
    from lattice_microbes_b200.solver import compose_seed
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[1] for x in res] == [True, False]
    assert [x[2] for x in res] == [compose_seed(2024, 0), compose_seed(2024, 1)]
    assert res[0][2] != res[1][2]
    assert all(x[3] == 150.0 for x in res)
    assert all(x[4] == pytest.approx(1000 * 2 / 0.15) for x in res)


def test_single_process_needs_no_group():
    from lattice_microbes_b200.replicas import Ranks, aggregate_rate
    r = Ranks(environ={}).init("gloo")
    assert (r.world, r.rank, r.leader, r.group) == (1, 0, True, False)
    assert r.max(12.5) == 12.5
    r.barrier()
    r.finish()
    assert aggregate_rate(500, 250.0, 1) == pytest.approx(2000.0)
