"""The multi-GPU path (independent replicas) with world_size 2 over gloo on the CPU: each rank advances
its own tank (the CPU oracle stands in for the device) and the run is aggregated as bench.py does."""
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


def _rank_main(rank, world, port, queue):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    from slosh_b200 import _abi as A, scenes
    from slosh_b200.replicas import reduce_run
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    sc = scenes.tiny(O.settings_default, n=16)
    o = O.Oracle(sc["settings"])
    o.set_emit_seed(sc["seed"])
    fi = A.frame_input(sc["settings"], emits=sc["emits"])
    substeps = 0
    for _ in range(2):
        o.step_frame(fi)
        substeps += o.results().substeps
        fi = A.frame_input(sc["settings"])
    total, dev_ms, wall_ms = reduce_run(substeps, 10.0 + rank, 20.0 + 3 * rank)
    queue.put((rank, substeps, total, dev_ms, wall_ms, o.results().fluid_cells))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=5) for _ in range(2))
    (r0, s0, t0, d0, w0, f0), (r1, s1, t1, d1, w1, f1) = out
    assert t0 == t1 == s0 + s1
    assert d0 == d1 == 11.0 and w0 == w1 == 23.0
    assert f0 == f1  # identical replicas


def _tanks_main(rank, world, port, queue):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import datetime

    import torch.distributed as dist

    from slosh_b200.replicas import gather_tank_stats, lpt_partition
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    costs = [5.0, 3.0, 8.0, 1.0, 4.0, 4.0, 2.0]
    plan = lpt_partition(costs, world)
    mine = [(i, 10 + i, 20 + rank, 100 * i) for i in plan[rank]]
    rows = gather_tank_stats(mine)
    # the benchmark's rows carry two more columns (batched and sequential substep latency)
    wide = gather_tank_stats([(i, 10 + i, 20 + rank, 100 * i, 0.5 + i, 0.25 * (rank + 1)) for i in plan[rank]], width=6)
    queue.put((rank, plan, rows, wide))
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_partition_plan():
    from slosh_b200.replicas import lpt_partition
    costs = [5.0, 3.0, 8.0, 1.0, 4.0, 4.0, 2.0]
    plan = lpt_partition(costs, 2)
    assert sorted(i for p in plan for i in p) == list(range(7))
    loads = [sum(costs[i] for i in p) for p in plan]
    assert abs(loads[0] - loads[1]) <= max(costs)
    assert plan == lpt_partition(costs, 2)  # deterministic
    assert lpt_partition(costs, 1) == [list(range(7))]


def test_two_rank_tank_batch_stats():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_tanks_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=5) for _ in range(2))
    (_, plan0, rows0, wide0), (_, plan1, rows1, wide1) = out
    assert plan0 == plan1
    assert rows0 == rows1
    assert wide0 == wide1 and all(len(r) == 6 for r in wide0)
    assert [int(r[0]) for r in wide0] == list(range(7))
    assert all(r[4] == 0.5 + r[0] and r[5] == 0.25 * (int(r[2]) - 19) for r in wide0)
    assert [int(r[0]) for r in rows0] == list(range(7))
    owner = {i: r for r, p in enumerate(plan0) for i in p}
    assert all(int(row[2]) == 20 + owner[int(row[0])] for row in rows0)
