"""Multi-rank host logic on CPU (gloo, world size 2): the batch of
independent meshes shards by the LPT partition with no data-path collective;
every rank derives the same partition, the shares cover the batch once, the
per-rank results assemble into the serial answer, and the job time is the
max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tool_godot_curvenet_b200.shard import lpt_partition, mesh_cost, rank_share, reduce_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _costs(n=37, seed=3):
    rng = np.random.default_rng(seed)
    nv = np.exp(rng.uniform(np.log(2000), np.log(60000), n)).astype(int)
    return [mesh_cost(v, 2 * v) for v in nv]


def _rank_main(rank, world, port, out_dir):
    from datetime import timedelta

    import torch.distributed as dist
    from oracle import oracle as O
    from tests.helpers import workload
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        costs = _costs()
        mine = rank_share(costs, world, rank)
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        # the job time is the max of the per-rank times
        t = reduce_over_ranks(dist, world, 10.0 + rank, "max")
        tot = reduce_over_ranks(dist, world, float(len(mine)), "sum")
        # each rank solves its share of four small systems with the oracle
        pos, tris, h, tg = workload("cyl_tiny")
        jobs = [(s, tg * (1.0 + 0.1 * s)) for s in range(4)]
        share = rank_share([1, 3, 2, 5], world, rank)
        ref = O.System(pos, tris, h)
        res = {s: ref.solve(jobs[s][1], mode=1, tol=1e-12)[1] for s in share}
        allres = [None] * world
        dist.all_gather_object(allres, res)
        if rank == 0:
            np.savez(os.path.join(out_dir, "r.npz"), parts=np.array(parts, dtype=object), t=t, tot=tot,
                     **{f"x{s}": x for d in allres for s, x in d.items()})
    finally:
        dist.destroy_process_group()


def test_lpt_partition_properties():
    costs = _costs()
    for world in (1, 2, 3, 8):
        parts = lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound


def test_two_ranks_gloo(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    d = np.load(tmp_path / "r.npz", allow_pickle=True)
    parts = [list(p) for p in d["parts"]]
    assert parts == lpt_partition(_costs(), world)
    assert float(d["t"]) == 11.0 and float(d["tot"]) == len(_costs())
    from oracle import oracle as O
    from tests.helpers import workload
    pos, tris, h, tg = workload("cyl_tiny")
    ref = O.System(pos, tris, h)
    for s in range(4):
        want = ref.solve(tg * (1.0 + 0.1 * s), mode=1, tol=1e-12)[1]
        assert np.array_equal(d[f"x{s}"], want)
