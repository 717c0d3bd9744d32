"""Island sharding across ranks: two gloo ranks on CPU each take their share
of a field's islands, process it, and the gathered rows cover every island
exactly once; the merged table is independent of the rank count."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from uniphot_b200.shard import merge_rows, shard_islands


def _plans():
    from uniphot_b200.synth import make_small_field
    from uniphot_b200.plan import plan_island_classes
    f = make_small_field(1)
    plans, _ = plan_island_classes(f.island_set, f.buckets, f.source_type, f.logre,
                                   f.sersic_n, 55)
    return plans


def test_partition_is_exact_and_balanced():
    plans = _plans()
    for world in (1, 2, 3, 8):
        assign = shard_islands(plans, world)
        seen = set()
        for rank in assign:
            for ci, rows in rank:
                for r in rows:
                    assert (ci, int(r)) not in seen
                    seen.add((ci, int(r)))
        assert len(seen) == sum(p.n_islands for p in plans)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    plans = _plans()
    mine = shard_islands(plans, world)[rank]
    rows = {"src": [], "island": []}
    for ci, rr in mine:
        for r in rr:
            m = plans[ci].midx[r][plans[ci].mmask[r]]
            rows["src"].extend(m.tolist())
            rows["island"].extend([int(plans[ci].isl_ids[r])] * m.size)
    part = {k: np.asarray(v) for k, v in rows.items()}
    out = [None] * world
    dist.all_gather_object(out, part)
    if rank == 0:
        q.put(merge_rows(out))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_two_ranks_cover_field(world):
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    plans = _plans()
    n_src = sum(int(p.mmask.sum()) for p in plans)
    assert merged["src"].size == n_src
    assert np.unique(merged["src"]).size == n_src
    assert np.all(np.diff(merged["src"]) > 0)


def test_shard_plan_slices_plans_and_host_arrays_consistently():
    """Every rank's share of a planned field: the class plans and host
    arrays sliced to the same rows, every fitted island on exactly one rank,
    the giants on rank 0 only."""
    from uniphot_b200.shard import shard_plan
    from uniphot_b200.solver import plan_field
    from uniphot_b200.synth import make_production_field
    f = make_production_field(1, side=320, n_bands=2, n_src=40, margin=40)
    fp = plan_field(**f.fit_kwargs("analytic"))
    full = {(p.key, int(i)) for p, _ in fp.classes for i in p.isl_ids}
    index = {(p.key, int(i)): (p, h, r) for p, h in fp.classes
             for r, i in enumerate(p.isl_ids)}
    for world in (1, 2, 3):
        seen = set()
        for rank in range(world):
            sp = shard_plan(fp, world, rank)
            assert (len(sp.capped) > 0) == (rank == 0 and len(fp.capped) > 0)
            for p, h in sp.classes:
                assert p.n_islands > 0
                for r, i in enumerate(p.isl_ids):
                    key = (p.key, int(i))
                    assert key not in seen
                    seen.add(key)
                    p0, h0, r0 = index[key]
                    np.testing.assert_array_equal(p.midx[r], p0.midx[r0])
                    np.testing.assert_array_equal(h["p0"][r], h0["p0"][r0])
                    np.testing.assert_array_equal(h["ox"][r], h0["ox"][r0])
        assert seen == full
