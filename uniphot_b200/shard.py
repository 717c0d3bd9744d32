"""Island sharding across ranks (one process per GPU).

Islands are independent (no pixel couples two islands), so a field's fitted
islands are partitioned across ranks with no collective on the data path;
each rank solves its share and the per-source result rows are gathered on
the host.  The partition is longest-processing-time over a per-island cost
estimate, like the reference's multi-GPU chunk queue
(``fit/grid_gpu/island_stage.py:561-1330``), but static and deterministic so
that every rank computes the same assignment without communication.
"""

from __future__ import annotations

import heapq

import numpy as np


def island_cost(plan) -> float:
    """Relative per-island cost: members x window pixels x render weight."""
    w = 4.0 if plan.kind == "mixed" else 1.0
    return float(plan.nsrc_class) * float(plan.bbox_class) ** 2 * w * \
        (float(plan.tier) / 31.0)


def shard_islands(plans, world: int) -> list:
    """Assign every (class index, row) to a rank.

    Returns ``assign[rank] = list of (class_index, np.ndarray rows)`` with
    rows ascending; every island appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    items = []
    for ci, p in enumerate(plans):
        c = island_cost(p)
        items.extend((c, ci, r) for r in range(p.n_islands))
    items.sort(key=lambda t: (-t[0], t[1], t[2]))
    heap = [(0.0, r) for r in range(world)]
    per = [dict() for _ in range(world)]
    for c, ci, r in items:
        load, rank = heapq.heappop(heap)
        per[rank].setdefault(ci, []).append(r)
        heapq.heappush(heap, (load + c, rank))
    return [[(ci, np.asarray(sorted(rows), np.int64)) for ci, rows in sorted(d.items())]
            for d in per]


def merge_rows(parts: list) -> dict:
    """Concatenate per-rank result-row dicts (same keys) and sort by source
    index, so the merged table is independent of the rank count."""
    keys = parts[0].keys()
    cat = {k: np.concatenate([p[k] for p in parts], axis=0) for k in keys}
    order = np.argsort(cat["src"], kind="stable")
    return {k: v[order] for k, v in cat.items()}


def shard_plan(fp, world: int, rank: int):
    """The rank's share of a planned field (``solver.plan_field``): per class,
    the rows ``shard_islands`` assigns to the rank, with the class plan's
    per-island arrays and the host arrays sliced to them (classes with no
    rows on this rank dropped).  The giant islands (seed rows, no fit) go to
    rank 0 alone, so the ranks' results together cover every source once.
    ``IslandFitJob(plan=...)`` solves the share."""
    import dataclasses
    plans = [p for p, _ in fp.classes]
    share = shard_islands(plans, world)[rank]
    classes = [slice_class(*fp.classes[ci], rows) for ci, rows in share]
    return dataclasses.replace(fp, classes=classes,
                               capped=fp.capped if rank == 0 else type(fp.capped)())


def slice_class(plan, host: dict, rows):
    """(class plan, host arrays) restricted to the given island rows: the
    plan's per-island arrays and every host array with one row per island."""
    import dataclasses
    rows = np.asarray(rows, np.int64)
    n = plan.n_islands
    sp = dataclasses.replace(plan, isl_ids=plan.isl_ids[rows], midx=plan.midx[rows],
                             mmask=plan.mmask[rows], bbox=plan.bbox[rows],
                             n_src_of=plan.n_src_of[rows])
    sh = {k: (v[rows] if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == n
              else v) for k, v in host.items()}
    return sp, sh
