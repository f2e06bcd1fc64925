"""Host side of the batched sweep: workload table, split of the domains over ranks
(greedy by cell count) and the gather of per-domain results, run as two gloo ranks on
the CPU with the oracle standing in for each rank's GPU batch."""
import os
import socket

import numpy as np
import pytest

from lbm3d_bb_b200 import sweep


def test_workload_table():
    p = sweep.sweep_params(512, seed=4)
    assert len(p) == 512 and p == sweep.sweep_params(512, seed=4)
    for q in p:
        assert q["nx"] in (48, 64, 96) and q["ny"] == q["nz"] in (32, 48)
        assert 3.0 <= q["r"] <= 8.0 and 5.0 <= q["Re"] <= 200.0
        assert q["nx"] / 4 <= q["center"][0] <= 3 * q["nx"] / 4
        assert abs(q["tau"] - (0.5 + 3 * 0.05 * 2 * q["r"] / q["Re"])) < 1e-12
    assert min(q["tau"] for q in p) > 0.5


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_complete_and_balanced(world):
    p = sweep.sweep_params(512, seed=4)
    parts = sweep.partition(p, world)
    assert sorted(i for q in parts for i in q) == list(range(512))
    loads = [sum(sweep.cells(p[i]) for i in q) for q in parts]
    assert max(loads) - min(loads) <= max(sweep.cells(q) for q in p)
    assert parts == sweep.partition(p, world)


def _tiny(count=6):
    out = []
    for q in sweep.sweep_params(count, seed=9):
        s = dict(q)
        s["nx"], s["ny"], s["nz"] = q["nx"] // 4, q["ny"] // 4, q["nz"] // 4
        s["r"] = q["r"] / 4 + 1.0
        s["center"] = tuple(c / 4 for c in q["center"])
        s["tau"] = 0.8
        out.append(s)
    return out


def _oracle_runner(params, steps):
    from oracle.oracle import OracleDomain

    res = []
    for p in params:
        d = sweep.make_domain(p, cls=OracleDomain)
        d.step(steps)
        fx = float(d.force()[0])
        res.append({"index": p["index"], "steps": steps, "stable": bool(np.isfinite(fx)), "fx": fx,
                    "cd": sweep.drag_coefficient(fx, p["r"])})
        d.close()
    return {"results": res, "cells": sum(sweep.cells(p) for p in params)}


def _rank(rank, world, port, q):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        out = sweep.run_sweep(_tiny(), 4, _oracle_runner, rank, world, dist)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_rank_sweep_gathers_every_domain(oracle_lib):
    import multiprocessing as mp

    single = sweep.run_sweep(_tiny(), 4, _oracle_runner)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    merged = got[0]
    assert merged["domains"] == single["domains"] == 6
    assert [r["index"] for r in merged["results"]] == list(range(6))
    for a, b in zip(merged["results"], single["results"]):
        assert a["fx"] == b["fx"]
    assert sorted(p["rank"] for p in merged["per_rank"]) == [0, 1]
