"""The multi-GPU layout on the host: replicas as gloo ranks (world size 2).

Each rank steps its own seeded disk with no exchange between ranks; the
process group carries only the timing (barriers and the max over ranks).  On
the GPUs the same calls run over NCCL.  Here the disks are stepped by the
CPU restatement, which stands in for the device step: the test covers the
rank layout, seeds, barrier, max-over-ranks reduction and job rate, an
ensemble split across the ranks by whole disks and gathered on rank 0, and
how a rank that fails or never joins surfaces on the others.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> None:
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})


def _small_disk():
    from penguin_b200 import params as P

    return P.reference_disk(32, 96).replace(kill_flag=0)


def _replica_rank(rank: int, world: int, port: int, out: str) -> None:
    """One rank of a replicas job: its own seeded disk, then the timing collectives."""
    _env(rank, world, port)
    from oracle.oracle import Oracle
    from penguin_b200 import initial as I
    from penguin_b200.replicas import Replicas

    job = Replicas("gloo", timeout_s=60)
    p = _small_disk()
    o = Oracle(p, I.disk_state(p, seed=job.seed(1234)), 0.0)
    if rank == 1:
        time.sleep(1.5)           # the other rank must wait for this one at the barrier
    t0 = time.perf_counter()
    job.barrier()
    waited = time.perf_counter() - t0
    n = o.run(3)
    ms = 10.0 * (rank + 1)        # stand-in device times: rank 1 is the slower
    worst = job.max_over_ranks(ms)
    rate = job.job_rate(p.cells * n, worst)
    r = o.interior()["r"]
    res = {"rank": job.rank, "world": job.world, "printer": job.printer, "waited": waited, "worst": worst,
           "rate": rate, "steps": n, "cells": p.cells, "r_sum": float(np.sum(r))}
    job.barrier()
    job.close()
    with open(out, "w") as f:
        json.dump(res, f)


def _run_ranks(target, world: int, tmp_path, timeout: float = 120.0, **kw):
    ctx = mp.get_context("spawn")
    port = _free_port()
    outs = [str(tmp_path / f"rank{r}.json") for r in range(world)]
    procs = [ctx.Process(target=target, args=(r, world, port, outs[r]), kwargs=kw) for r in range(world)]
    for q in procs:
        q.start()
    for q in procs:
        q.join(timeout)
    for q in procs:
        if q.is_alive():
            q.kill()
            q.join()
    return procs, outs


def test_two_replicas_gloo(tmp_path):
    procs, outs = _run_ranks(_replica_rank, 2, tmp_path)
    assert [q.exitcode for q in procs] == [0, 0]
    res = [json.load(open(o)) for o in outs]
    assert [r["rank"] for r in res] == [0, 1]
    assert all(r["world"] == 2 for r in res)
    assert [r["printer"] for r in res] == [True, False]
    # the barrier held rank 0 until the late rank arrived
    assert res[0]["waited"] > 0.75
    # every rank sees the slowest rank's time, and counts both ranks' zone-updates
    assert all(r["worst"] == 20.0 for r in res)
    for r in res:
        assert r["rate"] == pytest.approx(r["cells"] * r["steps"] * 2 / 0.020, rel=1e-12)
    # each replica stepped its own disk: the same result as a lone run with that seed
    from oracle.oracle import Oracle
    from penguin_b200 import initial as I

    p = _small_disk()
    for r in res:
        o = Oracle(p, I.disk_state(p, seed=1234 + r["rank"]), 0.0)
        o.run(3)
        assert r["r_sum"] == float(np.sum(o.interior()["r"]))
    assert res[0]["r_sum"] != res[1]["r_sum"]


def _leaving_rank(rank: int, world: int, port: int, out: str) -> None:
    """Rank 1 leaves between steps (after a barrier, nothing in flight); rank 0's
    next collective must end with an error, not wait for good."""
    _env(rank, world, port)
    from penguin_b200.replicas import Replicas

    job = Replicas("gloo", timeout_s=10)
    job.barrier()
    if rank == 1:
        os._exit(0)
    t0 = time.perf_counter()
    try:
        job.max_over_ranks(1.0)
        res = {"error": None}
    except Exception as e:  # the peer's departure surfaces as an exception
        res = {"error": type(e).__name__}
    res["seconds"] = time.perf_counter() - t0
    with open(out, "w") as f:
        json.dump(res, f)
    os._exit(0)


def test_rank_that_leaves_is_detected(tmp_path):
    procs, outs = _run_ranks(_leaving_rank, 2, tmp_path)
    assert [q.exitcode for q in procs] == [0, 0]
    res = json.load(open(outs[0]))
    assert res["error"] is not None
    assert res["seconds"] < 60.0


def _lonely_rank(rank: int, world: int, port: int, out: str) -> None:
    _env(rank, world, port)
    from penguin_b200.replicas import Replicas

    t0 = time.perf_counter()
    try:
        Replicas("gloo", timeout_s=3)
        res = {"error": None}
    except Exception as e:
        res = {"error": type(e).__name__}
    res["seconds"] = time.perf_counter() - t0
    with open(out, "w") as f:
        json.dump(res, f)


def test_rank_that_never_joins_times_out(tmp_path):
    """Only rank 0 of two starts: the rendezvous ends with an error at its timeout."""
    ctx = mp.get_context("spawn")
    out = str(tmp_path / "rank0.json")
    q = ctx.Process(target=_lonely_rank, args=(0, 2, _free_port(), out))
    q.start()
    q.join(120)
    if q.is_alive():
        q.kill()
        q.join()
    assert q.exitcode == 0
    res = json.load(open(out))
    assert res["error"] is not None
    assert res["seconds"] < 60.0


def test_single_rank_is_local():
    from penguin_b200.replicas import Replicas

    job = Replicas("gloo", env={"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert job.dist is None and job.printer and job.world == 1
    job.barrier()
    assert job.max_over_ranks(3.5) == 3.5
    assert job.job_rate(1000, 2.0) == pytest.approx(5.0e5)
    assert job.seed(1234) == 1234
    job.close()
    with pytest.raises(ValueError):
        job.job_rate(1000, 0.0)


@pytest.mark.parametrize("env", [{"WORLD_SIZE": "2", "RANK": "2"}, {"WORLD_SIZE": "0"},
                                 {"WORLD_SIZE": "2", "RANK": "0", "LOCAL_RANK": "-1"}])
def test_bad_rank_layout(env):
    from penguin_b200.replicas import Replicas

    with pytest.raises(ValueError):
        Replicas("gloo", env=env)


def test_reference_arm_under_torchrun():
    """The driver's launch of the reference arm at N=2: rank 0 alone prints one
    JSON line, the other rank exits 0 without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "10", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS=str(max(1, (os.cpu_count() or 2) // 2)))
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference" and j["n_gpus"] == 2 and j["value"] > 0
    assert j["e2e"]["h2d_bytes_per_step"] == 0 and j["cpu_baseline"]["kind"] == "port"


def test_partition_balances_whole_units():
    from penguin_b200 import params as P
    from penguin_b200.replicas import partition

    cells = [p.cells for p in P.disk_ensemble()]
    for world in (1, 2, 3, 8):
        parts = partition(cells, world)
        assert sorted(k for q in parts for k in q) == list(range(len(cells)))
        loads = [sum(cells[k] for k in q) for q in parts]
        # greedy heaviest-first: no rank exceeds the mean by more than one disk
        assert max(loads) <= sum(cells) / world + max(cells)
        assert parts == partition(cells, world)
    assert partition([5.0, 1.0], 4) == [[0], [1], [], []]
    assert partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)
    with pytest.raises(ValueError):
        partition([-1.0], 2)


def _ensemble_disks():
    from penguin_b200 import params as P

    return [P.reference_disk(nr, 3 * nr, q=q).replace(kill_flag=0)
            for nr, q in ((32, 1e-3), (64, 3e-4), (32, 0.0), (48, 1e-4), (32, 5e-4))]


def _ensemble_rank(rank: int, world: int, port: int, out: str) -> None:
    """One rank of a partitioned ensemble: its share of the disks, then the gather."""
    _env(rank, world, port)
    from oracle.oracle import Oracle
    from penguin_b200 import initial as I
    from penguin_b200.replicas import Replicas

    job = Replicas("gloo", timeout_s=60)
    ps = _ensemble_disks()
    mine = job.share([p.cells for p in ps])
    res = {}
    for k in mine:
        o = Oracle(ps[k], I.disk_state(ps[k], seed=100 + k), 0.0)
        o.run(2)
        res[k] = float(np.sum(o.interior()["r"]))
    allres = job.gather({"rank": job.rank, "disks": mine, "r_sum": res})
    job.close()
    if job.printer:
        with open(out, "w") as f:
            json.dump(allres, f)


def test_partitioned_ensemble_gloo(tmp_path):
    procs, outs = _run_ranks(_ensemble_rank, 2, tmp_path)
    assert [q.exitcode for q in procs] == [0, 0]
    allres = json.load(open(outs[0]))
    assert [r["rank"] for r in allres] == [0, 1]
    got = {int(k): v for r in allres for k, v in r["r_sum"].items()}
    ps = _ensemble_disks()
    assert sorted(got) == list(range(len(ps)))
    assert all(r["disks"] for r in allres)
    from oracle.oracle import Oracle
    from penguin_b200 import initial as I

    for k, p in enumerate(ps):
        o = Oracle(p, I.disk_state(p, seed=100 + k), 0.0)
        o.run(2)
        assert got[k] == float(np.sum(o.interior()["r"]))
