"""The N > 1 replica path on CPU: two gloo ranks.  Each rank serves its own
share of a seeded job stream on a scheduler-only server; the replicas'
reductions (maximum time, summed work) and the partition of the stream are
checked against a single-process run."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from beamform_project_b200.replicas import Replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from beamform_project_b200 import serve
    r = Replicas(backend="gloo", timeout_s=60)
    try:
        assert r.max(rank + 1.5) == world + 0.5
        assert r.sum(rank + 1) == world * (world + 1) / 2
        jobs = serve.poisson_mix(seed=4, duration_s=0.1)
        mine = [jobs[i] for i in Replicas.partition(len(jobs), rank, world)]
        with serve.Server(60 * 10**9, max_jobs=64, host_only=True) as s:
            serve.run_stream(s, mine)
            st = s.stats()
        r.barrier()
        total_windows = r.sum(st["job_windows"])
        total_samples = r.sum(st["beam_samples"])
        out.put((rank, len(mine), total_windows, total_samples))
    finally:
        r.close()


def test_two_gloo_replicas_cover_the_stream():
    from beamform_project_b200 import serve
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    jobs = serve.poisson_mix(seed=4, duration_s=0.1)
    assert sum(n for _, n, _, _ in res) == len(jobs)
    assert all(w == sum(j.n_spectra // 320 for j in jobs) for _, _, w, _ in res)
    assert all(s == sum(j.beam_samples() for j in jobs) for _, _, _, s in res)


@pytest.mark.parametrize("n,world", [(10, 3), (2, 4), (0, 2), (7, 1)])
def test_partition_is_balanced_and_complete(n, world):
    parts = [Replicas.partition(n, r, world) for r in range(world)]
    assert [i for p in parts for i in p] == list(range(n))
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
