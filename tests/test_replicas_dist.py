"""Replica ownership and the end-of-run gather across processes (gloo, CPU).

Two ranks each build the bins of their own replica range (src/replica_mpi.c
ownership) and gather them to rank 0, which must see exactly the
replica-major arrays of a single-process run and format the same
observables rows (the reference's MPI path, src/main.c:1140-1430).
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

dq = pytest.importorskip("dqmc_b200")
from dqmc_b200 import replicas  # noqa: E402

NREP, NBETA, NBIN = 5, 2, 3


def fake_bins(replica):
    """Valid bins of one replica: one sample each, sign +-1, deterministic."""
    s = np.zeros((NBETA, NBIN, dq.NBIN_FIELDS))
    for b in range(NBETA):
        for bi in range(NBIN):
            sign = -1.0 if (replica + b + bi) % 4 == 3 else 1.0
            x = 0.1 * replica + 0.01 * b + 0.001 * bi
            s[b, bi, :6] = sign * np.array([-1.0 + x, -2.0 + x, -0.5 + x, 1.0 + x, 0.2 + x, 1.0])
            s[b, bi, 6] = 1.0
            s[b, bi, 7], s[b, bi, 8] = 3 + replica, 10 + bi
    return s


def worker(rank, world, store, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"file://{store}", rank=rank,
                            world_size=world)
    try:
        first, count = replicas.rank_range(NREP, world, rank)
        local = {"scal": np.stack([fake_bins(r) for r in range(first, first + count)])
                 if count else np.zeros((0, NBETA, NBIN, dq.NBIN_FIELDS)),
                 "owner": np.full(count, rank)}
        got = replicas.gather_bins(local, NREP, rank, world)
        if rank == 0:
            rows = [replicas.observables_row(1.0 / (b + 1), got["scal"][:, b], NREP * NBIN)
                    for b in range(NBETA)]
            q.put((got["scal"], got["owner"], rows))
        else:
            q.put(got)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gather_assembles_replica_major(tmp_path, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "store")
    ps = [ctx.Process(target=worker, args=(r, world, store, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = [o for o in out if o is not None]
    assert len(full) == 1
    scal, owner, rows = full[0]
    want = np.stack([fake_bins(r) for r in range(NREP)])
    np.testing.assert_array_equal(scal, want)
    assert list(owner) == [replicas.rank_for_replica(NREP, world, r) for r in range(NREP)]
    serial = [replicas.observables_row(1.0 / (b + 1), want[:, b], NREP * NBIN)
              for b in range(NBETA)]
    assert rows == serial
    assert len(rows[0].split()) == 14


def test_gather_layout_matches_ranges():
    for nrep, world in [(10, 3), (2, 4), (5, 2)]:
        rc, dp = replicas.gather_layout(nrep, NBIN, world, dq.NBIN_FIELDS)
        for r in range(world):
            first, count = replicas.rank_range(nrep, world, r)
            assert rc[r] == count * NBIN * dq.NBIN_FIELDS
            assert dp[r] == first * NBIN * dq.NBIN_FIELDS
