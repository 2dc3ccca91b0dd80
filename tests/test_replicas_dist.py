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
PKG = os.path.dirname(os.path.dirname(os.path.abspath(dq.__file__)))
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


def test_spawn_local_runs_a_gloo_world_of_two(tmp_path):
    """bench.py --gpus N spawns its own ranks when not under torchrun
    (dqmc_b200.launch): the children get RANK/WORLD_SIZE/MASTER_* and form a
    process group; rank 0's output comes back, the others' is dropped."""
    import subprocess
    import sys
    script = tmp_path / "child.py"
    script.write_text(
        "import torch, torch.distributed as dist\n"
        "dist.init_process_group('gloo')\n"
        "t = torch.tensor([float(dist.get_rank() + 1)])\n"
        "dist.all_reduce(t)\n"
        "print('rank', dist.get_rank(), 'of', dist.get_world_size(), 'sum', int(t.item()))\n"
        "dist.destroy_process_group()\n")
    out = subprocess.run([sys.executable, "-c",
                          "import sys; sys.path.insert(0, %r); from dqmc_b200 import launch; "
                          "sys.exit(launch.spawn_local(2, [sys.executable, %r], timeout=120))"
                          % (PKG, str(script))],
                         capture_output=True, text=True, timeout=180)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "rank 0 of 2 sum 3"


def test_spawn_local_reports_a_failing_rank(tmp_path):
    import sys
    from dqmc_b200 import launch
    script = tmp_path / "fail.py"
    script.write_text("import os, sys\nsys.exit(3 if os.environ['RANK'] == '1' else 0)\n")
    assert launch.spawn_local(2, [sys.executable, str(script)], timeout=60) == 3
