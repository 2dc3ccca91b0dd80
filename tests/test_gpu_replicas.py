"""The one-process-per-GPU replica runner on the GPU: two gloo ranks whose
engines share the one device (independent chains, no kernel waits on
another) give rank 0 the same observables rows as one rank running every
replica."""
import multiprocessing as mp

import pytest

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

ARGS = dict(lattice="square", Lx=4, Ly=4, U=4.0, dtau=0.1, beta_list=(0.5, 1.0), nrep=3,
            seed=5, nwarm=10, nmeas=20, nbin=4, stab=5)


def worker(rank, world, store, q):
    import torch.distributed as dist
    from dqmc_b200 import replicas
    dist.init_process_group("gloo", init_method=f"file://{store}", rank=rank,
                            world_size=world)
    try:
        q.put((rank, replicas.run(rank, world, 0, **ARGS)))
    finally:
        dist.destroy_process_group()


def launch(world, store):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=worker, args=(r, world, store, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_two_ranks_equal_one(tmp_path):
    one = launch(1, str(tmp_path / "s1"))
    two = launch(2, str(tmp_path / "s2"))
    assert two[1] is None
    assert one[0] == two[0]
    assert len(one[0]) == 2 and all(len(r.split()) == 14 for r in one[0])
