"""The entry point that allocates no device memory, dqmc_udv_green_noalloc.

Some callers cannot let a library call cudaMalloc: their device memory is
owned by their own allocator (a framework's caching pool that has reserved
the GPU, where an outside allocation fails or fragments the pool).  For them the UDV -> G computation is offered
with its scratch held in a fixed array inside the library (n <= 128).  These
checks call it through the C ABI and require the same G and sign as the
allocating entry point dqmc_udv_green, at the tolerance of the reference's
own fixture test (1e-9 relative), on two different calls in a row -- the
second one must not see anything the first left in the shared array.  The
array is placed on the device by the first call there; after that, calls
must take no device memory (free memory unchanged) and must leave the
caller's current device as it was.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")


def random_udv(n, seed):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((n, n)))
    D = np.exp(rng.uniform(-40.0, 40.0, n)) * rng.choice([-1.0, 1.0], n)
    T = np.triu(rng.uniform(-1.0, 1.0, (n, n)), 1) + np.eye(n)
    return U, D, T


def test_noalloc_matches_allocating_entry_point_twice():
    g = golden("udv_fixture")
    cases = [(g["U"], g["D"], g["T"]), random_udv(dq_max(), 5)]
    for U, D, T in cases:
        G_ref, s_ref = dq.udv_green(U, D, T)
        G, s = dq.udv_green_noalloc(U, D, T)
        assert s == s_ref and s != 0
        assert rel_err(G, G_ref) <= 1e-9
    # the reference fixture's own answer as well
    G, s = dq.udv_green_noalloc(g["U"], g["D"], g["T"])
    assert s == int(g["det_sign"]) and rel_err(G, g["G"]) <= 1e-9


def test_noalloc_takes_no_device_memory_after_the_first_call():
    torch = pytest.importorskip("torch")
    U, D, T = random_udv(64, 9)
    dq.udv_green_noalloc(U, D, T)          # places the array and the kernel
    torch.cuda.synchronize(0)
    for seed in (10, 11, 12):
        U, D, T = random_udv(96, seed)
        G_ref, s_ref = dq.udv_green(U, D, T) if seed == 10 else (None, None)
        free_before, _ = torch.cuda.mem_get_info(0)
        G, s = dq.udv_green_noalloc(U, D, T)
        free_after, _ = torch.cuda.mem_get_info(0)
        assert free_after == free_before
        if G_ref is not None:
            assert s == s_ref and rel_err(G, G_ref) <= 1e-9


def test_noalloc_restores_the_current_device():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    U, D, T = random_udv(32, 3)
    dq.udv_green_noalloc(U, D, T, device=0)
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_sizes_beyond_its_limit():
    U, D, T = random_udv(dq_max() + 1, 1)
    with pytest.raises(dq.DqmcError, match="scratch limit"):
        dq.udv_green_noalloc(U, D, T)


def dq_max():
    return 128
