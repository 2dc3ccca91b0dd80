"""Replicas across processes, one per GPU.

The reference's MPI runner (SAI-QMC src/main.c:1140-1430) gives each rank a
contiguous range of the nrep replicas of every beta (src/replica_mpi.c:13-37),
runs them with no exchange, and gathers per replica and bin the 8 bin
doubles (sign-weighted sums, accepted, attempts), the bin counts and the
S(q) numerators to rank 0 in replica-major order (MPI_Gatherv,
src/main.c:1404-1420); rank 0 alone forms the jackknife rows.  Here a rank is
a process driving one engine on its own GPU (torch.distributed over NCCL;
gloo for the host logic on CPU), the ownership comes from the same C helpers
as the dqmc_gpu driver's ``gpu_devices`` split, and the end-of-run gather is
one ``gather_object`` to rank 0.
"""
import ctypes as C

import numpy as np

from . import NBIN_FIELDS, Engine, chain_lattice, lib, square_lattice

_bound = False


def _host():
    global _bound
    L = lib()
    if not _bound:
        L.dqmc_replica_rank_range.argtypes = [C.c_int] * 3 + [C.POINTER(C.c_int)] * 2
        L.dqmc_replica_rank_for_replica.argtypes = [C.c_int] * 3
        L.dqmc_replica_gather_layout.argtypes = [C.c_int] * 4 + [C.c_void_p] * 2
        L.dqmc_replica_seed.restype = C.c_ulonglong
        L.dqmc_replica_seed.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
        L.dqmc_bin_values.argtypes = [C.c_void_p, C.c_void_p]
        L.dqmc_format_row.argtypes = [C.c_char_p, C.c_size_t, C.c_double] + \
            [C.c_void_p] * 7 + [C.c_int]
        _bound = True
    return L


def rank_range(nrep, nranks, rank):
    """(first replica, count) owned by ``rank`` (src/replica_mpi.c:13-37)."""
    f, c = C.c_int(), C.c_int()
    _host().dqmc_replica_rank_range(nrep, nranks, rank, C.byref(f), C.byref(c))
    return f.value, c.value


def rank_for_replica(nrep, nranks, replica):
    """Owner rank of a replica, -1 if out of range (src/replica_mpi.c:39-53)."""
    return _host().dqmc_replica_rank_for_replica(nrep, nranks, replica)


def gather_layout(nrep, nbin, nranks, width):
    """Per-rank element counts and displacements of a replica-major
    (replica, bin, width) gather (src/replica_mpi.c:55-89)."""
    rc = np.zeros(nranks, np.int32)
    dp = np.zeros(nranks, np.int32)
    if _host().dqmc_replica_gather_layout(nrep, nbin, nranks, width, rc.ctypes.data,
                                          dp.ctypes.data):
        raise ValueError("gather layout overflows int")
    return rc, dp


def gather_bins(local, nrep, rank, world, group=None):
    """Gather the local replicas' bins to rank 0 in replica order.

    ``local`` maps a name to an array whose first axis is this rank's
    replicas (its rank_range, in order); rank 0 gets each name concatenated
    over ranks, i.e. indexed by global replica, and checks every rank sent
    the count the ownership rule gives it.  Other ranks get None.
    """
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None
    for r, p in enumerate(parts):
        _, count = rank_range(nrep, world, r)
        for k, v in p.items():
            if len(v) != count:
                raise RuntimeError(f"rank {r} sent {len(v)} replicas of {k}, owns {count}")
    return {k: np.concatenate([p[k] for p in parts], axis=0) for k in local}


def observables_row(T, scal, nbin_total):
    """The reference's 14-column observables row (src/main.c:221-265) from
    gathered bins ``scal`` of shape (nrep, nbin, NBIN_FIELDS)."""
    L = _host()
    flat = np.ascontiguousarray(scal.reshape(-1, NBIN_FIELDS))
    series = np.zeros((7, len(flat)))
    v = np.zeros(6)
    for o, bf in enumerate(flat):
        bf = np.ascontiguousarray(bf)
        if L.dqmc_bin_values(bf.ctypes.data, v.ctypes.data):
            raise RuntimeError(f"invalid bin {o}")
        series[:6, o] = v
        att = bf[8]
        series[6, o] = bf[7] / att if att > 0 else 0.0
    series = np.ascontiguousarray(series)
    buf = C.create_string_buffer(512)
    if L.dqmc_format_row(buf, 512, T, *[series[i].ctypes.data for i in range(7)], nbin_total):
        raise RuntimeError("non-finite or empty jackknife input")
    return buf.value.decode()


def run(rank, world, device, lattice="square", Lx=4, Ly=4, U=4.0, dtau=0.1,
        beta_list=(1.0,), nrep=2, seed=1, nwarm=20, nmeas=40, nbin=4, stab=8,
        delay_rank=0, group=None):
    """One rank's share of a replica run: for every beta the rank's replica
    range on ``device``, then the gather; rank 0 returns the observables
    rows (one per beta), other ranks None."""
    if lattice == "chain":
        T, bp = chain_lattice(Lx)
        Ly = 1
    else:
        T, bp = square_lattice(Lx, Ly)
    first, count = rank_range(nrep, world, rank)
    L = _host()
    Ltrs = [int(round(b / dtau)) for b in beta_list]
    local = {"scal": np.zeros((count, len(beta_list), nbin, NBIN_FIELDS)),
             "status": np.zeros((count, len(beta_list)), np.int64)}
    if count:
        eng = Engine(device=device, delay_rank=delay_rank)
        m = eng.add_model(T, bp, U, dtau, Lx, Ly)
        for b, Ltr in enumerate(Ltrs):
            for r in range(first, first + count):
                eng.add_chain(m, Ltr, stab, L.dqmc_replica_seed(seed, b, r))
        eng.prepare(nbin)
        eng.sweep(nwarm)
        for bi in range(nbin):
            eng.sweep_measure(nmeas // nbin, bi)
        eng.sync()
        for b in range(len(Ltrs)):
            for j in range(count):
                c = b * count + j
                sc, _, _ = eng.bins(c)
                local["scal"][j, b] = sc
                local["status"][j, b] = eng.counters(c)["status"]
        eng.close()
    allb = gather_bins(local, nrep, rank, world, group)
    if allb is None:
        return None
    if np.any(allb["status"]):
        raise RuntimeError("a replica failed")
    rows = []
    for b, Ltr in enumerate(Ltrs):
        rows.append(observables_row(1.0 / (Ltr * dtau), allb["scal"][:, b], nrep * nbin))
    return rows
