"""One process per GPU on one node, launched from a plain ``python`` call.

The reference runs replicas as MPI ranks (src/main.c:1140-1430).  Here the
ranks are ``torch.distributed`` processes: ``spawn_local`` starts ``nprocs``
copies of a command with the environment torchrun would give them (RANK,
LOCAL_RANK, WORLD_SIZE, LOCAL_WORLD_SIZE, MASTER_ADDR=127.0.0.1 and a free
MASTER_PORT), forwards rank 0's standard output, and returns the largest
exit status.  A command already running under torchrun (WORLD_SIZE set) is
never re-spawned.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys
import time


def free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def under_launcher() -> bool:
    return "WORLD_SIZE" in os.environ


def spawn_local(nprocs: int, argv: list[str], timeout: float | None = None,
                quiet_ranks: bool = True) -> int:
    """Run ``argv`` (a full command line) as ``nprocs`` ranks on this node.
    Rank 0 writes to this process's stdout; the other ranks' stdout is
    discarded (their stderr is kept).  A rank that exits non-zero, or the
    timeout, ends the others; returns the worst exit status (124 on
    timeout)."""
    port = free_port()
    procs = []
    for r in range(nprocs):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(nprocs),
                   LOCAL_WORLD_SIZE=str(nprocs), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        out = None if r == 0 or not quiet_ranks else subprocess.DEVNULL
        procs.append(subprocess.Popen(argv, env=env, stdout=out))
    rc = 0
    t0 = time.monotonic()
    try:
        while True:
            codes = [p.poll() for p in procs]
            bad = [c for c in codes if c not in (None, 0)]
            if bad:
                rc = max(c if c >= 0 else 128 - c for c in bad)
                break
            if all(c == 0 for c in codes):
                break
            if timeout is not None and time.monotonic() - t0 > timeout:
                rc = 124
                break
            time.sleep(0.1)
    finally:
        for p in procs:
            if p.poll() is None:
                p.terminate()
                try:
                    p.wait(timeout=30)
                except subprocess.TimeoutExpired:
                    p.kill()
    return rc


def main_self(nprocs: int, timeout: float | None = None) -> int:
    """Re-run the current script (sys.argv) as ``nprocs`` ranks."""
    return spawn_local(nprocs, [sys.executable, *sys.argv], timeout=timeout)
