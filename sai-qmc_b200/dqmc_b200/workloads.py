"""Chain lists of the batched workloads the engine is measured and tested on.

Each chain is what one invocation of the reference program runs with
``beta_list=<beta>`` and ``seed=<seed>``: beta index 0 keeps the seed
unchanged (replica_seed, src/replica.c:17-34), so a chain here and that
invocation share their xoshiro256** stream, field and trajectory.
"""
from __future__ import annotations

import numpy as np

DTAU = 0.1


def uneven_batch(count=64, draw_seed=2024):
    """64 independent chains of uneven n and L in one launch: square periodic
    lattices cycling through 4x4, 6x6, 8x8, 10x10 and 12x12 (n = 16..144),
    U drawn from {2, 4, 6} and beta from {1, 2, 4, 6, 8, 10} (L = 10..100 at
    dtau = 0.1) by a fixed seeded draw, seeds 1..64."""
    rng = np.random.default_rng(draw_seed)
    us = rng.choice([2.0, 4.0, 6.0], size=count)
    betas = rng.choice([1.0, 2.0, 4.0, 6.0, 8.0, 10.0], size=count)
    out = []
    for c in range(count):
        Lx = (4, 6, 8, 10, 12)[c % 5]
        beta = float(betas[c])
        out.append(dict(Lx=Lx, n=Lx * Lx, U=float(us[c]), dtau=DTAU, beta=beta,
                        L=int(round(beta / DTAU)), seed=c + 1))
    return out


def chain_cost(n, L):
    """Relative cost of one sweep of a chain: the wrap and B-block products
    dominate, O(n^3 L)."""
    return float(n) ** 3 * L


# Large low-temperature batch: 24x24 periodic square lattice (n = 576),
# U = 8, dtau = 0.05, beta = 10 (L = 200), stabilization every 5 slices,
# delay rank 64, seeds 101..108.
LOWT = dict(Lx=24, U=8.0, dtau=0.05, beta=10.0, L=200, stab=5, delay_rank=64,
            seeds=tuple(range(101, 109)))
