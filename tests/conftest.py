import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sai-qmc_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)


CASES = ["chain4_b2", "chain4_u0", "sq4_b4", "sq6_b2", "sq8_b4"]


def case_args(g):
    kind, Lx, Ly, L, stab, seed, sweeps = (int(x) for x in g["params"])
    return dict(kind=kind, Lx=Lx, Ly=Ly, U=float(g["U"]), dtau=float(g["dtau"]),
                L=L, stab=stab, seed=seed, sweeps=sweeps, selector=str(g["selector"]))


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="session")
def oracle():
    from oracle import build as ob
    ob.build_oracle()
    from oracle.bind import Oracle
    return Oracle()


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
