"""The exact-diagonalization checker (tests/ed_hubbard.py) against the
reference's own FullDiag table for the 4-site U=4 chain
(data/benchmark_L468_U4_full_diag_20260626/reference/L4_U4_FullDiag.dat,
rows copied to tests/golden/ed_chain4_u4.npz by make_golden.py).  The GPU
long-run test compares the full C1 workload with this ED."""
import numpy as np

from conftest import golden
from ed_hubbard import HubbardED, chain_hopping


def test_ed_matches_reference_fulldiag_table():
    g = golden("ed_chain4_u4")
    ed = HubbardED(chain_hopping(4), float(g["U"]), float(g["mu"]))
    for k, T in enumerate(g["T"]):
        E, N, D = ed.thermal(1.0 / T)
        assert abs(E - g["E_gc"][k]) < 1e-9, (T, E, g["E_gc"][k])
        # the table's N and D_total carry up to ~3e-7 of its own numerical
        # noise (its N drifts from 4 by 1e-8); E_gc agrees to 1e-10
        assert abs(N - g["N"][k]) < 1e-7 and abs(D - g["D_total"][k]) < 5e-7


def test_ed_free_fermions():
    """U = 0: E_gc = sum_k e_k 2 f(e_k) for the chain's single-particle
    levels (mu = 0)."""
    T = chain_hopping(4)
    ed = HubbardED(T, 0.0, 0.0)
    e = np.linalg.eigvalsh(T)
    for beta in (0.5, 2.0, 8.0):
        f = 1.0 / (np.exp(beta * e) + 1.0)
        E, N, _ = ed.thermal(beta)
        assert abs(E - 2 * np.sum(e * f)) < 1e-10 and abs(N - 2 * np.sum(f)) < 1e-10
