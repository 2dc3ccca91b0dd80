"""Exact diagonalization of a small Hubbard chain (a known-answer checker).

Grand-canonical H = sum_{ij,s} t_ij c+_is c_js + U sum_i n_iu n_id - mu N on
the 4^L Fock space (L <= 5), built on occupation bit strings with the
fermionic sign of an ordered mode list (up modes 0..L-1, down modes
L..2L-1).  Thermal averages at inverse temperature beta give the columns
the reference's FullDiag tables report (E_gc = <H>, N, D_total =
sum_i <n_iu n_id>; data/benchmark_L468_U4_full_diag_20260626/README.md).
"""
from __future__ import annotations

import numpy as np


def chain_hopping(L, t=-1.0, pbc=True):
    T = np.zeros((L, L))
    for x in range(L):
        j = x + 1 if x + 1 < L else (0 if pbc and L > 1 else -1)
        if j >= 0:
            T[x, j] += t
            T[j, x] += t
    return T


class HubbardED:
    def __init__(self, T, U, mu):
        L = T.shape[0]
        nm = 2 * L
        dim = 1 << nm
        H = np.zeros((dim, dim))
        occ = np.array([[(s >> m) & 1 for m in range(nm)] for s in range(dim)])
        for s in range(dim):
            for spin in range(2):
                for i in range(L):
                    mi = i + spin * L
                    if not occ[s, mi]:
                        continue
                    for j in range(L):
                        if T[j, i] == 0.0:
                            continue
                        mj = j + spin * L
                        if mj == mi:
                            H[s, s] += T[j, i]
                            continue
                        if occ[s, mj]:
                            continue
                        # c+_j c_i: the sign counts the occupied modes
                        # strictly between i and j in the ordered list
                        lo, hi = min(mi, mj), max(mi, mj)
                        between = int(occ[s, lo + 1:hi].sum())
                        s2 = s ^ (1 << mi) ^ (1 << mj)
                        H[s2, s] += T[j, i] * (-1.0) ** between
        dbl = (occ[:, :L] * occ[:, L:]).sum(axis=1).astype(float)
        num = occ.sum(axis=1).astype(float)
        H += np.diag(U * dbl - mu * num)
        self.E, self.V = np.linalg.eigh(H)
        self.dbl_k = np.einsum("ik,i,ik->k", self.V, dbl, self.V)
        self.num_k = np.einsum("ik,i,ik->k", self.V, num, self.V)
        self.L, self.mu = L, mu

    def thermal(self, beta):
        """(E_gc, N, D_total) at inverse temperature beta."""
        w = np.exp(-beta * (self.E - self.E.min()))
        Z = w.sum()
        return (float((w * self.E).sum() / Z), float((w * self.num_k).sum() / Z),
                float((w * self.dbl_k).sum() / Z))
