"""Exact diagonalisation of the J1-J2 Heisenberg model in the Sz = 0 sector (TEST INFRASTRUCTURE).

Pins the oracle's local energy: the Hamiltonian matrix is built here independently of the oracle,
from the bond list of bond_map (calc_phys_quantity.f90:382-427) and the matrix elements of
calc_local_energy_correlation (calc_phys_quantity.f90:331-375):

    <x|H|x>  = sum_bonds J sigma_i sigma_j              (Pauli units)
    <x'|H|x> = 2 J s_bond   for x' = x with the antiparallel spins i, j exchanged,
               s_bond = -1 on J1 bonds (Marshall gauge on sublattice B), +1 on J2 bonds.

``gauge=False`` gives the ungauged H = sum J sigma_i . sigma_j, unitarily equivalent to the gauged
form (U = prod_{i in B} sigma^z_i), so both have the same spectrum.
"""
from __future__ import annotations

import itertools

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def bonds(L: int):
    """(i1, i2, J-kind, sign) for i0 = 1..4 and every site, 0-based sites i = ix*L + iy."""
    out = []
    for i0 in (1, 2, 3, 4):
        for i1 in range(L * L):
            ix, iy = divmod(i1, L)
            if i0 == 1:
                ix = (ix + 1) % L
            elif i0 == 2:
                iy = (iy + 1) % L
            elif i0 == 3:
                ix, iy = (ix + 1) % L, (iy + 1) % L
            else:
                ix, iy = (ix + 1) % L, (iy - 1) % L
            out.append((i1, ix * L + iy, 1 if i0 <= 2 else 2, -1.0 if i0 <= 2 else 1.0))
    return out


def sz0_basis(N: int) -> np.ndarray:
    """All configurations with N/2 up spins, as rows of +-1 (lexicographic in the up positions)."""
    confs = []
    for ups in itertools.combinations(range(N), N // 2):
        x = -np.ones(N, dtype=np.int32)
        x[list(ups)] = 1
        confs.append(x)
    return np.array(confs, dtype=np.int32)


def hamiltonian(L: int, J1: float, J2: float, basis: np.ndarray, gauge: bool = True) -> sp.csr_matrix:
    N = L * L
    weights = (1 << np.arange(N, dtype=np.int64))
    keys = ((basis > 0).astype(np.int64) * weights).sum(axis=1)
    index = {int(k): n for n, k in enumerate(keys)}
    rows, cols, vals = [], [], []
    bl = bonds(L)
    for n, x in enumerate(basis):
        diag = 0.0
        for (i1, i2, kind, sgn) in bl:
            J = J1 if kind == 1 else J2
            diag += J * x[i1] * x[i2]
            if x[i1] != x[i2]:
                y = x.copy()
                y[i1], y[i2] = x[i2], x[i1]
                m = index[int(((y > 0).astype(np.int64) * weights).sum())]
                rows.append(m)
                cols.append(n)
                vals.append(2.0 * J * (sgn if gauge else 1.0))
        rows.append(n)
        cols.append(n)
        vals.append(diag)
    dim = len(basis)
    return sp.csr_matrix((vals, (rows, cols)), shape=(dim, dim))


def ground_state_energy(L: int, J1: float, J2: float, gauge: bool = True) -> float:
    basis = sz0_basis(L * L)
    H = hamiltonian(L, J1, J2, basis, gauge)
    w = spla.eigsh(H, k=1, which="SA", tol=1e-12)[0]
    return float(w[0])
