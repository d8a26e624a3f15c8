"""Numpy restatement of block FSAI (factorised sparse approximate inverse, Kolotilina and
Yeremin) on a node-block lower pattern. Test infrastructure only: the checker for the GPU
setup kernel (mphyfem_b200/csrc/fsai.cu), not part of the product.

The reference has no such preconditioner (its PC comes from PETSc options,
src/mySolvers/SolverPetsc.cpp:117-140); this file restates the published algorithm:
for block row n with lower pattern P (neighbour nodes m <= n, n last, at most max_lower of the
largest), solve A[P,P] Y = E_n, factor Y_nn = L L^T, and set G[n, P] = L^{-1} Y^T.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def full_operator(n_node, fixed, rowptr, col, val):
    """The node-major operator with prescribed DOFs as identity rows/columns (how the GPU stores it)."""
    nd = 3 * n_node
    free = np.flatnonzero(fixed == 0)
    Af = sp.csr_matrix((val, col, rowptr), shape=(len(free), len(free))).tocoo()
    rows = np.concatenate([free[Af.row], np.flatnonzero(fixed)])
    cols = np.concatenate([free[Af.col], np.flatnonzero(fixed)])
    vals = np.concatenate([Af.data, np.ones(int(fixed.sum()))])
    return sp.csr_matrix((vals, (rows, cols)), shape=(nd, nd))


def block_fsai(A_full, node_nbrs, max_lower=16):
    """node_nbrs[n]: ascending neighbour nodes of n. Returns (rowptr, col, blocks[n_lower,3,3])."""
    A = A_full.tocsr()
    n_node = len(node_nbrs)
    rowptr = [0]
    cols, blocks = [], []
    for n in range(n_node):
        lower = [m for m in node_nbrs[n] if m <= n][-max_lower:]
        dofs = np.concatenate([np.arange(3 * m, 3 * m + 3) for m in lower])
        M = A[dofs][:, dofs].toarray()
        N = len(dofs)
        E = np.zeros((N, 3))
        E[N - 3:, :] = np.eye(3)
        try:
            L = np.linalg.cholesky(M)
            Y = np.linalg.solve(L.T, np.linalg.solve(L, E))
            Ynn = 0.5 * (Y[N - 3:] + Y[N - 3:].T)
            Ln = np.linalg.cholesky(Ynn)
            G = np.linalg.solve(Ln, Y.T)  # 3 x N
        except np.linalg.LinAlgError:
            G = np.zeros((3, N))
            d = np.abs(np.diag(M)[N - 3:])
            G[:, N - 3:] = np.diag(np.where(d > 0, 1.0 / np.sqrt(d), 1.0))
        for k, m in enumerate(lower):
            cols.append(m)
            blocks.append(G[:, 3 * k:3 * k + 3])
        rowptr.append(len(cols))
    return np.array(rowptr), np.array(cols, np.int32), np.array(blocks)


def node_neighbours(conn, n_node):
    nb = [set() for _ in range(n_node)]
    for el in conn:
        for a in el:
            nb[a].update(int(b) for b in el)
    return [sorted(s) for s in nb]
