"""Numpy restatement of the two-level additive preconditioner
    M^{-1} = D^{-1} + Z (Z^T A Z)^{-1} Z^T
with Z the six rigid-body modes (or the twelve linear-displacement modes) of every box of a
regular grid of boxes over the reference coordinates (zero on prescribed DOFs). Test infrastructure only: the checker for
mphyfem_b200/csrc/coarse.cu and the coarse path of csrc/krylov.cu. The reference has no such
preconditioner (its PC comes from PETSc options, src/mySolvers/SolverPetsc.cpp:117-140).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp


def aggregates(coords, grid):
    lo, hi = coords.min(0), coords.max(0)
    L = np.maximum(hi - lo, 1e-30)
    g = np.asarray(grid)
    c = np.minimum(((coords - lo) / L * g).astype(int), g - 1)
    return c[:, 0] + g[0] * (c[:, 1] + g[1] * c[:, 2]), L / g


def prolongation(coords, fixed, grid, modes=6):
    """Z: 6 rigid-body modes per box (translations, rotations about the centroid), or 12 linear
    modes u = a + B d (a at columns 0..2, B_ck at 3 + 3c + k), d = (x - centroid) / box diagonal."""
    if modes == 12:
        return _prolongation_linear(coords, fixed, grid)
    agg, box = aggregates(coords, grid)
    n_agg = int(np.prod(grid))
    boxd = np.sqrt((box ** 2).sum())
    cent = np.zeros((n_agg, 3))
    np.add.at(cent, agg, coords)
    cnt = np.bincount(agg, minlength=n_agg)
    cent /= np.maximum(cnt, 1)[:, None]
    d = (coords - cent[agg]) / boxd
    n = coords.shape[0]
    rows, cols, vals = [], [], []
    modes = [((0, 1.0, None),), ((1, 1.0, None),), ((2, 1.0, None),),
             ((0, -1.0, 1), (1, 1.0, 0)), ((1, -1.0, 2), (2, 1.0, 1)), ((0, 1.0, 2), (2, -1.0, 0))]
    for j, terms in enumerate(modes):
        for comp, sgn, dcomp in terms:
            v = sgn * (np.ones(n) if dcomp is None else d[:, dcomp])
            rows.append(3 * np.arange(n) + comp)
            cols.append(6 * agg + j)
            vals.append(v)
    Z = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(3 * n, 6 * n_agg))
    return sp.diags((np.asarray(fixed) == 0).astype(float)) @ Z


def _prolongation_linear(coords, fixed, grid):
    agg, box = aggregates(coords, grid)
    n_agg = int(np.prod(grid))
    boxd = np.sqrt((box ** 2).sum())
    cent = np.zeros((n_agg, 3))
    np.add.at(cent, agg, coords)
    cnt = np.bincount(agg, minlength=n_agg)
    cent /= np.maximum(cnt, 1)[:, None]
    d = (coords - cent[agg]) / boxd
    n = coords.shape[0]
    rows, cols, vals = [], [], []
    for comp in range(3):
        rows.append(3 * np.arange(n) + comp)
        cols.append(12 * agg + comp)
        vals.append(np.ones(n))
        for k in range(3):
            rows.append(3 * np.arange(n) + comp)
            cols.append(12 * agg + 3 + 3 * comp + k)
            vals.append(d[:, k])
    Z = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(3 * n, 12 * n_agg))
    return sp.diags((np.asarray(fixed) == 0).astype(float)) @ Z


def preconditioner(A, coords, fixed, grid, modes=6):
    """Returns a function r -> M^{-1} r (A: the node-major operator with identity prescribed rows)."""
    Z = prolongation(coords, fixed, grid, modes)
    E = (Z.T @ A @ Z).toarray()
    dg = np.diag(E)
    keep = dg > 1e-13 * dg.max()
    Zk = Z[:, keep]
    cf = sla.cho_factor(E[np.ix_(keep, keep)])
    d = A.diagonal()
    return lambda r: r / d + Zk @ sla.cho_solve(cf, Zk.T @ r)


def pcg(A, b, Minv, rtol=1e-8, maxit=100000, norm_type=0):
    """KSPCG semantics, x0 = 0; the test on ||z|| (norm_type 0, KSP_NORM_PRECONDITIONED) or on
    ||r|| (norm_type 1, KSP_NORM_UNPRECONDITIONED)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = Minv(r)
    p = z.copy()
    rz = r @ z
    dp0 = np.linalg.norm(r if norm_type == 1 else z)
    for i in range(maxit):
        q = A @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        z = Minv(r)
        if np.linalg.norm(r if norm_type == 1 else z) <= rtol * dp0:
            return x, i + 1
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, maxit
