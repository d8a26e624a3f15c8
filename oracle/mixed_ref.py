"""Mixed u-p problems (Elem_Solid_3D_Mixed1: tet10 displacement with linear vertex pressure, or
hex27 displacement with trilinear corner pressure): numpy/scipy restatement of the two-field
assembly and of the Newton load stepping with pressure unknowns.

TEST INFRASTRUCTURE ONLY: the checker for the GPU mixed path (tests/). The element matrices come
from the C oracle (orc_problem_elements_mixed); this module restates:

* prepareDataForMixedElements (femSolidmechanics1.cpp:274-380): the pressure nodes are the
  elements' vertex nodes, numbered in ascending global node order; no pressure is prescribed;
* the matrix pattern and SolverPetsc::assembleMatrixAndVector2field (femSolidmechanics2.cpp:
  327-371, SolverPetsc.cpp:434-502): the unknowns are the free displacement DOFs (the
  displacement pattern's numbering) followed by the pressure DOFs at offset dispDOF;
  prescribed displacement rows and columns are left out; the reactions collect every FlocalU;
* solveWithNewtonRaphson (femSolidmechanics2.cpp:730-851) with factoriseSolveAndUpdate
  (:1127-1200): the norm runs over both fields, the update adds the pressure part to the
  vertex pressures, a cut restores displacements and pressures (SolutionDataSolid::reset).
  The linear solve is a sparse LU, as the reference's sample options run MUMPS LU
  (sample-inputs/.../petsc_options.dat: -ksp_type preonly -pc_type lu).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import binding as B


def pressure_dofs(prob):
    """(pressure nodes ascending, id_pres [n_node] with -1 off the pressure nodes)."""
    pn = np.unique(np.asarray(prob.conn)[:, :B.mixed_pressure_nodes(prob.npe)])
    idp = -np.ones(prob.n_node, np.int64)
    idp[pn] = np.arange(len(pn))
    return pn, idp


class MixedProblem:
    def __init__(self, prob):
        if prob.npe not in (10, 27):
            raise ValueError("mixed u-p problems are tet10 or hex27")
        self.prob = prob
        self.ns, self.NP = 3 * prob.npe, B.mixed_pressure_nodes(prob.npe)
        self.op = B.OracleProblem(prob)
        self.afs, self.fav, _, _ = self.op.pattern()
        self.nu = self.op.n_free
        self.pn, self.idp = pressure_dofs(prob)
        self.np = len(self.pn)
        lib = B.lib()
        lib.orc_problem_elements_mixed.argtypes = [C.c_void_p, B._d, B._d, B._d, B._d, B._d, B._d, B._d, B._d, C.c_int]
        lib.orc_problem_elements_mixed.restype = C.c_int64

    def elements(self, disp, disp_prev, pres, nthreads=1):
        ne, ns, NP = self.prob.n_elem, self.ns, self.NP
        Kuu, Kup, Kpp = np.zeros((ne, ns, ns)), np.zeros((ne, ns, NP)), np.zeros((ne, NP, NP))
        FU, FP = np.zeros((ne, ns)), np.zeros((ne, NP))
        d, dp, p = (np.ascontiguousarray(a, np.float64) for a in (disp, disp_prev, pres))
        bad = B.lib().orc_problem_elements_mixed(self.op.h, B._p(d, B._d), B._p(dp, B._d), B._p(p, B._d),
                                                 B._p(Kuu, B._d), B._p(Kup, B._d), B._p(Kpp, B._d), B._p(FU, B._d),
                                                 B._p(FP, B._d), nthreads)
        return Kuu, Kup, Kpp, FU, FP, int(bad)

    def assemble(self, disp, disp_prev, pres, nthreads=1):
        """(A [nu+np, nu+np] CSR, rhs [nu+np], reactions [3 n_node], first bad element or -1)."""
        Kuu, Kup, Kpp, FU, FP, bad = self.elements(disp, disp_prev, pres, nthreads)
        nu, n, ns, NP = self.nu, self.nu + self.np, self.ns, self.NP
        fav = self.fav.astype(np.int64)
        pdof = nu + self.idp[np.asarray(self.prob.conn)[:, :NP]]  # [ne, NP]
        rows, cols, vals = [], [], []

        def add(r, c, v):
            m = (r >= 0) & (c >= 0)
            rows.append(r[m])
            cols.append(c[m])
            vals.append(v[m])

        add(np.repeat(fav, ns, axis=1).ravel(), np.tile(fav, (1, ns)).ravel(), Kuu.ravel())
        add(np.repeat(fav, NP, axis=1).ravel(), np.tile(pdof, (1, ns)).ravel(), Kup.ravel())
        add(np.tile(pdof, (1, ns)).ravel(), np.repeat(fav, NP, axis=1).ravel(), Kup.ravel())
        add(np.repeat(pdof, NP, axis=1).ravel(), np.tile(pdof, (1, NP)).ravel(), Kpp.ravel())
        A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
        rhs = np.zeros(n)
        m = fav >= 0
        np.add.at(rhs, fav[m], FU[m])
        np.add.at(rhs, pdof.ravel(), FP.ravel())
        gdof = (3 * np.asarray(self.prob.conn, np.int64)[:, :, None] + np.arange(3)).reshape(-1, ns)
        reac = np.zeros(self.prob.n_dof)
        np.add.at(reac, gdof.ravel(), FU.ravel())
        return A, rhs, reac, bad

    def newton(self, tol_rel=None, tol_abs=0.0, max_newton=10, nthreads=1):
        """(disp [3 n_node], pres [n_node], rows [step, iter, ||R||])."""
        p = self.prob
        tol_rel = p.newton_rtol if tol_rel is None else tol_rel
        disp, pres = np.zeros(p.n_dof), np.zeros(p.n_node)
        fext = np.asarray(p.fnodal, np.float64)[self.afs]
        t, dt, dt0, steps, hist = 0.0, p.dt, p.dt, 1, []
        while t <= p.t_final - 1e-10 and steps <= p.max_steps:
            t += dt
            lam = t
            disp_prev, pres_prev = disp.copy(), pres.copy()
            converged, norm, norm_prev, tol = False, -1.0, -1.0, tol_abs
            for it in range(1, max_newton + 1):
                A, rhs, _, bad = self.assemble(disp, disp_prev, pres, nthreads)
                if bad >= 0:
                    break
                rhs[:self.nu] += lam * fext
                norm_prev, norm = norm, float(np.linalg.norm(rhs))
                if it == 1:
                    tol = max(tol_abs, tol_rel * norm)
                stop = False
                if norm < tol:
                    converged = stop = True
                elif it > 3 and (np.isnan(norm) or (norm_prev > -0.1 and norm / norm_prev > 1e7)):
                    stop = True
                else:
                    x = spla.spsolve(A.tocsc(), rhs)
                    disp[self.afs] += x[:self.nu]
                    pres[self.pn] += x[self.nu:]
                hist.append((steps, it, norm))
                if stop:
                    break
            if converged:
                steps += 1
            else:
                t -= dt
                dt *= 0.5
                if dt < 0.01 * dt0:
                    raise RuntimeError("oracle mixed Newton: time step size fell below 1% of the initial value")
                disp, pres = disp_prev, pres_prev
        return disp, pres, np.array(hist, dtype=np.float64).reshape(-1, 3)
