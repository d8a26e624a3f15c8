"""ctypes binding of the CPU FP64 oracle (oracle/liboracle.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs, never by the product package. Parity status: unpinned against the
reference binary (it cannot be built here); see oracle/oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)


class NewtonOpts(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("t_final", C.c_double), ("max_steps", C.c_int),
        ("max_newton", C.c_int), ("tol_rel", C.c_double), ("tol_abs", C.c_double),
        ("cg_rtol", C.c_double), ("cg_maxit", C.c_int), ("nthreads", C.c_int),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (system g++)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f))
                                          for f in ("oracle.cpp", "oracle.h", "Makefile"))):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_nh_stress_tangent.argtypes = [_d, C.c_double, C.c_double, C.c_int, _d, _d]
        L.orc_set_consistent_tangent.argtypes = [C.c_int]
        L.orc_set_pattern_mode.argtypes = [C.c_int]
        L.orc_vol_dU.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_vol_dU.restype = C.c_double
        L.orc_vol_d2U.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_vol_d2U.restype = C.c_double
        L.orc_elem_stiffness_residual.argtypes = [C.c_int, _d, _d, C.c_double, C.c_double, C.c_int, _d, _d]
        L.orc_gauss_rule.argtypes = [C.c_int, _d, _d, _d, _d]
        L.orc_material_stress_tangent.argtypes = [C.c_int, _d, C.c_double, C.c_int, _d, _d, _d]
        L.orc_elem_stiffness_residual_mat.argtypes = [C.c_int, _d, _d, C.c_int, _d, C.c_double, C.c_int, _d, _d]
        L.orc_problem_set_materials.argtypes = [C.c_void_p, C.c_int, _i32, _d]
        L.orc_material_stress_tangent_mixed.argtypes = [C.c_int, _d, C.c_double, C.c_int, _d, C.c_double, _d, _d]
        L.orc_mixed_constants.argtypes = [C.c_int, C.c_double, C.c_double, _d, _d]
        L.orc_elem_mixed.argtypes = [C.c_int, _d, _d, _d, _d, C.c_int, _d, C.c_double, C.c_int, _d, _d, _d, _d,
                                     _d, _d]
        L.orc_elem_mixed0.argtypes = [C.c_int, _d, _d, _d, C.c_double, C.c_int, _d, C.c_double, C.c_int, _d, _d,
                                      _d, _d, _d]
        L.orc_problem_set_mixed_p0.argtypes = [C.c_void_p, C.c_int]
        L.orc_problem_set_prescribed.argtypes = [C.c_void_p, _d, _d]
        L.orc_problem_p0_pressure.argtypes = [C.c_void_p, _d, _d]
        L.orc_problem_p0_pressure.restype = None
        L.orc_problem_save_step.argtypes = [C.c_void_p, _d]
        L.orc_problem_save_step.restype = None
        L.orc_problem_create.argtypes = [C.c_int, _d, C.c_int, C.c_int, _i32, _i32, C.c_int, _d, _u8]
        L.orc_problem_create.restype = C.c_void_p
        L.orc_problem_destroy.argtypes = [C.c_void_p]
        L.orc_problem_nfree.argtypes = [C.c_void_p]
        L.orc_problem_nnz.argtypes = [C.c_void_p]
        L.orc_problem_nnz.restype = C.c_int64
        L.orc_problem_export_pattern.argtypes = [C.c_void_p, _i32, _i32, _i64, _i32]
        L.orc_problem_elements.argtypes = [C.c_void_p, _d, _d, _d, C.c_int]
        L.orc_problem_elements.restype = C.c_int64
        L.orc_problem_assemble.argtypes = [C.c_void_p, _d, _d, _d, _d, C.c_int]
        L.orc_problem_assemble.restype = C.c_int64
        L.orc_cg_jacobi.argtypes = [C.c_void_p, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int,
                                    C.POINTER(C.c_int), _d]
        L.orc_cg_jacobi_norm.argtypes = [C.c_void_p, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_int), _d]
        L.orc_newton_run.argtypes = [C.c_void_p, _d, C.POINTER(NewtonOpts), _d, _d, C.c_int]
        L.orc_arclength_run.argtypes = [C.c_void_p, _d, C.POINTER(NewtonOpts), _d, _d, C.c_int,
                                        C.POINTER(C.c_int), _d, C.c_int]
        _lib = L
    return _lib


def set_consistent_tangent(on: bool) -> None:
    lib().orc_set_consistent_tangent(1 if on else 0)


def set_pattern_mode(mode: int) -> None:
    lib().orc_set_pattern_mode(int(mode))


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def nh_stress_tangent(F, mu, Kinv, utype=3):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    s, Cm = np.zeros(9), np.zeros(81)
    lib().orc_nh_stress_tangent(_p(F, _d), mu, Kinv, utype, _p(s, _d), _p(Cm, _d))
    return s, Cm.reshape(9, 9)


def elem_stiffness_residual(X, u, mu, Kinv, utype=3):
    X = np.ascontiguousarray(X, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    npe = X.shape[0]
    K, R = np.zeros((3 * npe, 3 * npe)), np.zeros(3 * npe)
    bad = lib().orc_elem_stiffness_residual(npe, _p(X, _d), _p(u, _d), mu, Kinv, utype, _p(K, _d), _p(R, _d))
    return K, R, bad


MAT_NEOHOOKEAN, MAT_MOONEYRIVLIN, MAT_GENT, MAT_ARRUDABOYCE = 0, 1, 2, 3
MAT_NDATA = 4


def _mat_data(data):
    d = np.zeros(MAT_NDATA)
    d[:len(data)] = data
    return d


def material_stress_tangent(model, data, F, Kinv, utype=3):
    """Stress (9) and tangent (9x9) of any hyperelastic model, reference index order."""
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    d = _mat_data(data)
    s, Cm = np.zeros(9), np.zeros(81)
    rc = lib().orc_material_stress_tangent(int(model), _p(d, _d), Kinv, utype, _p(F, _d), _p(s, _d), _p(Cm, _d))
    if rc:
        raise ValueError(f"oracle: unknown material model {model}")
    return s, Cm.reshape(9, 9)


def elem_stiffness_residual_mat(X, u, model, data, Kinv, utype=3):
    X = np.ascontiguousarray(X, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    d = _mat_data(data)
    npe = X.shape[0]
    K, R = np.zeros((3 * npe, 3 * npe)), np.zeros(3 * npe)
    bad = lib().orc_elem_stiffness_residual_mat(npe, _p(X, _d), _p(u, _d), int(model), _p(d, _d), Kinv, utype,
                                                _p(K, _d), _p(R, _d))
    return K, R, bad


def material_stress_tangent_mixed(model, data, F, Kinv, pres, utype=3):
    """Mixed (u-p) branch: the pressure replaces U'(J) in the stress and tangent."""
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    d = _mat_data(data)
    s, Cm = np.zeros(9), np.zeros(81)
    if lib().orc_material_stress_tangent_mixed(int(model), _p(d, _d), Kinv, utype, _p(F, _d), pres, _p(s, _d),
                                               _p(Cm, _d)):
        raise ValueError(f"oracle: unknown material model {model}")
    return s, Cm.reshape(9, 9)


def mixed_pressure_nodes(npe: int) -> int:
    """Pressure nodes of Elem_Solid_3D_Mixed1: the 4 vertices of a tet10, the 8 corners of a hex27."""
    return {10: 4, 27: 8}[npe]


def elem_mixed(X, u, u_prev, pn, model, data, Kinv, utype=3):
    """Mixed u-p element, Elem_Solid_3D_Mixed1: tet10 with linear vertex pressure, or hex27 with
    trilinear corner pressure (P2-P1). Returns Kuu, Kup, Kpu, Kpp, FU, FP, bad."""
    X, u, up, pn = (np.ascontiguousarray(a, dtype=np.float64) for a in (X, u, u_prev, pn))
    npe = X.shape[0]
    if npe not in (10, 27):
        raise ValueError("oracle: the mixed element is tet10 or hex27")
    ns, NP = 3 * npe, mixed_pressure_nodes(npe)
    d = _mat_data(data)
    Kuu, Kup, Kpu, Kpp = np.zeros((ns, ns)), np.zeros((ns, NP)), np.zeros((NP, ns)), np.zeros((NP, NP))
    FU, FP = np.zeros(ns), np.zeros(NP)
    bad = lib().orc_elem_mixed(npe, _p(X, _d), _p(u, _d), _p(up, _d), _p(pn, _d), int(model), _p(d, _d), Kinv,
                               utype, _p(Kuu, _d), _p(Kup, _d), _p(Kpu, _d), _p(Kpp, _d), _p(FU, _d), _p(FP, _d))
    if bad == 2:
        raise ValueError("oracle: the mixed element is tet10 or hex27")
    return Kuu, Kup, Kpu, Kpp, FU, FP, bad


def elem_mixed0(X, u, u_prev, pres, model, data, Kinv, utype=3):
    """Constant-pressure u-p element (hex8 or tet10), condensed: K, F, kup (= Kpu), Kpp, FP, bad."""
    X, u, up = (np.ascontiguousarray(a, dtype=np.float64) for a in (X, u, u_prev))
    npe = X.shape[0]
    d = _mat_data(data)
    ns = 3 * npe
    K, F, kup = np.zeros((ns, ns)), np.zeros(ns), np.zeros(ns)
    kpp, fp = np.zeros(1), np.zeros(1)
    bad = lib().orc_elem_mixed0(npe, _p(X, _d), _p(u, _d), _p(up, _d), float(pres), int(model), _p(d, _d), Kinv, utype,
                                _p(K, _d), _p(F, _d), _p(kup, _d), _p(kpp, _d), _p(fp, _d))
    if bad == 2:
        raise ValueError("oracle: the constant-pressure element is hex8 or tet10")
    return K, F, kup, float(kpp[0]), float(fp[0]), bad


def gauss_rule(npe):
    xi, w = np.zeros((27, 3)), np.zeros(27)
    N, dN = np.zeros((27, npe)), np.zeros((27, 3, npe))
    ngp = lib().orc_gauss_rule(npe, _p(xi, _d), _p(w, _d), _p(N, _d), _p(dN, _d))
    return xi[:ngp], w[:ngp], N[:ngp], dN[:ngp]


class OracleProblem:
    """A mesh with its DOF map and CSR pattern, restating prepareMatrixPattern."""

    def __init__(self, prob):
        self.prob = prob
        self._keep = [np.ascontiguousarray(prob.coords, np.float64), np.ascontiguousarray(prob.conn, np.int32),
                      np.ascontiguousarray(prob.mat_id, np.int32), np.ascontiguousarray(prob.mats, np.float64),
                      np.ascontiguousarray(prob.fixed, np.uint8)]
        c, cn, m, mt, fx = self._keep
        self.h = lib().orc_problem_create(prob.n_node, _p(c, _d), prob.n_elem, prob.npe, _p(cn, _i32),
                                          _p(m, _i32), mt.shape[0], _p(mt, _d), _p(fx, _u8))
        if not self.h:
            raise ValueError("oracle: unsupported element type")
        models = getattr(prob, "mat_model", None)
        if models is not None:
            mdl = np.ascontiguousarray(models, np.int32)
            dat = np.ascontiguousarray(prob.mat_data, np.float64).reshape(len(mdl), MAT_NDATA)
            self._keep += [mdl, dat]
            if lib().orc_problem_set_materials(self.h, len(mdl), _p(mdl, _i32), _p(dat, _d)):
                raise ValueError("oracle: invalid material models")
        self.n_free = lib().orc_problem_nfree(self.h)
        self.nnz = lib().orc_problem_nnz(self.h)
        ramp, cst = getattr(prob, "presc_ramp", None), getattr(prob, "presc_const", None)
        if ramp is not None or cst is not None:
            r = None if ramp is None else np.ascontiguousarray(ramp, np.float64)
            c = None if cst is None else np.ascontiguousarray(cst, np.float64)
            self._keep += [r, c]
            lib().orc_problem_set_prescribed(self.h, _p(r, _d), _p(c, _d))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_problem_destroy(self.h)
            self.h = None

    def set_mixed_p0(self, enable=True):
        """Elem_Solid_3D_Mixed0 for every element (condensed element pressures, zero to start)."""
        if lib().orc_problem_set_mixed_p0(self.h, int(enable)):
            raise ValueError("oracle: Utype -1 has no constant-pressure element (Kpp = 0)")

    def p0_pressure(self, set_to=None):
        out = np.zeros(self.prob.n_elem)
        src = None if set_to is None else np.ascontiguousarray(set_to, np.float64)
        lib().orc_problem_p0_pressure(self.h, _p(src, _d), _p(out, _d))
        return out

    def save_step(self, disp):
        d = np.ascontiguousarray(disp, np.float64)
        lib().orc_problem_save_step(self.h, _p(d, _d))

    def pattern(self):
        ns = 3 * self.prob.npe
        afs = np.zeros(self.n_free, np.int32)
        fav = np.zeros((self.prob.n_elem, ns), np.int32)
        rp = np.zeros(self.n_free + 1, np.int64)
        col = np.zeros(self.nnz, np.int32)
        lib().orc_problem_export_pattern(self.h, _p(afs, _i32), _p(fav, _i32), _p(rp, _i64), _p(col, _i32))
        return afs, fav, rp, col

    def elements(self, disp, nthreads=1):
        ns = 3 * self.prob.npe
        disp = np.ascontiguousarray(disp, np.float64)
        Ke = np.zeros((self.prob.n_elem, ns, ns))
        Re = np.zeros((self.prob.n_elem, ns))
        bad = lib().orc_problem_elements(self.h, _p(disp, _d), _p(Ke, _d), _p(Re, _d), nthreads)
        return Ke, Re, int(bad)

    def assemble(self, disp, nthreads=1, want_val=True, want_reac=True):
        disp = np.ascontiguousarray(disp, np.float64)
        val = np.zeros(self.nnz) if want_val else None
        rhs = np.zeros(self.n_free)
        reac = np.zeros(self.prob.n_dof) if want_reac else None
        bad = lib().orc_problem_assemble(self.h, _p(disp, _d), _p(val, _d), _p(rhs, _d), _p(reac, _d), nthreads)
        return val, rhs, reac, int(bad)

    def cg(self, val, b, rtol=1e-12, abstol=1e-50, maxit=10000, nthreads=1, norm_type=0):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n_free)
        its, fn = C.c_int(0), C.c_double(0.0)
        st = lib().orc_cg_jacobi_norm(self.h, _p(val, _d), _p(b, _d), _p(x, _d), rtol, abstol, maxit, nthreads,
                                      norm_type, C.byref(its), C.byref(fn))
        return x, its.value, fn.value, st

    def newton(self, tol_rel=None, tol_abs=0.0, cg_rtol=None, cg_maxit=10000, max_newton=10,
               nthreads=1, disp=None, max_hist=4096):
        p = self.prob
        o = NewtonOpts(p.dt, p.t_final, p.max_steps, max_newton,
                       p.newton_rtol if tol_rel is None else tol_rel, tol_abs,
                       p.cg_rtol if cg_rtol is None else cg_rtol, cg_maxit, nthreads)
        u = np.zeros(p.n_dof) if disp is None else np.array(disp, np.float64)
        f = np.ascontiguousarray(p.fnodal, np.float64)
        hist = np.zeros((max_hist, 4))
        rows = lib().orc_newton_run(self.h, _p(f, _d), C.byref(o), _p(u, _d), _p(hist, _d), max_hist)
        if rows < 0:
            raise RuntimeError("oracle Newton: time step size fell below 1% of the initial value")
        return u, hist[:rows]

    def arclength(self, tol_rel=0.0, tol_abs=None, cg_rtol=None, cg_maxit=10000, max_newton=10, nthreads=1,
                  disp=None, max_hist=4096):
        """solveWithArclength: (disp, load factors of the converged steps, history rows
        [step, iter, ||R||, CG its of both solves, load factor])."""
        p = self.prob
        o = NewtonOpts(p.dt, p.t_final, p.max_steps, max_newton, tol_rel,
                       p.meta.get("tolerance", 0.0) if tol_abs is None else tol_abs,
                       p.cg_rtol if cg_rtol is None else cg_rtol, cg_maxit, nthreads)
        u = np.zeros(p.n_dof) if disp is None else np.array(disp, np.float64)
        f = np.ascontiguousarray(p.fnodal, np.float64)
        lam = np.zeros(max(1, p.max_steps))
        nl = C.c_int(0)
        hist = np.zeros((max_hist, 5))
        rows = lib().orc_arclength_run(self.h, _p(f, _d), C.byref(o), _p(u, _d), _p(lam, _d), len(lam), C.byref(nl),
                                       _p(hist, _d), max_hist)
        if rows < 0:
            raise RuntimeError("oracle arc-length: the first step did not converge")
        return u, lam[:min(nl.value, len(lam))], hist[:rows]
