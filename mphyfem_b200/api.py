"""Host-side mirror of the reference's element, material and solver interfaces over libmphy.so.

Names follow chennachaos/mphyfem so that a caller of the reference finds the same surface:

* :class:`SolverGpu` -- ``SolverPetsc`` (src/mySolvers/SolverPetsc.h:16-96): ``initialise``,
  ``zeroMtx``, ``assembleMatrixAndVector``, ``factoriseAndSolve``, ``currentStatus``;
* :meth:`SolverGpu.calcStiffnessAndResidual` -- ``femSolidmechanics::calcStiffnessAndResidual``
  (femSolidmechanics2.cpp:1047-1120), every element fused with the scatter;
* :func:`calc_stiffness_and_residual` -- ``ElementBase::calcStiffnessAndResidual`` batched;
* :func:`compute_stress_and_tangent` -- ``MaterialBase::computeStressAndTangent``;
* :class:`FemSolidmechanicsGpu` -- ``femSolidmechanics::prepareMatrixPattern`` / ``setSolver`` /
  ``solveWithNewtonRaphson``.

Device arrays are torch CUDA tensors (plumbing only); all arithmetic runs in libmphy.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise L.MphyError(L.ERR_NO_DEVICE, "no CUDA device visible")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _np(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Context:
    """One device + one CUDA stream (replaces PetscInitialize, femSolidmechanics.cpp:49)."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.mphy_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def synchronize(self):
        L.check(self.lib.mphy_ctx_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Mesh:
    """Device-resident mesh of a :class:`mphyfem_b200.meshgen.Problem`."""

    def __init__(self, ctx: Context, prob):
        self.ctx, self.prob = ctx, prob
        self.lib = ctx.lib
        c = _np(prob.coords, np.float64)
        cn = _np(prob.conn, np.int32)
        mi = _np(prob.mat_id, np.int32)
        mt = _np(prob.mats, np.float64)
        fx = _np(prob.fixed, np.uint8)
        h = C.c_void_p()
        L.check(self.lib.mphy_mesh_create(ctx.h, prob.n_node, c.ctypes.data_as(L._d), prob.n_elem, prob.npe,
                                          cn.ctypes.data_as(L._i32), mi.ctypes.data_as(L._i32), mt.shape[0],
                                          mt.ctypes.data_as(L._d), fx.ctypes.data_as(L._u8), C.byref(h)))
        self.h = h
        if getattr(prob, "mat_model", None) is not None:
            self.set_materials(prob.mat_model, prob.mat_data)
        if getattr(prob, "presc_ramp", None) is not None or getattr(prob, "presc_const", None) is not None:
            self.set_prescribed(prob.presc_ramp, prob.presc_const)

    def set_prescribed(self, ramp=None, const=None):
        """Nonzero prescribed displacements: t * ramp + const on the prescribed DOFs at time t."""
        r = None if ramp is None else _np(ramp, np.float64)
        c = None if const is None else _np(const, np.float64)
        L.check(self.lib.mphy_mesh_set_prescribed(self.h, None if r is None else r.ctypes.data_as(L._d),
                                                  None if c is None else c.ctypes.data_as(L._d)))

    def set_materials(self, model, data):
        """Per-material hyperelastic model (MAT_*) and parameters [n_mat, MAT_NDATA]
        (mphy_mesh_set_materials); Kinv and Utype stay those of the mesh's material rows."""
        mdl = _np(model, np.int32)
        dat = np.zeros((mdl.shape[0], L.MAT_NDATA))
        d = np.asarray(data, np.float64).reshape(mdl.shape[0], -1)
        dat[:, :d.shape[1]] = d
        L.check(self.lib.mphy_mesh_set_materials(self.h, mdl.shape[0], mdl.ctypes.data_as(L._i32),
                                                 dat.ctypes.data_as(L._d)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Pattern:
    """DOF map + sparsity built on the device (prepareMatrixPattern, femSolidmechanics2.cpp:121-478)."""

    def __init__(self, mesh: Mesh):
        self.mesh, self.lib = mesh, mesh.lib
        h = C.c_void_p()
        L.check(self.lib.mphy_pattern_build(mesh.ctx.h, mesh.h, C.byref(h)))
        self.h = h
        nf, nnz, nb, sb = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
        L.check(self.lib.mphy_pattern_info(h, C.byref(nf), C.byref(nnz), C.byref(nb), C.byref(sb)))
        self.n_free, self.nnz, self.n_blocks, self.stored_blocks = nf.value, nnz.value, nb.value, sb.value

    def export_csr(self):
        rp = np.zeros(self.n_free + 1, np.int64)
        col = np.zeros(self.nnz, np.int32)
        L.check(self.lib.mphy_pattern_export_csr(self.h, rp.ctypes.data_as(L._i64), col.ctypes.data_as(L._i32)))
        return rp, col

    def export_dofmap(self):
        p = self.mesh.prob
        afs = np.zeros(self.n_free, np.int32)
        fav = np.zeros((p.n_elem, 3 * p.npe), np.int32)
        L.check(self.lib.mphy_pattern_export_dofmap(self.h, afs.ctypes.data_as(L._i32), fav.ctypes.data_as(L._i32)))
        return afs, fav

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_pattern_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def default_solver_opts(**kw) -> L.SolverOpts:
    o = L.SolverOpts()
    L.load().mphy_solver_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class SolverGpu:
    """The ``SolverPetsc`` surface on the GPU (SolverPetsc.h:16-96)."""

    def __init__(self, mesh: Mesh, pattern: Pattern, **opts):
        self.mesh, self.pattern, self.lib = mesh, pattern, mesh.lib
        self.opts = default_solver_opts(**opts)
        h = C.c_void_p()
        L.check(self.lib.mphy_solver_create(mesh.ctx.h, mesh.h, pattern.h, C.byref(self.opts), C.byref(h)))
        self.h = h

    @property
    def currentStatus(self) -> int:  # noqa: N802 (reference name)
        s = C.c_int32()
        L.check(self.lib.mphy_solver_get_state(self.h, C.byref(s)))
        return s.value

    def zeroMtx(self):  # noqa: N802
        L.check(self.lib.mphy_solver_zero(self.h))

    def calcStiffnessAndResidual(self, disp_dev):  # noqa: N802
        """Fused element evaluation + scatter. Raises MphyError(ERR_NEG_JACOBIAN) on det F < 0."""
        bad = C.c_int64(-1)
        L.check(self.lib.mphy_solver_assemble(self.h, _ptr(disp_dev), C.byref(bad)))

    def assembleMatrixAndVector(self, Ke_dev, Re_dev, elem_ids_dev=None):  # noqa: N802
        n = Ke_dev.shape[0]
        ids = _ptr(elem_ids_dev) if elem_ids_dev is not None else None
        L.check(self.lib.mphy_solver_assemble_batch(self.h, n, ids, _ptr(Ke_dev), _ptr(Re_dev)))

    def addExternalForces(self, fext_dev, scale: float):  # noqa: N802
        L.check(self.lib.mphy_solver_add_nodal_forces(self.h, _ptr(fext_dev), float(scale)))

    def rhsNorm(self) -> float:  # noqa: N802
        v = C.c_double()
        L.check(self.lib.mphy_solver_rhs_norm(self.h, C.byref(v)))
        return v.value

    def factoriseAndSolve(self, allow_fail: bool = False):  # noqa: N802
        its, fn = C.c_int32(), C.c_double()
        rc = self.lib.mphy_solver_solve(self.h, C.byref(its), C.byref(fn))
        if not allow_fail:
            L.check(rc)
        return rc, its.value, fn.value

    def spmv(self, x_dev, y_dev):
        """y = A x with the assembled operator (MatMult); ordered on the library stream."""
        L.check(self.lib.mphy_solver_spmv(self.h, _ptr(x_dev), _ptr(y_dev)))

    def spmv_dot(self, x_dev, y_dev, want_dot: bool = True):
        """y = A x and (x, y) in one pass, the CG iteration's SpMV kernel; returns (x, y) (or None
        without a host wait when want_dot is False)."""
        v = C.c_double()
        L.check(self.lib.mphy_solver_spmv_dot(self.h, _ptr(x_dev), _ptr(y_dev), C.byref(v) if want_dot else None))
        return v.value if want_dot else None

    def matrix_info(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(self.lib.mphy_solver_matrix_info(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return {"stored_blocks": a.value, "true_blocks": b.value, "value_bytes": c.value}

    @property
    def stream(self) -> int:
        return self.lib.mphy_ctx_stream(self.mesh.ctx.h) or 0

    # ---- factorised preconditioner M = G^T G (pc_type FSAI / FSAI_LEARNED)
    def pc_pattern(self):
        n = C.c_int64()
        L.check(self.lib.mphy_solver_pc_pattern(self.h, C.byref(n), None, None))
        rp = np.zeros(self.mesh.prob.n_node + 1, np.int64)
        col = np.zeros(n.value, np.int32)
        L.check(self.lib.mphy_solver_pc_pattern(self.h, None, rp.ctypes.data_as(L._i64), col.ctypes.data_as(L._i32)))
        return rp, col

    def pc_setup(self) -> int:
        nf = C.c_int32()
        L.check(self.lib.mphy_solver_pc_setup(self.h, C.byref(nf)))
        return nf.value

    def pc_get_blocks(self):
        torch = _torch()
        rp, _ = self.pc_pattern()
        out = torch.empty((int(rp[-1]), 3, 3), dtype=torch.float32, device="cuda")
        L.check(self.lib.mphy_solver_pc_get_blocks(self.h, _ptr(out)))
        return out

    def pc_set_blocks(self, blocks_dev):
        torch = _torch()
        b = blocks_dev.contiguous().to(torch.float32)
        L.check(self.lib.mphy_solver_pc_set_blocks(self.h, _ptr(b)))

    def true_residual(self) -> float:
        """||b - A x|| / ||b|| of the last solve, FP64."""
        v = C.c_double()
        L.check(self.lib.mphy_solver_true_residual(self.h, C.byref(v)))
        return v.value

    def pc_last(self):
        fb, ms, st, it, rr = C.c_int32(), C.c_float(), C.c_int32(), C.c_int32(), C.c_double()
        L.check(self.lib.mphy_solver_pc_last(self.h, C.byref(fb), C.byref(ms), C.byref(st), C.byref(it), C.byref(rr)))
        return {"fallback": bool(fb.value), "setup_ms": ms.value, "first_status": st.value, "first_its": it.value,
                "first_relres": rr.value}

    def coarse_info(self):
        g = (C.c_int32 * 3)()
        k = C.c_int32()
        ms = C.c_float()
        L.check(self.lib.mphy_solver_coarse_info(self.h, g, C.byref(k), C.byref(ms)))
        return {"grid": tuple(g), "coarse_size": k.value, "setup_ms": ms.value}

    def solution(self):
        torch = _torch()
        x = torch.empty(self.mesh.prob.n_dof, dtype=torch.float64, device="cuda")
        L.check(self.lib.mphy_solver_get_solution(self.h, _ptr(x)))
        return x

    def export(self, want_val=True, want_rhs=True, want_reac=True):
        val = np.zeros(self.pattern.nnz) if want_val else None
        rhs = np.zeros(self.pattern.n_free) if want_rhs else None
        reac = np.zeros(self.mesh.prob.n_dof) if want_reac else None
        p = lambda a: a.ctypes.data_as(L._d) if a is not None else None  # noqa: E731
        L.check(self.lib.mphy_solver_export(self.h, p(val), p(rhs), p(reac)))
        return val, rhs, reac

    def set_mixed_p0(self, enable: bool = True):
        """Elem_Solid_3D_Mixed0: one condensed pressure per element (zero to start)."""
        L.check(self.lib.mphy_solver_set_mixed_p0(self.h, int(enable)))

    def p0_pressure(self, set_to=None) -> np.ndarray:
        """Element pressures of the constant-pressure element; set_to [n_elem] replaces them first."""
        out = np.zeros(self.mesh.prob.n_elem)
        src = None if set_to is None else _np(set_to, np.float64)
        L.check(self.lib.mphy_solver_p0_pressure(self.h, None if src is None else src.ctypes.data_as(L._d),
                                                 out.ctypes.data_as(L._d)))
        return out

    def save_step(self, disp_dev):
        """The converged state of a load step (disp and the element pressures)."""
        L.check(self.lib.mphy_solver_save_step(self.h, _ptr(disp_dev)))

    def newton_iteration(self, disp_dev, fext_dev, lam: float, tol_abs: float = 0.0) -> L.IterStats:
        st = L.IterStats()
        L.check(self.lib.mphy_newton_iteration(self.h, _ptr(disp_dev), _ptr(fext_dev) if fext_dev is not None else None,
                                               float(lam), float(tol_abs), C.byref(st)))
        return st

    def newton_iteration_host(self, disp_host: np.ndarray, fext_host: np.ndarray | None, lam: float,
                              tol_abs: float = 0.0) -> L.IterStats:
        st = L.IterStats()
        f = fext_host.ctypes.data_as(L._d) if fext_host is not None else None
        L.check(self.lib.mphy_newton_iteration_host(self.h, disp_host.ctypes.data_as(L._d), f, float(lam),
                                                    float(tol_abs), C.byref(st)))
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def compute_stress_and_tangent(ctx: Context, F_dev, mu: float, Kinv: float, utype: int = 3,
                               tangent: int = L.TANGENT_REFERENCE):
    """Batched MaterialBase::computeStressAndTangent: F [n,3,3] -> stre [n,9], Cmat [n,9,9]."""
    torch = _torch()
    n = F_dev.shape[0]
    F = F_dev.contiguous().to(torch.float64)
    s = torch.empty((n, 9), dtype=torch.float64, device=F.device)
    Cm = torch.empty((n, 9, 9), dtype=torch.float64, device=F.device)
    L.check(ctx.lib.mphy_material_nh_eval(ctx.h, n, _ptr(F), mu, Kinv, utype, tangent, _ptr(s), _ptr(Cm)))
    return s, Cm


def material_stress_and_tangent(ctx: Context, F_dev, model: int, data, Kinv: float, utype: int = 3,
                                tangent: int = L.TANGENT_REFERENCE):
    """Batched computeStressAndTangent of any hyperelastic model (MAT_*): F [n,3,3] -> stre [n,9],
    Cmat [n,9,9]. data: the model's parameters (mu; c1 c2; mu Im; mu N)."""
    torch = _torch()
    n = F_dev.shape[0]
    F = F_dev.contiguous().to(torch.float64)
    d = np.zeros(L.MAT_NDATA)
    d[:len(data)] = data
    s = torch.empty((n, 9), dtype=torch.float64, device=F.device)
    Cm = torch.empty((n, 9, 9), dtype=torch.float64, device=F.device)
    L.check(ctx.lib.mphy_material_eval(ctx.h, n, _ptr(F), int(model), d.ctypes.data_as(L._d), Kinv, utype, tangent,
                                       _ptr(s), _ptr(Cm)))
    return s, Cm


def calc_stiffness_and_residual(mesh: Mesh, disp_dev, tangent: int = L.TANGENT_REFERENCE, tensor_cores: bool = False):
    """Batched ElementBase::calcStiffnessAndResidual over every element: Ke, Re, first bad element.
    tensor_cores: the MPHY_PREC_MIXED_TC kernel (FP64 residual, split-BF16 tangent contraction)."""
    torch = _torch()
    p = mesh.prob
    ns = 3 * p.npe
    Ke = torch.empty((p.n_elem, ns, ns), dtype=torch.float64, device="cuda")
    Re = torch.empty((p.n_elem, ns), dtype=torch.float64, device="cuda")
    bad = C.c_int64(-1)
    fn = mesh.lib.mphy_elem_eval_tc if tensor_cores else mesh.lib.mphy_elem_eval
    rc = fn(mesh.ctx.h, mesh.h, _ptr(disp_dev), tangent, _ptr(Ke), _ptr(Re), C.byref(bad))
    L.check(rc, allow=(L.ERR_NEG_JACOBIAN,))
    return Ke, Re, bad.value


@dataclass
class NewtonResult:
    disp: np.ndarray
    # rows (step, iter, ||R||, krylov its, krylov status, t_assembly_ms, t_solve_ms), and for the
    # displacement solver (newton_run) an eighth column: the library kernels the iteration launched
    hist: np.ndarray
    status: int


def newton_run(solver: "SolverGpu", prob, max_newton: int = 10, tol_rel: float | None = None, tol_abs: float = 0.0,
               disp: np.ndarray | None = None, max_hist: int = 4096, t_final: float | None = None,
               max_steps: int | None = None) -> NewtonResult:
    """solveWithNewtonRaphson (femSolidmechanics2.cpp:730-851) on an existing solver: load steps of
    prob.dt up to t_final (default prob.t_final, at most max_steps), each iterated until
    ||R|| < max(tol_abs, tol_rel ||R_first||), with the reference's cuts."""
    p = prob
    o = L.NewtonOpts(p.dt, p.t_final if t_final is None else t_final, p.max_steps if max_steps is None else max_steps,
                     max_newton, p.newton_rtol if tol_rel is None else tol_rel, tol_abs)
    u = np.zeros(p.n_dof) if disp is None else np.array(disp, np.float64)
    f = _np(p.fnodal, np.float64)
    hist = (L.IterStats * max_hist)()
    n = C.c_int32(0)
    rc = solver.lib.mphy_newton_run(solver.h, f.ctypes.data_as(L._d), C.byref(o), u.ctypes.data_as(L._d),
                                    hist, max_hist, C.byref(n))
    L.check(rc, allow=(L.ERR_TIME_STEP,))
    rows = np.array([[h.step, h.iter, h.rhs_norm, h.krylov_its, h.status, h.t_assembly_ms, h.t_solve_ms,
                      h.kernel_launches] for h in hist[:n.value]], dtype=np.float64).reshape(-1, 8)
    return NewtonResult(disp=u, hist=rows, status=rc)


class FemSolidmechanicsGpu:
    """femSolidmechanics on the GPU: setSolver (pattern + solver) and solveWithNewtonRaphson."""

    def __init__(self, prob, ctx: Context | None = None, mixed_p0: bool = False, **solver_opts):
        self.prob = prob
        self.ctx = ctx or Context(0)
        self.mesh = Mesh(self.ctx, prob)
        self.pattern = Pattern(self.mesh)
        opts = dict(rtol=prob.cg_rtol)
        opts.update(solver_opts)
        self.solver = SolverGpu(self.mesh, self.pattern, **opts)
        if mixed_p0 or prob.meta.get("element") == "ELEM_SOLID_3D_MIXED0":
            self.solver.set_mixed_p0(True)

    @classmethod
    def from_reference_inputs(cls, config_path, ctx: Context | None = None, **solver_opts):
        """The reference's inputs (a config file and the Gmsh 2.2 mesh it names, see
        reference_io); solve_reference() then applies its Solver block."""
        from . import reference_io
        return cls(reference_io.read_config(config_path), ctx, **solver_opts)

    def solve_reference(self) -> "NewtonResult":
        """solveWithNewtonRaphson with the config's absolute `tolerance` and `maximumIterations`
        (femSolidmechanics1.cpp:616-622: converged when ||R|| < tolerance)."""
        m = self.prob.meta
        return self.solveWithNewtonRaphson(max_newton=int(m["maximumIterations"]), tol_rel=0.0,
                                           tol_abs=float(m["tolerance"]))

    def solveWithNewtonRaphson(self, max_newton: int = 10, tol_rel: float | None = None, tol_abs: float = 0.0,  # noqa: N802
                               disp: np.ndarray | None = None, max_hist: int = 4096) -> NewtonResult:
        return newton_run(self.solver, self.prob, max_newton, tol_rel, tol_abs, disp, max_hist)

    def solveWithArclength(self, max_newton: int = 10, tol_rel: float = 0.0, tol_abs: float | None = None,  # noqa: N802
                           disp: np.ndarray | None = None, max_hist: int = 4096) -> "ArclengthResult":
        """Arc-length continuation (femSolidmechanics2.cpp:855-1039): see solve_with_arclength."""
        return solve_with_arclength(self, max_newton, tol_rel, tol_abs, disp, max_hist)


@dataclass
class MixedNewtonResult:
    disp: np.ndarray
    pres: np.ndarray  # nodal pressures [n_node] (vertex nodes carry the pressure DOFs)
    hist: np.ndarray  # rows (step, iter, ||R||, MINRES its, status, t_assembly_ms, t_solve_ms)
    status: int


class MixedSolidGpu:
    """A mixed u-p problem (Elem_Solid_3D_Mixed1: tet10 displacement with linear vertex pressure,
    or the P2-P1 hex27 with trilinear corner pressure) on the GPU: two-field assembly, MINRES
    solve and Newton load stepping (mphy_mixed_*)."""

    def __init__(self, prob, ctx: Context | None = None, tangent: int = L.TANGENT_REFERENCE, rtol: float = 1e-10,
                 max_it: int = 20000, coarse_aggregates: int = 0, coarse_modes: int = 0):
        self.prob = prob
        self.ctx = ctx or Context(0)
        self.lib = self.ctx.lib
        self.mesh = Mesh(self.ctx, prob)
        self.pattern = Pattern(self.mesh)
        o = L.MixedOpts()
        self.lib.mphy_mixed_opts_default(C.byref(o))
        o.tangent, o.rtol, o.max_it, o.coarse_aggregates, o.coarse_modes = (tangent, rtol, max_it, coarse_aggregates,
                                                                             coarse_modes)
        h = C.c_void_p()
        L.check(self.lib.mphy_mixed_create(self.ctx.h, self.mesh.h, self.pattern.h, C.byref(o), C.byref(h)))
        self.h = h
        npres, nb, nc = C.c_int32(), C.c_int64(), C.c_int64()
        L.check(self.lib.mphy_mixed_info(h, C.byref(npres), C.byref(nb), C.byref(nc)))
        self.n_pres, self.nnz_coupling, self.nnz_pp = npres.value, nb.value, nc.value
        self.n = prob.n_dof + self.n_pres

    def pressure_nodes(self) -> np.ndarray:
        out = np.zeros(self.n_pres, np.int32)
        L.check(self.lib.mphy_mixed_pressure_nodes(self.h, out.ctypes.data_as(L._i32)))
        return out

    def elements(self, disp, disp_prev, pres):
        """(Kuu, FU, Kup, Kpp, FP, first bad) per element, device tensors."""
        torch = _torch()
        ne = self.prob.n_elem
        dev = dict(dtype=torch.float64, device="cuda")
        ns, NP = 3 * self.prob.npe, {10: 4, 27: 8}[self.prob.npe]  # pressure nodes per element
        Kuu, FU = torch.empty((ne, ns, ns), **dev), torch.empty((ne, ns), **dev)
        Kup, Kpp, FP = torch.empty((ne, ns, NP), **dev), torch.empty((ne, NP, NP), **dev), torch.empty((ne, NP), **dev)
        bad = C.c_int64(-1)
        rc = self.lib.mphy_mixed_elem_eval(self.h, _ptr(disp), _ptr(disp_prev), _ptr(pres), _ptr(Kuu), _ptr(FU),
                                           _ptr(Kup), _ptr(Kpp), _ptr(FP), C.byref(bad))
        L.check(rc, allow=(L.ERR_NEG_JACOBIAN,))
        return Kuu, FU, Kup, Kpp, FP, bad.value

    def assemble(self, disp, disp_prev, pres, lam: float = 0.0, fext=None) -> float:
        nrm, bad = C.c_double(), C.c_int64(-1)
        L.check(self.lib.mphy_mixed_assemble(self.h, _ptr(disp), _ptr(disp_prev), _ptr(pres), float(lam),
                                             _ptr(fext) if fext is not None else None, C.byref(nrm), C.byref(bad)))
        return nrm.value

    def apply(self, x):
        torch = _torch()
        y = torch.empty_like(x)
        L.check(self.lib.mphy_mixed_apply(self.h, _ptr(x), _ptr(y)))
        return y

    def vectors(self):
        """(rhs [3 n_node + n_pres], reactions [3 n_node], solution [3 n_node + n_pres])."""
        torch = _torch()
        dev = dict(dtype=torch.float64, device="cuda")
        rhs, reac, x = torch.empty(self.n, **dev), torch.empty(self.prob.n_dof, **dev), torch.empty(self.n, **dev)
        L.check(self.lib.mphy_mixed_vectors(self.h, _ptr(rhs), _ptr(reac), _ptr(x)))
        return rhs, reac, x

    def solve(self, allow_fail: bool = False):
        its, rr = C.c_int32(), C.c_double()
        rc = self.lib.mphy_mixed_solve(self.h, C.byref(its), C.byref(rr))
        if not allow_fail:
            L.check(rc)
        return rc, its.value, rr.value

    def solveWithNewtonRaphson(self, max_newton: int = 10, tol_rel: float | None = None,  # noqa: N802
                               tol_abs: float = 0.0, max_hist: int = 4096) -> MixedNewtonResult:
        p = self.prob
        o = L.NewtonOpts(p.dt, p.t_final, p.max_steps, max_newton, p.newton_rtol if tol_rel is None else tol_rel,
                         tol_abs)
        u, pres = np.zeros(p.n_dof), np.zeros(p.n_node)
        f = _np(p.fnodal, np.float64)
        hist = (L.IterStats * max_hist)()
        n = C.c_int32(0)
        rc = self.lib.mphy_mixed_newton_run(self.h, f.ctypes.data_as(L._d), C.byref(o), u.ctypes.data_as(L._d),
                                            pres.ctypes.data_as(L._d), hist, max_hist, C.byref(n))
        L.check(rc, allow=(L.ERR_TIME_STEP,))
        rows = np.array([[h.step, h.iter, h.rhs_norm, h.krylov_its, h.status, h.t_assembly_ms, h.t_solve_ms]
                         for h in hist[:n.value]], dtype=np.float64).reshape(-1, 7)
        return MixedNewtonResult(disp=u, pres=pres, hist=rows, status=rc)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_mixed_destroy(self.h)
            self.h = None
        for obj in ("pattern", "mesh"):
            o = getattr(self, obj, None)
            if o is not None:
                o.close()

    def __del__(self):
        self.close()


@dataclass
class ArclengthResult:
    disp: np.ndarray
    load_factors: np.ndarray  # load factor of each converged step
    hist: np.ndarray  # rows (step, iter, ||R||, krylov its of both solves, status, load factor after the update)
    status: int


def solve_with_arclength(fem: "FemSolidmechanicsGpu", max_newton: int = 10, tol_rel: float = 0.0,
                         tol_abs: float | None = None, disp: np.ndarray | None = None,
                         max_hist: int = 4096) -> ArclengthResult:
    """femSolidmechanics::solveWithArclength (mphy_arclength_run) on fem's solver. The first
    step is a Newton solve at load factor prob.dt; max_newton is iterationsMax (iterations
    1..max_newton-1); tol_abs defaults to the config's tolerance (0 when absent)."""
    p = fem.prob
    tol_abs = float(p.meta.get("tolerance", 0.0)) if tol_abs is None else tol_abs
    o = L.NewtonOpts(p.dt, p.t_final, p.max_steps, max_newton, tol_rel, tol_abs)
    u = np.zeros(p.n_dof) if disp is None else np.array(disp, np.float64)
    f = _np(p.fnodal, np.float64)
    lam = np.zeros(max(1, p.max_steps))
    hl = np.zeros(max_hist)
    hist = (L.IterStats * max_hist)()
    nl, n = C.c_int32(0), C.c_int32(0)
    rc = fem.ctx.lib.mphy_arclength_run(fem.solver.h, f.ctypes.data_as(L._d), C.byref(o), u.ctypes.data_as(L._d),
                                        lam.ctypes.data_as(L._d), len(lam), C.byref(nl), hist,
                                        hl.ctypes.data_as(L._d), max_hist, C.byref(n))
    L.check(rc, allow=(L.ERR_NOT_CONVERGED,))
    rows = np.array([[h.step, h.iter, h.rhs_norm, h.krylov_its, h.status, hl[k]]
                     for k, h in enumerate(hist[:n.value])], dtype=np.float64).reshape(-1, 6)
    return ArclengthResult(disp=u, load_factors=lam[:min(nl.value, len(lam))], hist=rows, status=rc)


class BatchGpu:
    """The batched form: independent problems as one block-diagonal union (meshgen.batch_union),
    assembled together and solved in one persistent launch (mphy_batch_*)."""

    def __init__(self, problems, ctx: Context | None = None, union=None, **solver_opts):
        from . import meshgen
        self.ctx = ctx or Context(0)
        self.problems = list(problems)
        self.union = union if union is not None else meshgen.batch_union(self.problems)
        self.node_ptr = np.ascontiguousarray(self.union.meta["inst_node_ptr"], np.int32)
        self.mesh = Mesh(self.ctx, self.union)
        self.pattern = Pattern(self.mesh)
        opts = dict(rtol=1e-10, norm_type=1)
        opts.update(solver_opts)
        self.solver = SolverGpu(self.mesh, self.pattern, **opts)
        self.lib = self.ctx.lib
        h = C.c_void_p()
        L.check(self.lib.mphy_batch_create(self.solver.h, len(self.node_ptr) - 1,
                                           self.node_ptr.ctypes.data_as(L._i32), C.byref(h)))
        self.h = h
        self.n_inst = len(self.node_ptr) - 1

    def schedule(self):
        c, t = C.c_int32(), C.c_int32()
        L.check(self.lib.mphy_batch_get_schedule(self.h, C.byref(c), C.byref(t)))
        return c.value, t.value

    def set_schedule(self, cluster: int, threads: int):
        L.check(self.lib.mphy_batch_set_schedule(self.h, cluster, threads))

    def set_coarse(self, slabs: int):
        """Two-level persistent solve: `slabs` rigid-body slabs per instance (0: Jacobi only)."""
        L.check(self.lib.mphy_batch_set_coarse(self.h, slabs))

    def autotune(self, maxit: int = 0):
        """Times every schedule on the assembled system (maxit <= 0: complete solves); keeps the
        fastest. Returns rows (cluster, threads, ms)."""
        n = C.c_int32()
        cl, th, ms = (C.c_int32 * 32)(), (C.c_int32 * 32)(), (C.c_float * 32)()
        L.check(self.lib.mphy_batch_autotune(self.h, maxit, 32, C.byref(n), cl, th, ms))
        return [(cl[i], th[i], ms[i]) for i in range(min(n.value, 32))]

    def solve(self, maxit: int = 0):
        """All instances' linear solves on the assembled system. Returns (its, status, relres, ms)."""
        its = np.zeros(self.n_inst, np.int32)
        st = np.zeros(self.n_inst, np.int32)
        rel = np.zeros(self.n_inst, np.float64)
        ms = C.c_float()
        L.check(self.lib.mphy_batch_solve(self.h, maxit, its.ctypes.data_as(L._i32), st.ctypes.data_as(L._i32),
                                          rel.ctypes.data_as(L._d), C.byref(ms)))
        return its, st, rel, ms.value

    def newton_run(self, max_newton: int = 10, tol_rel: float | None = None, tol_abs: float = 0.0,
                   disp: np.ndarray | None = None):
        """Load stepping of every instance. Returns dict(disp, newton_its [steps, n_inst],
        krylov_its, status, stats)."""
        p = self.union
        o = L.NewtonOpts(p.dt, p.t_final, p.max_steps, max_newton, p.newton_rtol if tol_rel is None else tol_rel,
                         tol_abs)
        u = np.zeros(p.n_dof) if disp is None else np.array(disp, np.float64)
        f = _np(p.fnodal, np.float64)
        nits = np.zeros((p.max_steps, self.n_inst), np.int32)
        kits = np.zeros(self.n_inst, np.int32)
        st = np.zeros(self.n_inst, np.int32)
        bs = L.BatchStats()
        rc = self.lib.mphy_batch_newton_run(self.h, f.ctypes.data_as(L._d), C.byref(o), u.ctypes.data_as(L._d),
                                            nits.ctypes.data_as(L._i32), kits.ctypes.data_as(L._i32),
                                            st.ctypes.data_as(L._i32), C.byref(bs))
        L.check(rc)
        tot, cuts, done = (np.zeros(self.n_inst, np.int32) for _ in range(3))
        tr = np.zeros(self.n_inst, np.float64)
        L.check(self.lib.mphy_batch_instance_info(self.h, tot.ctypes.data_as(L._i32), cuts.ctypes.data_as(L._i32),
                                                  done.ctypes.data_as(L._i32), tr.ctypes.data_as(L._d)))
        return dict(disp=u, newton_its=nits[:bs.steps], krylov_its=kits, status=st, newton_total=tot, cuts=cuts,
                    steps_done=done, t=tr,
                    stats=dict(steps=bs.steps, graph_replays=bs.graph_replays, kernel_launches=bs.kernel_launches,
                               t_ms=bs.t_ms))

    def instance_slice(self, i: int):
        """DOF range of instance i in the union vectors."""
        return slice(3 * int(self.node_ptr[i]), 3 * int(self.node_ptr[i + 1]))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
