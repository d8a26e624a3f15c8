"""GPU parity against the CPU oracle, through the C ABI (config 1 and small tet10 meshes).

Tolerances: integer/index results (DOF numbering, CSR pattern) are bit-exact. FP64 element
matrices, assembled values and residuals agree to 1e-12 relative to the largest entry (the only
differences are summation order, cbrt vs pow, and cofactor vs LU inverses). Solutions agree to
1e-9 relative (CG to rtol 1e-12 in different summation orders). Newton residual norms agree to
1e-6 relative above the 1e-9*||R_0|| roundoff floor.
"""
import os

import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cantilever_32x8x8.npz")


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no GPU")
    return t


@pytest.fixture(scope="module")
def api(torch):
    from mphyfem_b200 import api as a, build
    build.build()
    return a


@pytest.fixture(scope="module")
def ctx(api):
    return api.Context(0)


def _small_tet10():
    p = meshgen.tet10_kuhn(4, 2, 2, lx=2.0)
    return p


def _mixed_constraints(p):
    p.fixed = p.fixed.copy()
    p.fixed[3 * (p.n_node - 1) + 1] = 1
    p.fixed[3 * (p.n_node // 2) + 2] = 1
    return p


def test_material_matches_oracle(api, ctx, oracle, torch):
    rng = np.random.default_rng(1)
    F = np.eye(3)[None] + 0.15 * rng.standard_normal((64, 3, 3))
    for utype in (3, 1, 4, 7):
        for tangent in (0, 1):
            oracle.set_consistent_tangent(bool(tangent))
            try:
                ref = [oracle.nh_stress_tangent(f, 0.8, 0.05, utype) for f in F]
            finally:
                oracle.set_consistent_tangent(False)
            s, Cm = api.compute_stress_and_tangent(ctx, torch.tensor(F, device="cuda"), 0.8, 0.05, utype, tangent)
            s, Cm = s.cpu().numpy(), Cm.cpu().numpy()
            for k in range(len(F)):
                assert np.abs(s[k] - ref[k][0]).max() <= 1e-12 * max(1.0, np.abs(ref[k][0]).max())
                assert np.abs(Cm[k] - ref[k][1]).max() <= 1e-12 * max(1.0, np.abs(ref[k][1]).max())


@pytest.mark.parametrize("mk", [meshgen.cantilever_small, _small_tet10])
def test_element_matrices_match_oracle(api, ctx, oracle, torch, mk):
    from tests.golden.make_golden import probe_displacement
    p = mk()
    u = probe_displacement(p, amp=0.01)
    mesh = api.Mesh(ctx, p)
    Ke, Re, bad = api.calc_stiffness_and_residual(mesh, torch.tensor(u, device="cuda"))
    assert bad == -1
    Ke, Re = Ke.cpu().numpy(), Re.cpu().numpy()
    Ko, Ro, bo = oracle.OracleProblem(p).elements(u)
    assert bo == -1
    kscale = np.abs(Ko).max(axis=(1, 2))
    rscale = np.abs(Ro).max(axis=1)
    assert np.all(np.abs(Ke - Ko).max(axis=(1, 2)) <= 1e-12 * kscale)
    assert np.all(np.abs(Re - Ro).max(axis=1) <= 1e-12 * rscale + 1e-18)


@pytest.mark.parametrize("mk", [meshgen.cantilever_small, _small_tet10,
                                lambda: _mixed_constraints(meshgen.hex8_cantilever(7, 3, 2)),
                                lambda: _mixed_constraints(_small_tet10())])
def test_pattern_bit_exact(api, ctx, oracle, mk):
    p = mk()
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    op = oracle.OracleProblem(p)
    afs, fav, rp, col = op.pattern()
    assert pat.n_free == op.n_free and pat.nnz == op.nnz
    g_rp, g_col = pat.export_csr()
    g_afs, g_fav = pat.export_dofmap()
    assert np.array_equal(g_rp, rp)
    assert np.array_equal(g_col, col)
    assert np.array_equal(g_afs, afs)
    assert np.array_equal(g_fav, fav)


def test_config1_pattern_matches_golden(api, ctx):
    import hashlib
    g = np.load(GOLD)
    pat = api.Pattern(api.Mesh(ctx, meshgen.cantilever_small()))
    rp, col = pat.export_csr()
    assert hashlib.sha256(rp.tobytes()).hexdigest() == str(g["rowptr_sha"])
    assert hashlib.sha256(col.astype(np.int32).tobytes()).hexdigest() == str(g["col_sha"])


@pytest.mark.parametrize("mk", [meshgen.cantilever_small, _small_tet10,
                                lambda: _mixed_constraints(meshgen.hex8_cantilever(7, 3, 2))])
def test_assembly_matches_oracle(api, ctx, oracle, torch, mk):
    from tests.golden.make_golden import probe_displacement
    p = mk()
    u = probe_displacement(p, amp=0.01)
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat)
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    assert sol.currentStatus == 3  # ASSEMBLY_OK
    val, rhs, reac = sol.export()
    oval, orhs, oreac, bad = oracle.OracleProblem(p).assemble(u)
    assert bad == -1
    assert np.abs(val - oval).max() <= 1e-12 * np.abs(oval).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    assert np.abs(reac - oreac).max() <= 1e-12 * np.abs(oreac).max()
    # the drop-in batch scatter of externally computed element matrices gives the same system
    Ke, Re, _ = api.calc_stiffness_and_residual(mesh, torch.tensor(u, device="cuda"))
    sol.zeroMtx()
    sol.assembleMatrixAndVector(Ke, Re)
    val2, rhs2, reac2 = sol.export()
    assert np.abs(val2 - oval).max() <= 1e-12 * np.abs(oval).max()
    assert np.abs(rhs2 - orhs).max() <= 1e-12 * np.abs(orhs).max()


def test_golden_probe_assembly(api, ctx, torch):
    g = np.load(GOLD)
    p = meshgen.cantilever_small()
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh))
    sol.calcStiffnessAndResidual(torch.tensor(g["probe_u"], device="cuda"))
    val, rhs, reac = sol.export()
    assert np.abs(rhs - g["probe_rhs"]).max() <= 1e-12 * np.abs(g["probe_rhs"]).max()
    assert np.abs(reac - g["probe_reac"]).max() <= 1e-12 * np.abs(g["probe_reac"]).max()
    assert abs(np.abs(val).sum() - float(g["probe_val_abs"])) <= 1e-12 * float(g["probe_val_abs"])


def test_pcg_matches_oracle(api, ctx, oracle, torch):
    p = meshgen.cantilever_small()
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), rtol=1e-12)
    sol.calcStiffnessAndResidual(torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"))
    sol.addExternalForces(torch.tensor(p.fnodal, device="cuda"), 0.2)
    rc, its, fn = sol.factoriseAndSolve()
    x = sol.solution().cpu().numpy()
    op = oracle.OracleProblem(p)
    val, _, _, _ = op.assemble(np.zeros(p.n_dof))
    b = 0.2 * p.fnodal[np.flatnonzero(p.fixed == 0)]
    xo, itso, fno, st = op.cg(val, b, rtol=1e-12)
    assert rc == 0 and st == 0
    assert abs(its - itso) <= 2
    free = np.flatnonzero(p.fixed == 0)
    assert np.linalg.norm(x[free] - xo) <= 1e-9 * np.linalg.norm(xo)
    assert np.all(x[p.fixed == 1] == 0.0)


def test_solve_before_assembly_is_refused(api, ctx):
    from mphyfem_b200 import _lib
    p = meshgen.hex8_cantilever(4, 2, 2)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh))
    rc, _, _ = sol.factoriseAndSolve(allow_fail=True)
    assert rc == _lib.ERR_STATE


def test_negative_jacobian_reports_first_element(api, ctx, torch):
    from mphyfem_b200 import _lib
    p = meshgen.hex8_cantilever(4, 2, 2)
    u = np.zeros((p.n_node, 3))
    bad_elems = [5, 9]
    for e in bad_elems:
        # collapse element e through itself: move its +x face behind its -x face
        for a in (1, 2, 5, 6):
            u[p.conn[e, a], 0] = -3.0 * (p.coords[p.conn[e, a], 0] - p.coords[p.conn[e, 0], 0])
    mesh = api.Mesh(ctx, p)
    _, _, bad = api.calc_stiffness_and_residual(mesh, torch.tensor(u.ravel(), device="cuda"))
    assert bad >= 0 and bad <= min(bad_elems)
    sol = api.SolverGpu(mesh, api.Pattern(mesh))
    with pytest.raises(_lib.MphyError) as ei:
        sol.calcStiffnessAndResidual(torch.tensor(u.ravel(), device="cuda"))
    assert ei.value.status == _lib.ERR_NEG_JACOBIAN


def test_newton_consistent_tangent_matches_golden(api, ctx):
    g = np.load(GOLD)
    p = meshgen.cantilever_small()
    fem = api.FemSolidmechanicsGpu(p, ctx, tangent=1)
    res = fem.solveWithNewtonRaphson(max_newton=15)
    gh = g["newton_consistent_hist"]
    h = res.hist
    assert res.status == 0
    assert h.shape[0] == gh.shape[0]
    assert np.array_equal(h[:, :2], gh[:, :2])
    floor = 1e-9 * gh[0, 2]
    big = gh[:, 2] > floor
    assert np.allclose(h[big, 2], gh[big, 2], rtol=1e-6)
    assert np.all(h[~big, 2] < 1e-10 * gh[0, 2])
    assert np.abs(res.disp - g["newton_consistent_u"]).max() <= 1e-9 * np.abs(g["newton_consistent_u"]).max()


def test_newton_reference_tangent_step_with_cut(api, ctx):
    g = np.load(GOLD)
    p = meshgen.cantilever_small()
    p.max_steps = 1
    fem = api.FemSolidmechanicsGpu(p, ctx)
    res = fem.solveWithNewtonRaphson(max_newton=10)
    h = res.hist
    assert h[0, 2] == pytest.approx(1.171875e-3, rel=1e-12)
    gh = g["newton_reference_step_hist"]
    assert h[2:, 2].shape == gh[:, 2].shape  # first attempt (2 rows) fails, retried at dt = 0.1
    floor = 1e-9 * gh[0, 2]
    big = gh[:, 2] > floor
    assert np.allclose(h[2:][big, 2], gh[big, 2], rtol=1e-6)
    assert np.abs(res.disp - g["newton_reference_step_u"]).max() <= 1e-9 * np.abs(g["newton_reference_step_u"]).max()
