"""Mixed precision (MPHY_PREC_MIXED) against the FP64 oracle.

The tangent is stored in FP32 and solved by an FP32 PCG inside an FP64 iterative-refinement
loop; the Newton residual stays FP64. Tolerances: FP32 matrix values within 1e-6 of the largest
entry (one rounding), FP64 residual within 1e-12, refined solutions within 1e-8 relative of the
FP64 solve at rtol 1e-10, Newton displacements within 1e-6 of the FP64 golden run.
"""
import os

import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cantilever_32x8x8.npz")


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return torch, api, _lib, api.Context(0)


def test_mixed_assembly_matches_oracle(env, oracle):
    from tests.golden.make_golden import probe_displacement
    torch, api, _lib, ctx = env
    p = meshgen.cantilever_small()
    u = probe_displacement(p, amp=0.01)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), precision=_lib.PREC_MIXED)
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    val, rhs, reac = sol.export()
    oval, orhs, oreac, _ = oracle.OracleProblem(p).assemble(u)
    # off-diagonal entries: one FP32 rounding; diagonal blocks: minus the sum of the rounded
    # off-diagonal blocks of the row (about 27 roundings)
    assert np.abs(val - oval).max() <= 1e-5 * np.abs(oval).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    assert sol.matrix_info()["value_bytes"] == 4 * 9 * sol.matrix_info()["stored_blocks"]


@pytest.mark.parametrize("prec", ["PREC_MIXED", "PREC_MIXED_F32VEC"])
def test_mixed_solve_refines_to_fp64_accuracy(env, oracle, prec):
    """The refined solution solves the FP32-stored operator A32 x = b to the FP64 tolerance; it
    differs from the FP64 operator's solution by about cond(A) * 6e-8 (here ~1e-3)."""
    import scipy.sparse as sp
    torch, api, _lib, ctx = env
    p = meshgen.cantilever_small()
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    zero = torch.zeros(p.n_dof, dtype=torch.float64, device="cuda")
    f = torch.tensor(p.fnodal, device="cuda")
    sol = api.SolverGpu(mesh, pat, precision=getattr(_lib, prec), rtol=1e-10, inner_rtol=1e-4, max_outer=50)
    sol.calcStiffnessAndResidual(zero)
    sol.addExternalForces(f, 0.2)
    rc, its, relres = sol.factoriseAndSolve()
    assert rc == 0 and relres <= 1e-10
    x = sol.solution().cpu().numpy()
    val32, _, _ = sol.export(want_rhs=False, want_reac=False)
    rp, col = pat.export_csr()
    free = np.flatnonzero(p.fixed == 0)
    A32 = sp.csr_matrix((val32, col, rp), shape=(pat.n_free, pat.n_free))
    b = 0.2 * p.fnodal[free]
    assert np.linalg.norm(b - A32 @ x[free]) <= 2e-10 * np.linalg.norm(b)
    op = oracle.OracleProblem(p)
    val, _, _, _ = op.assemble(np.zeros(p.n_dof))
    xo, _, _, _ = op.cg(val, b, rtol=1e-13)
    assert np.linalg.norm(x[free] - xo) <= 1e-2 * np.linalg.norm(xo)
    assert np.all(x[p.fixed == 1] == 0.0)


@pytest.mark.parametrize("prec", ["PREC_FP64", "PREC_MIXED"])
def test_stored_operator_annihilates_translations(env, prec):
    """Null-space-preserving storage: the FP32 operator's diagonal blocks are minus the sums of the
    stored off-diagonal blocks, so A t = 0 for a rigid translation t on every block row whose
    neighbours are all free -- exactly up to FP64 summation, not up to FP32 rounding."""
    from tests.golden.make_golden import probe_displacement
    torch, api, _lib, ctx = env
    p = meshgen.two_phase_inclusions(24, 6, 6, seed=3, r_range=(0.15, 0.3))
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), precision=getattr(_lib, prec))
    sol.calcStiffnessAndResidual(torch.tensor(probe_displacement(p, amp=0.005), device="cuda"))
    near_clamp = p.coords[:, 0] <= 4.0 / 24 + 1e-12
    for d in range(3):
        t = np.zeros((p.n_node, 3))
        t[:, d] = 1.0
        t[p.fixed.reshape(-1, 3) == 1] = 0.0
        y = torch.empty(p.n_dof, dtype=torch.float64, device="cuda")
        sol.spmv(torch.tensor(t.ravel(), device="cuda"), y)
        torch.cuda.synchronize()
        y = y.cpu().numpy().reshape(-1, 3)
        val, _, _ = sol.export(want_rhs=False, want_reac=False)
        assert np.abs(y[~near_clamp]).max() <= 1e-12 * np.abs(val).max()


def test_mixed_newton_reaches_fp64_solution(env):
    torch, api, _lib, ctx = env
    g = np.load(GOLD)
    p = meshgen.cantilever_small()
    fem = api.FemSolidmechanicsGpu(p, ctx, tangent=1, precision=_lib.PREC_MIXED, rtol=1e-8)
    res = fem.solveWithNewtonRaphson(max_newton=20)
    assert res.status == 0
    h = res.hist
    for s in np.unique(h[:, 0]):
        r = h[h[:, 0] == s, 2]
        assert r[-1] < 1e-10 * r[0]
    u_ref = g["newton_consistent_u"]
    assert np.abs(res.disp - u_ref).max() <= 1e-6 * np.abs(u_ref).max()


@pytest.mark.parametrize("case", ["hex8_two_phase", "tet10_kuhn"])
@pytest.mark.parametrize("tangent", [0, 1], ids=["reference", "consistent"])
def test_fp32_tangent_kernel_matches_oracle(env, oracle, case, tangent):
    """The mixed-precision element kernel (FP64 kinematics, stress and residual; FP32 tangent
    blocks, each symmetric pair formed once) against the FP64 oracle: off-diagonal entries within
    1e-5 of the largest entry (FP32 arithmetic and storage), the operator's diagonal blocks (minus
    the stored rows' sums) likewise, residual and reactions within 1e-12 (FP64)."""
    from tests.golden.make_golden import probe_displacement
    torch, api, _lib, ctx = env
    if case == "hex8_two_phase":
        p = meshgen.two_phase_inclusions(16, 4, 4, seed=3, r_range=(0.15, 0.3))
    else:
        p = meshgen.tet10_kuhn(6, 3, 3)
    u = probe_displacement(p, amp=0.005)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), precision=_lib.PREC_MIXED, tangent=tangent)
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    val, rhs, reac = sol.export()
    oracle.set_consistent_tangent(bool(tangent))
    try:
        oval, orhs, oreac, bad = oracle.OracleProblem(p).assemble(u)
    finally:
        oracle.set_consistent_tangent(False)
    assert bad == -1
    assert np.abs(val - oval).max() <= 1e-5 * np.abs(oval).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    assert np.abs(reac - oreac).max() <= 1e-12 * np.abs(oreac).max()
