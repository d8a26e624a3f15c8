"""Two-level coarse correction (rigid-body or linear modes) against its numpy restatement and the FP64 oracle.

Same aggregate grid on both sides: iteration counts agree within 3 % (summation order only);
solutions agree with the oracle's FP64 CG to 1e-9 (FP64 path) at rtol 1e-12, and the coarse
correction needs at most half the Jacobi iterations on the cantilever."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return torch, api, _lib, api.Context(0)


def _solve(api, _lib, ctx, p, torch, **opts):
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, **opts)
    sol.calcStiffnessAndResidual(torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"))
    sol.addExternalForces(torch.tensor(p.fnodal, device="cuda"), 0.2)
    rc, its, fn = sol.factoriseAndSolve()
    return sol, pat, rc, its, sol.solution().cpu().numpy()


@pytest.mark.parametrize("modes", [6, 12])
@pytest.mark.parametrize("mk", [meshgen.cantilever_small,
                                lambda: meshgen.two_phase_inclusions(32, 8, 8, seed=23, r_range=(0.1, 0.25))])
def test_coarse_matches_restatement_and_oracle(env, oracle, mk, modes):
    from oracle import fsai_ref, twolevel_ref
    torch, api, _lib, ctx = env
    p = mk()
    sol, pat, rc, its, x = _solve(api, _lib, ctx, p, torch, rtol=1e-12, coarse_aggregates=24, coarse_modes=modes)
    assert rc == 0
    info = sol.coarse_info()
    _, _, _, itj, _ = _solve(api, _lib, ctx, p, torch, rtol=1e-12)
    assert its <= 0.5 * itj, (its, itj)
    op = oracle.OracleProblem(p)
    val, _, _, _ = op.assemble(np.zeros(p.n_dof))
    free = np.flatnonzero(p.fixed == 0)
    xo, _, _, _ = op.cg(val, 0.2 * p.fnodal[free], rtol=1e-13)
    assert np.linalg.norm(x[free] - xo) <= 1e-9 * np.linalg.norm(xo)
    _, _, rp, col = op.pattern()
    A = fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val)
    assert info["coarse_size"] == modes * int(np.prod(info["grid"]))
    Minv = twolevel_ref.preconditioner(A, p.coords, p.fixed, info["grid"], modes)
    _, its_ref = twolevel_ref.pcg(A, 0.2 * p.fnodal * (p.fixed == 0), Minv, rtol=1e-12)
    assert abs(its - its_ref) <= max(2, 0.03 * its_ref), (its, its_ref)


def test_coarse_mixed_and_newton(env):
    torch, api, _lib, ctx = env
    p = meshgen.cantilever_small()
    _, _, rc, its, x = _solve(api, _lib, ctx, p, torch, rtol=1e-10, coarse_aggregates=24, precision=_lib.PREC_MIXED)
    _, _, rc2, its2, x2 = _solve(api, _lib, ctx, p, torch, rtol=1e-10, coarse_aggregates=24)
    assert rc == 0 and rc2 == 0 and abs(its - its2) <= max(3, 0.05 * its2)
    fem = api.FemSolidmechanicsGpu(p, ctx, tangent=1, rtol=1e-10, coarse_aggregates=24)
    res = fem.solveWithNewtonRaphson(max_newton=15)
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "cantilever_32x8x8.npz"))
    assert res.status == 0
    assert np.abs(res.disp - g["newton_consistent_u"]).max() <= 1e-8 * np.abs(g["newton_consistent_u"]).max()


def test_linear_modes_need_fewer_iterations(env):
    # the linear-displacement space contains the rigid-body one: at equal aggregates it can only
    # help, and at equal coarse size (half the aggregates) it still beats it on the cantilever
    torch, api, _lib, ctx = env
    p = meshgen.hex8_cantilever(64, 16, 16)
    its = {}
    for agg, modes in ((64, 6), (64, 12), (32, 12)):
        _, _, rc, it, _ = _solve(api, _lib, ctx, p, torch, rtol=1e-10, coarse_aggregates=agg, coarse_modes=modes,
                                 norm_type=1)
        assert rc == 0
        its[(agg, modes)] = it
    assert its[(64, 12)] < its[(64, 6)], its


def test_many_aggregates_one_item_each(env, oracle):
    """About 1,400 aggregates, more than two per resident CTA of the E = Z^T A Z kernel and of the
    restriction. Both then take one work item per aggregate, with no cross-CTA part sums. The
    checks are the same as above: the FP64 oracle's solution, and the iteration count of the
    numpy restatement on the same aggregate grid."""
    from oracle import fsai_ref, twolevel_ref
    torch, api, _lib, ctx = env
    p = meshgen.hex8_cantilever(40, 20, 20)
    sol, pat, rc, its, x = _solve(api, _lib, ctx, p, torch, rtol=1e-12, coarse_aggregates=1500)
    assert rc == 0
    info = sol.coarse_info()
    assert int(np.prod(info["grid"])) >= 1184, info  # 2 x (4 CTAs per SM x 148 SMs)
    op = oracle.OracleProblem(p)
    val, _, _, _ = op.assemble(np.zeros(p.n_dof))
    free = np.flatnonzero(p.fixed == 0)
    xo, _, _, _ = op.cg(val, 0.2 * p.fnodal[free], rtol=1e-13)
    assert np.linalg.norm(x[free] - xo) <= 1e-9 * np.linalg.norm(xo)
    _, _, rp, col = op.pattern()
    A = fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val)
    Minv = twolevel_ref.preconditioner(A, p.coords, p.fixed, info["grid"])
    _, its_ref = twolevel_ref.pcg(A, 0.2 * p.fnodal * (p.fixed == 0), Minv, rtol=1e-12)
    assert abs(its - its_ref) <= max(2, 0.03 * its_ref), (its, its_ref)
