"""GPU arc-length continuation (mphy_arclength_run) against the oracle's restatement of
femSolidmechanics::solveWithArclength: the same attempts and iterations per step, load factors
to 1e-9 relative, final displacements to 1e-8 (FP64; consistent tangent, CG to 1e-12), and to
1e-6 in mixed precision."""
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
    return api, _lib, api.Context(0)


@pytest.fixture
def consistent(oracle):
    oracle.set_consistent_tangent(True)
    yield
    oracle.set_consistent_tangent(False)


def _cantilever(steps=6):
    p = meshgen.hex8_cantilever(8, 2, 2, traction=(0.0, 0.0, -0.05))
    p.dt, p.t_final, p.max_steps = 0.1, 2.0, steps
    return p


def _attempts(hist, n):
    return [int(((hist[:, 0] == k) & (hist[:, 1] == 1)).sum()) for k in range(1, n + 1)]


def test_arclength_matches_oracle(env, oracle, consistent):
    api, _lib, ctx = env
    p = _cantilever()
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-12, tangent=_lib.TANGENT_CONSISTENT)
    res = fem.solveWithArclength(max_newton=10, tol_abs=1e-10)
    assert res.status == 0
    u, lam, hist = oracle.OracleProblem(p).arclength(tol_abs=1e-10, cg_rtol=1e-12, max_newton=10)
    assert np.array_equal(res.hist[:, :2], hist[:, :2])
    assert np.allclose(res.load_factors, lam, rtol=1e-9, atol=0.0)
    assert np.allclose(res.hist[:, 5], hist[:, 4], rtol=1e-9, atol=0.0)
    big = hist[:, 2] > 1e-9 * hist[0, 2]
    assert np.allclose(res.hist[big, 2], hist[big, 2], rtol=1e-6)
    assert np.linalg.norm(res.disp - u) <= 1e-8 * np.linalg.norm(u)


def test_failed_attempt_and_retry_match_oracle(env, oracle, consistent):
    api, _lib, ctx = env
    p = _cantilever(steps=5)
    x = p.coords
    u0 = np.zeros_like(x)
    s = x[:, 0] / x[:, 0].max()
    u0[:, 2] = 0.3 * s * s
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-12, tangent=_lib.TANGENT_CONSISTENT)
    res = fem.solveWithArclength(max_newton=12, tol_abs=1e-9, disp=u0.ravel())
    assert res.status == 0
    u, lam, hist = oracle.OracleProblem(p).arclength(tol_abs=1e-9, cg_rtol=1e-12, max_newton=12, disp=u0.ravel())
    assert _attempts(res.hist, 5) == _attempts(hist, 5) == [1, 2, 1, 1, 1]
    assert np.allclose(res.load_factors, lam, rtol=1e-9, atol=0.0)
    assert np.linalg.norm(res.disp - u) <= 1e-8 * np.linalg.norm(u)


def test_mixed_precision_arclength(env, oracle, consistent):
    api, _lib, ctx = env
    p = _cantilever()
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-10, tangent=_lib.TANGENT_CONSISTENT, precision=_lib.PREC_MIXED,
                                   norm_type=1)
    res = fem.solveWithArclength(max_newton=10, tol_abs=1e-9)
    assert res.status == 0
    u, lam, _ = oracle.OracleProblem(p).arclength(tol_abs=1e-9, cg_rtol=1e-12, max_newton=10)
    assert len(res.load_factors) == len(lam)
    assert np.allclose(res.load_factors, lam, rtol=1e-6, atol=0.0)
    assert np.linalg.norm(res.disp - u) <= 1e-6 * np.linalg.norm(u)


def test_first_step_failure_is_reported(env):
    api, _lib, ctx = env
    p = _cantilever()
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-12, tangent=_lib.TANGENT_CONSISTENT)
    res = fem.solveWithArclength(max_newton=2, tol_abs=1e-10)  # one iteration per step
    assert res.status == _lib.ERR_NOT_CONVERGED
    assert len(res.load_factors) == 0 and res.hist.shape[0] == 1


def test_repeated_solve_reuses_the_preconditioner(env):
    # two solves on one assembly (the arc-length pattern) give the same answers as two assemblies
    import torch
    api, _lib, ctx = env
    p = meshgen.hex8_cantilever(8, 3, 3)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), rtol=1e-12, coarse_aggregates=8, norm_type=1)
    u = torch.zeros(p.n_dof, dtype=torch.float64, device="cuda")
    f = torch.tensor(p.fnodal, device="cuda")
    sol.calcStiffnessAndResidual(u)
    sol.addExternalForces(f, 0.2)
    rc1, its1, _ = sol.factoriseAndSolve()
    x1 = sol.solution().clone()
    sol.addExternalForces(f, 0.2)  # rhs = 0.4 f: a second solve on the same operator
    rc2, its2, _ = sol.factoriseAndSolve()
    x2 = sol.solution().clone()
    assert rc1 == rc2 == 0
    assert torch.linalg.norm(x2 - 2.0 * x1).item() <= 1e-9 * torch.linalg.norm(x2).item()
