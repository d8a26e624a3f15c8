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


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_coarse_with_residual_norm_matches_restatement(env, oracle, prec):
    """The ||r|| test (the iteration completes (r, z) from (r, D^-1 r) and (Z^T r, E^-1 Z^T r) and
    forms z only inside the direction update). FP64: iteration count within 3 % of the numpy
    restatement with the same test, solution to 1e-9 of the FP64 oracle's. Mixed: the solve is of
    the FP32-stored operator (on this two-phase mesh its solution differs from the FP64 one by
    the FP32 rounding times the condition number), so it is held to its own FP64 true residual
    (1e-8, up to four refinement sweeps; this mesh's FP64 round-off floor is about 6e-10) and to
    the FP64 solve's iteration count at the same settings (5 %)."""
    from oracle import fsai_ref, twolevel_ref
    torch, api, _lib, ctx = env
    p = meshgen.two_phase_inclusions(32, 8, 8, seed=23, r_range=(0.1, 0.25))
    precision = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
    if prec == "mixed":
        sol, pat, rc, its, x = _solve(api, _lib, ctx, p, torch, rtol=1e-8, coarse_aggregates=24, norm_type=1,
                                      precision=precision, max_outer=4)
        assert rc == 0
        assert sol.true_residual() <= 1e-8
        _, _, rc64, its64, _ = _solve(api, _lib, ctx, p, torch, rtol=1e-8, coarse_aggregates=24, norm_type=1,
                                      max_outer=4)
        assert rc64 == 0 and abs(its - its64) <= max(3, 0.05 * its64), (its, its64)
        return
    sol, pat, rc, its, x = _solve(api, _lib, ctx, p, torch, rtol=1e-12, coarse_aggregates=24, norm_type=1)
    assert rc == 0
    info = sol.coarse_info()
    op = oracle.OracleProblem(p)
    val, _, _, _ = op.assemble(np.zeros(p.n_dof))
    free = np.flatnonzero(p.fixed == 0)
    xo, _, _, _ = op.cg(val, 0.2 * p.fnodal[free], rtol=1e-13)
    assert np.linalg.norm(x[free] - xo) <= 1e-9 * np.linalg.norm(xo)
    if prec == "fp64":
        _, _, rp, col = op.pattern()
        A = fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val)
        Minv = twolevel_ref.preconditioner(A, p.coords, p.fixed, info["grid"], 6)
        _, its_ref = twolevel_ref.pcg(A, 0.2 * p.fnodal * (p.fixed == 0), Minv, rtol=1e-12, norm_type=1)
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


def test_coarse_lag_keeps_the_operator(env, oracle):
    """coarse_lag = 2: a solve forms the coarse operator and the next two solves keep it (setup
    time 0), whatever their matrices; each solve still meets its own tolerance, so the solutions
    agree with the FP64 oracle's on each solve's own matrix. In Newton, the first iteration of
    every load step forms it afresh, and the converged displacements equal the golden ones."""
    from tests.golden.make_golden import probe_displacement
    torch, api, _lib, ctx = env
    p = meshgen.cantilever_small()
    mesh = api.Mesh(ctx, p)
    # the consistent tangent at displacements small enough that it stays positive definite (the
    # oracle's CG converges on each), as CG needs
    sol = api.SolverGpu(mesh, api.Pattern(mesh), rtol=1e-12, coarse_aggregates=24, coarse_lag=2, norm_type=1,
                        tangent=_lib.TANGENT_CONSISTENT)
    op = oracle.OracleProblem(p)
    free = np.flatnonzero(p.fixed == 0)
    formed = []
    oracle.set_consistent_tangent(True)
    try:
        for k in range(4):
            u = 0.1 * probe_displacement(p, seed=5 + k, amp=0.005)  # small enough for an SPD tangent
            sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
            sol.addExternalForces(torch.tensor(p.fnodal, device="cuda"), 0.2)
            rc, its, _ = sol.factoriseAndSolve()
            assert rc == 0
            formed.append(sol.coarse_info()["setup_ms"] > 0.0)
            val, rhs, _, _ = op.assemble(u)
            xo, _, _, _ = op.cg(val, rhs + 0.2 * p.fnodal[free], rtol=1e-13)
            x = sol.solution().cpu().numpy()
            assert np.linalg.norm(x[free] - xo) <= 1e-9 * np.linalg.norm(xo)
    finally:
        oracle.set_consistent_tangent(False)
    assert formed == [True, False, False, True], formed
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "cantilever_32x8x8.npz"))
    fem = api.FemSolidmechanicsGpu(p, ctx, tangent=1, rtol=1e-10, coarse_aggregates=24, coarse_lag=3, norm_type=1)
    r = fem.solveWithNewtonRaphson(max_newton=15)
    assert r.status == 0
    assert np.abs(r.disp - g["newton_consistent_u"]).max() <= 1e-8 * np.abs(g["newton_consistent_u"]).max()


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
    """About 1,400 aggregates (19,600 (aggregate, slot) CTAs of the E = Z^T A Z sum kernel), more
    than two per resident CTA of the restriction, which then takes one work item per aggregate,
    with no cross-CTA part sums. The checks are the same as above: the FP64 oracle's solution,
    and the iteration count of the numpy restatement on the same aggregate grid."""
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


@pytest.mark.parametrize("prec,modes", [("fp64", 6), ("mixed", 6), ("fp64", 12)])
def test_coarse_operator_is_bitwise_reproducible(env, prec, modes):
    """E = Z^T A Z is summed in a fixed order, with no atomics: per-row sums per neighbour box,
    then a fixed list per (aggregate, neighbour). Two solves of one assembled system, each
    forming E and its inverse afresh, give bitwise equal solutions and equal iteration counts."""
    torch, api, _lib, ctx = env
    p = meshgen.hex8_cantilever(48, 12, 12)
    mesh = api.Mesh(ctx, p)
    opts = dict(rtol=1e-10, coarse_aggregates=60, coarse_modes=modes, norm_type=1)
    if prec == "mixed":
        opts["precision"] = _lib.PREC_MIXED
    sol = api.SolverGpu(mesh, api.Pattern(mesh), **opts)
    sol.calcStiffnessAndResidual(torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"))
    sol.addExternalForces(torch.tensor(p.fnodal, device="cuda"), 0.2)
    runs = []
    for _ in range(2):
        rc, its, _ = sol.factoriseAndSolve()
        assert rc == 0
        assert sol.coarse_info()["setup_ms"] > 0.0  # formed by this solve
        runs.append((its, sol.solution().cpu().numpy().copy()))
    assert runs[0][0] == runs[1][0], (runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_coarse_numbering_follows_the_long_axis(env):
    """The aggregates are numbered with the axis of most boxes slowest, so E is banded and the
    factorisation skips the tiles outside the band, whichever physical axis that is. The
    cantilever along x and the same cantilever turned (a cyclic permutation of the axes) to lie
    along y give the same iteration count (within 2) and the same displacements (to 1e-9)."""
    import dataclasses
    torch, api, _lib, ctx = env
    p = meshgen.hex8_cantilever(48, 12, 12)
    perm = [2, 0, 1]  # new axis k is old axis perm[k]; a proper rotation
    q = dataclasses.replace(p, coords=np.ascontiguousarray(p.coords[:, perm]),
                            fixed=np.ascontiguousarray(p.fixed.reshape(-1, 3)[:, perm].ravel()),
                            fnodal=np.ascontiguousarray(p.fnodal.reshape(-1, 3)[:, perm].ravel()))
    s1, _, rc1, its1, x1 = _solve(api, _lib, ctx, p, torch, rtol=1e-10, coarse_aggregates=60, norm_type=1)
    s2, _, rc2, its2, x2 = _solve(api, _lib, ctx, q, torch, rtol=1e-10, coarse_aggregates=60, norm_type=1)
    assert rc1 == 0 and rc2 == 0
    g1, g2 = s1.coarse_info()["grid"], s2.coarse_info()["grid"]
    assert list(g2) == [g1[a] for a in perm], (g1, g2)
    assert abs(its1 - its2) <= 2, (its1, its2)
    back = x2.reshape(-1, 3)[:, np.argsort(perm)].ravel()
    assert np.linalg.norm(back - x1) <= 1e-9 * np.linalg.norm(x1)
