"""The constant-pressure mixed element (Elem_Solid_3D_Mixed0: hex8 or tet10 displacement, one
pressure per element, condensed) on the GPU against the oracle's restatement.

Tolerances: the condensed system assembled at a probe state (displacement, last-step displacement,
element pressures) within 1e-12 of the largest entry (FP64), and a near-incompressible Newton run
(kappa/mu = 1e3, consistent tangent, two load steps, Newton to 1e-8: the FP64 residual floor lies
near 1e-10 of the first residual) with the oracle's residual history (1e-6 relative above
round-off), displacements and element pressures within 1e-8.
"""
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


def _mesh(kind):
    if kind == "hex8":
        return meshgen.hex8_cantilever(12, 3, 3, kappa=1.0e3)
    return meshgen.tet10_kuhn(6, 2, 2, kappa=1.0e3)


@pytest.mark.parametrize("kind", ["hex8", "tet10"])
@pytest.mark.parametrize("tangent", [0, 1], ids=["reference", "consistent"])
def test_condensed_assembly_matches_oracle(env, oracle, kind, tangent):
    from tests.golden.make_golden import probe_displacement
    torch, api, _lib, ctx = env
    p = _mesh(kind)
    rng = np.random.default_rng(9)
    u = probe_displacement(p, amp=0.004)
    up = 0.5 * u
    pe = 0.05 * rng.standard_normal(p.n_elem)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), tangent=tangent)
    sol.set_mixed_p0(True)
    sol.p0_pressure(pe)
    sol.save_step(torch.tensor(up, device="cuda"))
    sol.p0_pressure(pe)
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    val, rhs, reac = sol.export()
    oracle.set_consistent_tangent(bool(tangent))
    try:
        op = oracle.OracleProblem(p)
        op.set_mixed_p0(True)
        op.save_step(up)
        op.p0_pressure(pe)
        oval, orhs, oreac, bad = op.assemble(u)
    finally:
        oracle.set_consistent_tangent(False)
    assert bad == -1
    assert np.abs(val - oval).max() <= 1e-12 * np.abs(oval).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    assert np.abs(reac - oreac).max() <= 1e-12 * np.abs(oreac).max()


@pytest.mark.parametrize("kind", ["hex8", "tet10"])
def test_newton_matches_oracle(env, oracle, kind):
    torch, api, _lib, ctx = env
    p = _mesh(kind)
    p.max_steps, p.t_final = 2, 2 * p.dt
    fem = api.FemSolidmechanicsGpu(p, ctx, mixed_p0=True, tangent=1, rtol=1e-12, max_it=50000)
    # Newton to 1e-8: kappa/mu = 1e3 puts the FP64 residual floor near 1e-10 of ||R_0||
    res = fem.solveWithNewtonRaphson(max_newton=15, tol_rel=1e-8)
    assert res.status == 0
    pe = fem.solver.p0_pressure()
    oracle.set_consistent_tangent(True)
    try:
        op = oracle.OracleProblem(p)
        op.set_mixed_p0(True)
        uo, ho = op.newton(tol_rel=1e-8, cg_rtol=1e-12, cg_maxit=50000, max_newton=15, nthreads=4)
        peo = op.p0_pressure()
    finally:
        oracle.set_consistent_tangent(False)
    h = res.hist
    assert h.shape[0] == ho.shape[0], (h[:, :3], ho)
    assert np.array_equal(h[:, :2], ho[:, :2])
    big = ho[:, 2] > 1e-9 * ho[:, 2].max()
    assert np.allclose(h[big, 2], ho[big, 2], rtol=1e-6)
    assert np.abs(res.disp - uo).max() <= 1e-8 * np.abs(uo).max()
    assert np.abs(pe - peo).max() <= 1e-8 * np.abs(peo).max()
    # near incompressibility: the element pressures carry the volumetric stress (nonzero)
    assert np.abs(peo).max() > 0.0
