"""Nonzero prescribed displacements on the GPU against the oracle: the increment of each load step
lifted into the first iteration (applyDirichletBCs) and added with its solution.

Stretch by a prescribed end displacement (hex8 and tet10, FP64): the oracle's Newton history
(residual norms within 1e-6 relative above round-off) and the closed-form homogeneous state
within 1e-9. Bending by a prescribed end displacement, with a constant prescribed part applied in
full from the first step: FP64 within 1e-9 of the oracle, mixed precision with the coarse space
within 1e-6."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen
from tests.test_oracle_prescribed import stretch_block, uniaxial_lateral_stretch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return api, _lib, api.Context(0)


def _oracle_newton(oracle, p, **kw):
    oracle.set_consistent_tangent(True)
    try:
        return oracle.OracleProblem(p).newton(**kw)
    finally:
        oracle.set_consistent_tangent(False)


@pytest.mark.parametrize("split", [False, True], ids=["hex8", "tet10"])
def test_prescribed_stretch_matches_oracle_and_closed_form(env, oracle, split):
    api, _lib, ctx = env
    p = stretch_block(split=split)
    fem = api.FemSolidmechanicsGpu(p, ctx, tangent=1, rtol=1e-13, max_it=20000)
    res = fem.solveWithNewtonRaphson(max_newton=15, tol_rel=1e-12, tol_abs=1e-14)
    assert res.status == 0
    uo, ho = _oracle_newton(oracle, p, tol_rel=1e-12, tol_abs=1e-14, cg_rtol=1e-13, max_newton=15)
    h = res.hist
    assert h.shape[0] == ho.shape[0] and np.array_equal(h[:, :2], ho[:, :2])
    big = ho[:, 2] > 1e-9 * ho[:, 2].max()
    assert np.allclose(h[big, 2], ho[big, 2], rtol=1e-6)
    l1, l2 = 1.1, uniaxial_lateral_stretch(1.1, 1.0, 10.0)
    X = p.coords
    exact = np.stack([(l1 - 1) * X[:, 0], (l2 - 1) * X[:, 1], (l2 - 1) * X[:, 2]], axis=1).ravel()
    assert np.abs(res.disp - exact).max() <= 1e-9
    assert np.abs(res.disp - uo).max() <= 1e-9


def _bending_block():
    """Cantilever 16x4x4 clamped at x = 0; on x = 4 the z-displacement is prescribed: -0.2 t, plus a
    constant 0.01 on the top edge's nodes (applied in full from the first step)."""
    p = meshgen.hex8_cantilever(16, 4, 4, traction=(0, 0, 0))
    X = p.coords
    fx = p.fixed.reshape(-1, 3).copy()
    end = np.isclose(X[:, 0], 4.0)
    fx[end, 2] = 1
    ramp = np.zeros((p.n_node, 3))
    cst = np.zeros((p.n_node, 3))
    ramp[end, 2] = -0.2
    cst[end & np.isclose(X[:, 2], 1.0), 2] = 0.01
    p.fixed = fx.ravel()
    p.presc_ramp, p.presc_const = ramp.ravel(), cst.ravel()
    p.fnodal = np.zeros(p.n_dof)
    return p


@pytest.mark.parametrize("precision", ["PREC_FP64", "PREC_MIXED"])
def test_prescribed_bending_matches_oracle(env, oracle, precision):
    api, _lib, ctx = env
    p = _bending_block()
    opts = dict(tangent=1, rtol=1e-12, max_it=40000, precision=getattr(_lib, precision), norm_type=1)
    if precision == "PREC_MIXED":
        opts.update(coarse_aggregates=8, max_outer=6)
    fem = api.FemSolidmechanicsGpu(p, ctx, **opts)
    res = fem.solveWithNewtonRaphson(max_newton=15, tol_rel=1e-10)
    assert res.status == 0
    uo, ho = _oracle_newton(oracle, p, tol_rel=1e-10, cg_rtol=1e-12, cg_maxit=40000, max_newton=15)
    scale = np.abs(uo).max()
    if precision == "PREC_FP64":
        assert res.hist.shape[0] == ho.shape[0]
        assert np.abs(res.disp - uo).max() <= 1e-9 * scale
    else:
        assert np.abs(res.disp - uo).max() <= 1e-6 * scale
    Xe = np.isclose(p.coords[:, 0], 4.0)
    uz = res.disp.reshape(-1, 3)[:, 2]
    top = Xe & np.isclose(p.coords[:, 2], 1.0)
    assert np.allclose(uz[Xe & ~top], -0.2 * p.t_final, atol=1e-14)
    assert np.allclose(uz[top], -0.2 * p.t_final + 0.01, atol=1e-14)
