"""Nonzero prescribed displacements in the oracle (setBoundaryConditions + the applyDirichletBCs
lift, ElementBase.cpp:567-594, femSolidmechanics2.cpp:1137-1145), pinned by a closed form: a block
on three symmetry planes stretched by a prescribed end displacement deforms homogeneously, with the
lateral stretch of the uniaxial Neo-Hookean state (sigma_22 = sigma_33 = 0)."""
import numpy as np
import pytest
from scipy.optimize import brentq

from mphyfem_b200 import meshgen


def stretch_block(nx=4, ny=2, nz=2, lx=2.0, eps=0.1, mu=1.0, kappa=10.0, split=False):
    """Symmetry planes x=0 (u_x), y=0 (u_y), z=0 (u_z); u_x = eps * lx * t on x = lx; no load."""
    p = meshgen.tet10_kuhn(nx, ny, nz, lx=lx, jitter=0.0, mu=mu, kappa=kappa, traction=(0, 0, 0)) if split \
        else meshgen.hex8_cantilever(nx, ny, nz, lx=lx, mu=mu, kappa=kappa, traction=(0, 0, 0))
    X = p.coords
    fx = np.zeros((p.n_node, 3), np.uint8)
    fx[np.isclose(X[:, 0], 0.0), 0] = 1
    fx[np.isclose(X[:, 1], 0.0), 1] = 1
    fx[np.isclose(X[:, 2], 0.0), 2] = 1
    end = np.isclose(X[:, 0], lx)
    fx[end, 0] = 1
    ramp = np.zeros((p.n_node, 3))
    ramp[end, 0] = eps * lx
    p.fixed = fx.ravel()
    p.presc_ramp = ramp.ravel()
    p.fnodal = np.zeros(p.n_dof)
    return p


def uniaxial_lateral_stretch(l1, mu, kappa):
    """lambda_2 with sigma_22 = mu J^-5/3 (l2^2 - Ib/3) + kappa (J - 1) = 0, J = l1 l2^2 (Utype 3)."""
    def s22(l2):
        J = l1 * l2 * l2
        return mu * J ** (-5.0 / 3.0) * (l2 * l2 - (l1 * l1 + 2 * l2 * l2) / 3.0) + kappa * (J - 1.0)
    return brentq(s22, 0.5, 1.5, xtol=1e-15)


@pytest.mark.parametrize("split", [False, True], ids=["hex8", "tet10"])
def test_prescribed_stretch_is_homogeneous(oracle, split):
    p = stretch_block(split=split)
    oracle.set_consistent_tangent(True)
    try:
        u, hist = oracle.OracleProblem(p).newton(tol_rel=1e-12, tol_abs=1e-14, cg_rtol=1e-13, max_newton=15)
    finally:
        oracle.set_consistent_tangent(False)
    steps = np.unique(hist[:, 0])
    assert len(steps) == p.max_steps
    l1 = 1.1
    l2 = uniaxial_lateral_stretch(l1, 1.0, 10.0)
    X = p.coords
    exact = np.stack([(l1 - 1) * X[:, 0], (l2 - 1) * X[:, 1], (l2 - 1) * X[:, 2]], axis=1)
    assert np.abs(u.reshape(-1, 3) - exact).max() <= 1e-9
    # the first iteration of every step carries the lifted increment: a nonzero residual
    first = hist[hist[:, 1] == 1]
    assert np.all(first[:, 2] > 0)
