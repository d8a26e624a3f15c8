"""Pins for the oracle's element restatement (src/femSolidmechanics/Elem_Solid_3D_Disp.cpp:196-373).

The reference's spatial tangent omits the volumetric geometric term U'(J) d_ik d_jl
(utilitiesmaterialHyperelastic.cpp:283-288 keeps the "without stress terms" volumetric line),
so K_ref = -dR/du - sum_gp dvol U'(J) (grad N_I . grad N_J) I_3. The central-difference
check (the 6-point stencil documented at src/utilities/ElementBase.cpp:1519-1524) verifies R,
K and that analytic correction at once."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

MU, KINV = 1.0, 0.1


def _ref_elem(npe, rng, jitter=0.05):
    if npe == 8:
        X = meshgen.HEX8_CORNERS.astype(float) * np.array([0.5, 0.3, 0.4])
    else:
        v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]]) * 0.6
        mids = [(0, 1), (1, 2), (0, 2), (0, 3), (2, 3), (1, 3)]
        X = np.vstack([v, [(v[a] + v[b]) / 2 for a, b in mids]])
    X = X + 0.02 * rng.standard_normal(X.shape)
    u = jitter * rng.standard_normal(X.shape)
    return X, u


def _vol_correction(oracle, npe, X, u):
    _, w, _, dN = oracle.gauss_rule(npe)
    corr = np.zeros((3 * npe, 3 * npe))
    x = X + u
    for q in range(len(w)):
        g0 = np.linalg.solve(dN[q] @ X, dN[q])
        F = np.eye(3) + u.T @ g0.T
        J = np.linalg.det(F)
        G = dN[q] @ x
        g = np.linalg.solve(G, dN[q])
        dvol = w[q] * np.linalg.det(G)
        corr += np.kron(dvol * (1.0 / KINV) * (J - 1.0) * (g.T @ g), np.eye(3))
    return corr


@pytest.mark.parametrize("npe", [8, 10])
def test_fd_tangent_with_reference_volumetric_term(oracle, npe):
    rng = np.random.default_rng(npe)
    X, u = _ref_elem(npe, rng)
    K, R, bad = oracle.elem_stiffness_residual(X, u, MU, KINV)
    assert bad == 0
    h = 1e-6
    Kfd = np.zeros_like(K)
    for j in range(3 * npe):
        up, um = u.ravel().copy(), u.ravel().copy()
        up[j] += h
        um[j] -= h
        Rp = oracle.elem_stiffness_residual(X, up.reshape(u.shape), MU, KINV)[1]
        Rm = oracle.elem_stiffness_residual(X, um.reshape(u.shape), MU, KINV)[1]
        Kfd[:, j] = -(Rp - Rm) / (2 * h)
    scale = np.abs(K).max()
    assert np.abs(K + _vol_correction(oracle, npe, X, u) - Kfd).max() < 1e-7 * scale
    # and the consistent-tangent switch closes the gap by itself
    oracle.set_consistent_tangent(True)
    try:
        Kc = oracle.elem_stiffness_residual(X, u, MU, KINV)[0]
    finally:
        oracle.set_consistent_tangent(False)
    assert np.abs(Kc - Kfd).max() < 1e-7 * scale


@pytest.mark.parametrize("npe", [8, 10])
def test_symmetry_zero_state_and_equilibrium(oracle, npe):
    rng = np.random.default_rng(10 + npe)
    X, u = _ref_elem(npe, rng)
    K, R, _ = oracle.elem_stiffness_residual(X, u, MU, KINV)
    assert np.abs(K - K.T).max() < 1e-13 * np.abs(K).max()
    # internal forces are self-equilibrated: sum over nodes vanishes
    assert np.abs(R.reshape(-1, 3).sum(axis=0)).max() < 1e-13 * np.abs(R).max()
    K0, R0, _ = oracle.elem_stiffness_residual(X, np.zeros_like(u), MU, KINV)
    assert np.abs(R0).max() == 0.0
    # at u = 0 the stiffness annihilates rigid translations
    for d in range(3):
        t = np.zeros_like(u)
        t[:, d] = 1.0
        assert np.abs(K0 @ t.ravel()).max() < 1e-12 * np.abs(K0).max()


@pytest.mark.parametrize("npe", [8, 10])
def test_rigid_rotation_is_stress_free(oracle, npe):
    rng = np.random.default_rng(20 + npe)
    X, _ = _ref_elem(npe, rng)
    th = 0.7
    Q = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    u = X @ Q.T - X
    _, R, bad = oracle.elem_stiffness_residual(X, u, MU, KINV)
    assert bad == 0
    assert np.abs(R).max() < 1e-13


def test_negative_jacobian_flag(oracle):
    X = meshgen.HEX8_CORNERS.astype(float)
    u = np.zeros_like(X)
    u[:, 0] = -2.5 * X[:, 0]  # invert the element along x
    _, _, bad = oracle.elem_stiffness_residual(X, u, MU, KINV)
    assert bad == 1


def test_homogeneous_patch(oracle):
    """Affine displacement on a small mesh: interior nodal residuals vanish."""
    p = meshgen.hex8_cantilever(3, 3, 3, lx=1.0)
    op = oracle.OracleProblem(p)
    A = np.array([[0.02, 0.01, 0.0], [0.0, -0.01, 0.03], [0.01, 0.0, 0.02]])
    u = (p.coords @ A.T).ravel()
    _, _, reac, bad = op.assemble(u)
    assert bad == -1
    c = p.coords
    inner = np.all((c > 1e-9) & (c < np.array([1.0, 1.0, 1.0]) - 1e-9), axis=1)
    r = reac.reshape(-1, 3)
    assert np.abs(r[inner]).max() < 1e-13 * np.abs(r).max()
