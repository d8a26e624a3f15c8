"""Pins for the oracle's mixed u-p element (tet10 displacement, linear vertex pressure;
ElementBase2.cpp:278-553 with Elem_Solid_3D_Mixed1) and its two-field Newton restatement:
finite-difference tangents of all four blocks, Kpu = Kup^T, the uniaxial patch test (mixed =
displacement formulation = the homogeneous solution, with a uniform pressure p = U'(J)), and
quadratic Newton convergence.
"""
import numpy as np
import pytest

from mphyfem_b200 import meshgen
from mphyfem_b200 import reference_io as rio


@pytest.fixture
def consistent(oracle):
    oracle.set_consistent_tangent(True)
    yield
    oracle.set_consistent_tangent(False)


def _tet10(seed):
    rng = np.random.default_rng(seed)
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    edges = [(0, 1), (1, 2), (0, 2), (0, 3), (2, 3), (1, 3)]
    X = np.vstack([V] + [0.5 * (V[a] + V[b]) for a, b in edges]) + 0.02 * rng.standard_normal((10, 3))
    return X, 0.05 * rng.standard_normal((10, 3)), 0.03 * rng.standard_normal((10, 3)), 0.3 * rng.standard_normal(4)


@pytest.mark.parametrize("model,data", [(0, [0.7]), (1, [0.35, 0.0]), (2, [0.7, 12.0]), (3, [0.7, 5.0])],
                         ids=["nh", "mr_c2_0", "gent", "ab"])
@pytest.mark.parametrize("utype", [3, 1])
def test_element_blocks_against_finite_differences(oracle, consistent, model, data, utype):
    X, u, up, pn = _tet10(5)
    Kuu, Kup, Kpu, Kpp, FU, FP, bad = oracle.elem_mixed(X, u, up, pn, model, data, 0.05, utype)
    assert bad == 0
    assert np.allclose(Kpu, Kup.T, rtol=1e-14, atol=1e-16)
    h = 1e-6
    KuuF, KpuF = np.zeros_like(Kuu), np.zeros_like(Kpu)
    for j in range(30):
        a, b = u.ravel().copy(), u.ravel().copy()
        a[j] += h
        b[j] -= h
        r1 = oracle.elem_mixed(X, a.reshape(10, 3), up, pn, model, data, 0.05, utype)
        r2 = oracle.elem_mixed(X, b.reshape(10, 3), up, pn, model, data, 0.05, utype)
        KuuF[:, j] = -(r1[4] - r2[4]) / (2 * h)
        KpuF[:, j] = -(r1[5] - r2[5]) / (2 * h)
    KupF, KppF = np.zeros_like(Kup), np.zeros_like(Kpp)
    for j in range(4):
        a, b = pn.copy(), pn.copy()
        a[j] += h
        b[j] -= h
        r1 = oracle.elem_mixed(X, u, up, a, model, data, 0.05, utype)
        r2 = oracle.elem_mixed(X, u, up, b, model, data, 0.05, utype)
        KupF[:, j] = -(r1[4] - r2[4]) / (2 * h)
        KppF[:, j] = -(r1[5] - r2[5]) / (2 * h)
    for K, KF in ((Kuu, KuuF), (Kup, KupF), (Kpu, KpuF), (Kpp, KppF)):
        assert np.abs(K - KF).max() <= 1e-7 * np.abs(K).max()


def test_arruda_boyce_written_pressure_term(oracle):
    # the reference's mixed Arruda-Boyce tangent carries -p d_jl d_ik (:661-664); the consistent
    # tangent does not
    F = np.eye(3) + 0.1 * np.random.default_rng(3).standard_normal((3, 3))
    _, C0 = oracle.material_stress_tangent_mixed(3, [0.7, 5.0], F, 0.05, 0.4)
    oracle.set_consistent_tangent(True)
    try:
        _, C1 = oracle.material_stress_tangent_mixed(3, [0.7, 5.0], F, 0.05, 0.4)
        _, Cd = oracle.material_stress_tangent(3, [0.7, 5.0], F, 0.05)
    finally:
        oracle.set_consistent_tangent(False)
    d = np.eye(3)
    D = np.array([[d[p // 3, q // 3] * d[p % 3, q % 3] for q in range(9)] for p in range(9)])  # d_jl d_ik
    dev_fix = Cd - oracle.material_stress_tangent(3, [0.7, 5.0], F, 0.05)[1]
    assert np.allclose(C1 - C0, 0.4 * D + dev_fix, rtol=1e-12, atol=1e-12)


def _patch(model=0, data=(1.0,), kappa=20.0):
    p = meshgen.tet10_kuhn(3, 2, 2, lx=2.0, traction=(0.0, 0.0, 0.0))
    X = p.coords
    fx = np.zeros((p.n_node, 3), np.uint8)
    fx[np.isclose(X[:, 0], 0.0), 0] = 1
    fx[np.isclose(X[:, 1], 0.0), 1] = 1
    fx[np.isclose(X[:, 2], 0.0), 2] = 1
    p.fixed = fx.ravel()
    faces = rio.boundary_faces(p, lambda Y: np.isclose(Y[:, 0], 2.0))
    # a dead load along x (s1 on dx/dxi1 is not used): the consistent nodal forces of 0.05 e_x
    F = np.zeros((p.n_node, 3))
    for fc in faces:
        fc = np.asarray(fc)
        a = 0.5 * np.linalg.norm(np.cross(X[fc[1]] - X[fc[0]], X[fc[2]] - X[fc[0]]))
        F[fc[3:], 0] += 0.05 * a / 3.0
    p.fnodal = F.ravel()
    p.mats = np.array([[data[0], 1.0 / kappa, 3.0]])
    if model:
        p.mat_model = np.array([model], np.int32)
        p.mat_data = np.array([list(data) + [0.0] * (4 - len(data))])
    p.dt, p.t_final, p.max_steps = 0.25, 1.0, 4
    p.newton_rtol = 1e-10
    return p


@pytest.mark.parametrize("model,data", [(0, (1.0,)), (2, (1.0, 10.0))], ids=["nh", "gent"])
def test_uniaxial_patch(oracle, consistent, model, data):
    from oracle.mixed_ref import MixedProblem
    p = _patch(model, data)
    u, pres, hist = MixedProblem(p).newton(max_newton=15)
    ud, _ = oracle.OracleProblem(p).newton(cg_rtol=1e-13, max_newton=15)
    assert np.linalg.norm(u - ud) <= 1e-9 * np.linalg.norm(ud)
    # homogeneous: u = (a x, b y, b z); uniform pressure U'(J) = K (J - 1)
    X = p.coords
    U = u.reshape(-1, 3)
    a = U[:, 0] @ X[:, 0] / (X[:, 0] @ X[:, 0])
    bb = U[:, 1] @ X[:, 1] / (X[:, 1] @ X[:, 1])
    assert np.abs(U[:, 0] - a * X[:, 0]).max() <= 1e-10 * abs(a)
    assert np.abs(U[:, 1] - bb * X[:, 1]).max() <= 1e-10 * abs(bb)
    J = (1 + a) * (1 + bb) ** 2
    vert = np.unique(p.conn[:, :4])
    assert np.allclose(pres[vert], 20.0 * (J - 1.0), rtol=1e-9)
    # quadratic convergence: every step ends within 5 iterations
    assert max(np.bincount(hist[:, 0].astype(int))[1:]) <= 5


@pytest.mark.parametrize("npe", [8, 10])
@pytest.mark.parametrize("model,data", [(0, [0.7]), (2, [0.7, 12.0])], ids=["nh", "gent"])
def test_constant_pressure_element_condensation(oracle, consistent, npe, model, data):
    """Elem_Solid_3D_Mixed0: FU and FP are linear in the element pressure, so the condensed residual
    F = FU - Kup FP / Kpp is FU at the pressure p* = p + FP / Kpp that zeroes FP, for any p; at p*
    the condensed tangent K = Kuu - Kup Kpu / Kpp is minus its derivative (finite differences)."""
    rng = np.random.default_rng(3)
    if npe == 10:
        X, u, up, _ = _tet10(7)
    else:
        X = meshgen.hex8_cantilever(1, 1, 1, lx=1.0).coords[meshgen.hex8_cantilever(1, 1, 1, lx=1.0).conn[0]]
        X = X + 0.02 * rng.standard_normal(X.shape)
        u, up = 0.05 * rng.standard_normal((8, 3)), 0.03 * rng.standard_normal((8, 3))
    ns = 3 * npe
    K0, F0, kup, kpp, fp, bad = oracle.elem_mixed0(X, u, up, 0.1, model, data, 0.05, 3)
    assert bad == 0 and kpp < 0
    pstar = 0.1 + fp / kpp
    K, F, _, _, fp2, _ = oracle.elem_mixed0(X, u, up, pstar, model, data, 0.05, 3)
    assert abs(fp2) <= 1e-12 * max(abs(fp), 1e-300) + 1e-15
    assert np.abs(F - F0).max() <= 1e-12 * np.abs(F0).max()  # the condensed residual does not depend on p
    assert np.abs(K - K.T).max() <= 1e-12 * np.abs(K).max() or model != 0
    h = 1e-6
    KF = np.zeros((ns, ns))
    for j in range(ns):
        a, b = u.ravel().copy(), u.ravel().copy()
        a[j] += h
        b[j] -= h
        r1 = oracle.elem_mixed0(X, a.reshape(npe, 3), up, pstar, model, data, 0.05, 3)
        r2 = oracle.elem_mixed0(X, b.reshape(npe, 3), up, pstar, model, data, 0.05, 3)
        KF[:, j] = -(r1[1] - r2[1]) / (2 * h)
    assert np.abs(K - KF).max() <= 1e-7 * np.abs(K).max()


def _hex27(seed):
    """One distorted 27-node hex: the reference cube's 27 nodes, jittered."""
    rng = np.random.default_rng(seed)
    pos = np.array([-1.0, 1.0, 0.0])
    X = 0.5 * (1.0 + pos[meshgen.HEX27_IJK]) + 0.02 * rng.standard_normal((27, 3))
    return X, 0.05 * rng.standard_normal((27, 3)), 0.03 * rng.standard_normal((27, 3)), 0.3 * rng.standard_normal(8)


@pytest.mark.parametrize("model,data", [(0, [0.7]), (2, [0.7, 12.0])], ids=["nh", "gent"])
def test_hex27_p2p1_blocks_against_finite_differences(oracle, consistent, model, data):
    """The P2-P1 hex (Elem_Solid_3D_Mixed1 with 27 nodes, the 3x3x3 rule, trilinear corner
    pressure): all four blocks are the derivatives of the two residuals, and Kpu = Kup^T."""
    X, u, up, pn = _hex27(11)
    Kuu, Kup, Kpu, Kpp, FU, FP, bad = oracle.elem_mixed(X, u, up, pn, model, data, 0.05, 3)
    assert bad == 0 and Kuu.shape == (81, 81) and Kup.shape == (81, 8) and Kpp.shape == (8, 8)
    assert np.allclose(Kpu, Kup.T, rtol=1e-14, atol=1e-16)
    h = 1e-6
    KuuF, KpuF = np.zeros_like(Kuu), np.zeros_like(Kpu)
    for j in range(81):
        a, b = u.ravel().copy(), u.ravel().copy()
        a[j] += h
        b[j] -= h
        r1 = oracle.elem_mixed(X, a.reshape(27, 3), up, pn, model, data, 0.05, 3)
        r2 = oracle.elem_mixed(X, b.reshape(27, 3), up, pn, model, data, 0.05, 3)
        KuuF[:, j] = -(r1[4] - r2[4]) / (2 * h)
        KpuF[:, j] = -(r1[5] - r2[5]) / (2 * h)
    KupF, KppF = np.zeros_like(Kup), np.zeros_like(Kpp)
    for j in range(8):
        a, b = pn.copy(), pn.copy()
        a[j] += h
        b[j] -= h
        r1 = oracle.elem_mixed(X, u, up, a, model, data, 0.05, 3)
        r2 = oracle.elem_mixed(X, u, up, b, model, data, 0.05, 3)
        KupF[:, j] = -(r1[4] - r2[4]) / (2 * h)
        KppF[:, j] = -(r1[5] - r2[5]) / (2 * h)
    for K, KF in ((Kuu, KuuF), (Kup, KupF), (Kpu, KpuF), (Kpp, KppF)):
        assert np.abs(K - KF).max() <= 1e-7 * np.abs(K).max()


def test_hex27_shape_functions(oracle):
    """The 27 triquadratic functions at the 27 Gauss points (3x3x3, weights summing to the
    cube's volume 8): a partition of unity, derivatives summing to zero, and exact interpolation
    of triquadratic fields on the node positions."""
    xi, w, N, dN = oracle.gauss_rule(27)
    assert xi.shape == (27, 3) and abs(w.sum() - 8.0) <= 1e-13
    assert np.allclose(xi, np.array([-0.774596669241483, 0.774596669241483, 0.0])[meshgen.HEX27_IJK])
    assert np.allclose(N.sum(axis=1), 1.0, atol=1e-14)
    assert np.allclose(dN.sum(axis=2), 0.0, atol=1e-13)
    pos = np.array([-1.0, 1.0, 0.0])[meshgen.HEX27_IJK]
    f = pos[:, 0] ** 2 * pos[:, 1] * pos[:, 2] + pos[:, 1] ** 2
    assert np.allclose(N @ f, xi[:, 0] ** 2 * xi[:, 1] * xi[:, 2] + xi[:, 1] ** 2, atol=1e-14)
    assert np.allclose(dN[:, 0, :] @ f, 2 * xi[:, 0] * xi[:, 1] * xi[:, 2], atol=1e-13)


@pytest.mark.parametrize("model,data", [(0, (1.0,)), (2, (1.0, 10.0))], ids=["nh", "gent"])
def test_hex27_uniaxial_patch(oracle, consistent, model, data):
    """P2-P1 hexes under a dead end load along x with symmetry supports: the homogeneous state
    u = (a x, b y, b z) with the uniform pressure U'(J) = K (J - 1) at the corners, reached with
    quadratic Newton convergence."""
    from oracle.mixed_ref import MixedProblem
    p = meshgen.hex27_cantilever(3, 2, 2, lx=2.0, traction=(0.05, 0.0, 0.0))
    X = p.coords
    fx = np.zeros((p.n_node, 3), np.uint8)
    fx[np.isclose(X[:, 0], 0.0), 0] = 1
    fx[np.isclose(X[:, 1], 0.0), 1] = 1
    fx[np.isclose(X[:, 2], 0.0), 2] = 1
    p.fixed = fx.ravel()
    p.mats = np.array([[data[0], 1.0 / 20.0, 3.0]])
    if model:
        p.mat_model = np.array([model], np.int32)
        p.mat_data = np.array([list(data) + [0.0] * (4 - len(data))])
    p.dt, p.t_final, p.max_steps = 0.25, 1.0, 4
    p.newton_rtol = 1e-10
    u, pres, hist = MixedProblem(p).newton(max_newton=15)
    U = u.reshape(-1, 3)
    a = U[:, 0] @ X[:, 0] / (X[:, 0] @ X[:, 0])
    bb = U[:, 1] @ X[:, 1] / (X[:, 1] @ X[:, 1])
    assert a > 0.0 and bb < 0.0
    assert np.abs(U[:, 0] - a * X[:, 0]).max() <= 1e-10 * abs(a)
    assert np.abs(U[:, 1] - bb * X[:, 1]).max() <= 1e-10 * abs(bb)
    assert np.abs(U[:, 2] - bb * X[:, 2]).max() <= 1e-10 * abs(bb)
    J = (1 + a) * (1 + bb) ** 2
    corners = np.unique(p.conn[:, :8])
    assert np.allclose(pres[corners], 20.0 * (J - 1.0), rtol=1e-9)
    assert max(np.bincount(hist[:, 0].astype(int))[1:]) <= 5
