"""Pins for the oracle's Mooney-Rivlin, Gent and Arruda-Boyce restatements
(src/material/utilitiesmaterialHyperelastic.cpp:300-677, compressible branch).

Each model is checked three ways:
  * against an independent numpy transcription of the reference's formulas (every stress and
    tangent entry, both tangent modes);
  * finite differences: the Kirchhoff stress tau = J sigma under F -> (I + e E_kl) F gives
    J C_ijkl = d tau_ij / d L_kl - tau_il d_jk (the convention of the element contraction); the
    element tangent against the central difference of the element residual;
  * reductions: stress-free at F = I, Mooney-Rivlin with c2 = 0 equals Neo-Hookean with mu = 2 c1,
    zero residual at u = 0 and invariance under a rigid rotation.
"""
import numpy as np
import pytest

MR, GENT, AB = 1, 2, 3
PARAMS = {MR: [0.4, 0.15], GENT: [0.7, 12.0], AB: [0.7, 5.0]}


def _d(i, j):
    return 1.0 if i == j else 0.0


def _kin(F, Kinv, utype, oracle):
    b = F @ F.T
    J = np.linalg.det(F)
    K = 1.0 / Kinv
    return b, b @ b, J, np.trace(b), oracle.lib().orc_vol_dU(utype, K, J), oracle.lib().orc_vol_d2U(utype, K, J)


def numpy_model(model, data, F, Kinv, utype, oracle, consistent=False):
    """The reference's formulas transcribed term by term (column-major stress, map_tensor4)."""
    b, b2, J, Ib, dU, d2U = _kin(F, Kinv, utype, oracle)
    I3 = np.eye(3)
    bd = b - Ib / 3.0 * I3
    C = np.zeros((9, 9))
    if model == MR:
        c1, c2 = data
        Jm5d3, Jm7d3 = J ** (-5.0 / 3.0), J ** (-5.0 / 3.0)  # r7d3 = 5/3 as written
        I1, I2 = Ib, 0.5 * (Ib * Ib - np.trace(b2))
        sig = (2 * c1 * Jm5d3 + 2 * c2 * Jm7d3 * I1) * b - 2 * c2 * Jm7d3 * b2 + \
            (-c1 * 2 / 3 * Jm5d3 * I1 - c2 * 4 / 3 * Jm7d3 * I2 + dU) * I3
        f1, f2, f3 = 2 * c1 * Jm5d3, 2 * c2 * Jm7d3, 4 / 3 * c2 * Jm7d3
    elif model == GENT:
        mu, Im = data
        gf = 1.0 / (1.0 - (J ** (-2 / 3) * Ib - 3.0) / Im)
        s1 = mu * J ** (-5 / 3) * gf
        sig = s1 * b + (-s1 / 3 * Ib + dU) * I3
        f1, f2, f3 = -2 / 3 * mu * J ** (-5 / 3) * gf, 2 * mu * J ** (-7 / 3) * gf * gf / Im, mu * J ** (-5 / 3) * gf
    else:
        mu, N = data
        c = [mu / 2, mu / 20 / N, mu * 11 / 1050 / N ** 2, mu * 19 / 7000 / N ** 3, mu * 519 / 673750 / N ** 4]
        x = J ** (-2 / 3) * Ib
        a1 = c[0] + 2 * c[1] * x + 3 * c[2] * x ** 2 + 4 * c[3] * x ** 3 + 5 * c[4] * x ** 4
        a2 = 2 * c[1] + 6 * c[2] * x + 12 * c[3] * x ** 2 + 20 * c[4] * x ** 3
        s1 = 2 * a1 * J ** (-5 / 3)
        sig = s1 * b + (-s1 / 3 * Ib + dU) * I3
        f1, f2 = 4 * J ** (-7 / 3) * a2, -4 / 3 * a1 * J ** (-5 / 3)
        f3, f4 = 2 / 3 * a1 * J ** (-5 / 3) * Ib, 4 / 9 * a1 * J ** (-5 / 3) * Ib
    f7, f8 = J * d2U + dU, -dU
    for p in range(9):
        i, j = p % 3, p // 3
        for q in range(9):
            k, l = q % 3, q // 3
            dij, dik, dil, djk, djl, dkl = _d(i, j), _d(i, k), _d(i, l), _d(j, k), _d(j, l), _d(k, l)
            if model == MR:
                v = f1 * (dik * b[j, l] + Ib / 3 * dil * djk + 2 / 9 * Ib * dij * dkl - 2 / 3 * b[i, j] * dkl
                          - 2 / 3 * b[k, l] * dij)
                v += f2 * (2 * b[i, j] * b[k, l] + Ib * dik * b[j, l] - b[i, k] * b[j, l] - b[i, l] * b[k, j]
                           - dik * b2[j, l])
                v += f3 * (I2 * dil * djk + 4 / 3 * I2 * dkl * dij + 2 * dij * b2[k, l] + 2 * dkl * b2[i, j]
                           - 2 * Ib * dkl * b[i, j] - 2 * Ib * dij * b[k, l])
            elif model == GENT:
                v = f1 * bd[i, j] * dkl + f2 * bd[i, j] * bd[k, l] + \
                    f3 * (dik * b[j, l] - 2 / 3 * b[k, l] * dij + Ib / 3 * dil * djk)
            else:
                v = f1 * bd[i, j] * bd[k, l] + f2 * (b[i, j] * dkl + b[k, l] * dij) + f3 * (dik * djl + dil * djk) \
                    + f4 * dij * dkl
                if consistent:
                    v += 2 * a1 * J ** (-5 / 3) * dik * (b[j, l] - Ib / 3 * djl)
            C[p, q] = v + f7 * dij * dkl + f8 * dil * djk
    return sig.T.ravel(), C


@pytest.fixture
def consistent(oracle):
    def set_(on):
        oracle.set_consistent_tangent(on)
    yield set_
    oracle.set_consistent_tangent(False)


def _F(seed, amp=0.15):
    return np.eye(3) + amp * np.random.default_rng(seed).standard_normal((3, 3))


@pytest.mark.parametrize("model", [MR, GENT, AB])
@pytest.mark.parametrize("utype", [3, 1, 5])
@pytest.mark.parametrize("cons", [False, True])
def test_matches_numpy_transcription(oracle, consistent, model, utype, cons):
    consistent(cons)
    for seed in range(4):
        F = _F(seed)
        s, C = oracle.material_stress_tangent(model, PARAMS[model], F, 0.05, utype)
        sr, Cr = numpy_model(model, PARAMS[model], F, 0.05, utype, oracle, consistent=cons)
        assert np.allclose(s, sr, rtol=1e-12, atol=1e-13)
        assert np.allclose(C, Cr, rtol=1e-12, atol=1e-12)
        assert np.allclose(C, C.T, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("model", [MR, GENT, AB])
def test_stress_free_at_identity(oracle, model):
    s, _ = oracle.material_stress_tangent(model, PARAMS[model], np.eye(3), 0.05)
    assert np.abs(s).max() < 1e-14


def _fd_tangent(oracle, model, data, F, Kinv):
    def tau(Fx):
        s, _ = oracle.material_stress_tangent(model, data, Fx, Kinv)
        return np.linalg.det(Fx) * s.reshape(3, 3).T
    J = np.linalg.det(F)
    sig = tau(F) / J
    h, out = 1e-6, np.zeros((9, 9))
    for q in range(9):
        k, l = q % 3, q // 3
        E = np.zeros((3, 3))
        E[k, l] = 1.0
        d = (tau((np.eye(3) + h * E) @ F) - tau((np.eye(3) - h * E) @ F)) / (2 * h) / J
        for p in range(9):
            i, j = p % 3, p // 3
            out[p, q] = d[i, j] - sig[i, l] * _d(j, k)
    return out, sig


@pytest.mark.parametrize("model,cons", [(GENT, False), (GENT, True), (AB, True)])
def test_consistent_tangent_is_stress_derivative(oracle, consistent, model, cons):
    consistent(cons)
    F = _F(11)
    _, C = oracle.material_stress_tangent(model, PARAMS[model], F, 0.05)
    Cfd, _ = _fd_tangent(oracle, model, PARAMS[model], F, 0.05)
    assert np.abs(C - Cfd).max() <= 1e-8 * np.abs(C).max()


def test_arruda_boyce_reference_tangent_is_the_symmetrised_form(oracle):
    # the written tangent misses 2 a1 J^-5/3 (d_ik b_jl - Ib/3 d_ik d_jl) of the exact derivative
    F = _F(12)
    mu, N = PARAMS[AB]
    _, C = oracle.material_stress_tangent(AB, PARAMS[AB], F, 0.05)
    Cfd, _ = _fd_tangent(oracle, AB, PARAMS[AB], F, 0.05)
    b, J, Ib = F @ F.T, np.linalg.det(F), np.trace(F @ F.T)
    x = J ** (-2 / 3) * Ib
    c = [mu / 2, mu / 20 / N, mu * 11 / 1050 / N ** 2, mu * 19 / 7000 / N ** 3, mu * 519 / 673750 / N ** 4]
    a1 = sum((n + 1) * c[n] * x ** n for n in range(5))
    D = np.array([[2 * a1 * J ** (-5 / 3) * _d(p % 3, q % 3) * (b[p // 3, q // 3] - Ib / 3 * _d(p // 3, q // 3))
                   for q in range(9)] for p in range(9)])
    assert np.abs(C - Cfd).max() > 1e-4 * np.abs(C).max()
    assert np.abs(C + D - Cfd).max() <= 1e-8 * np.abs(C).max()


def test_mooney_rivlin_exponent_quirk(oracle, consistent):
    # r7d3 = 5/3 (utilitiesmaterialHyperelastic.cpp:303): the c2 stress is J^{2/3} times an energy's
    # stress, so the exact derivative is the written tangent plus (2/3) sigma_c2 (x) I. Both modes
    # keep the written (symmetric) tangent.
    c1, c2 = PARAMS[MR]
    F = _F(13)
    for cons in (False, True):
        consistent(cons)
        _, C = oracle.material_stress_tangent(MR, PARAMS[MR], F, 0.05)
        Cfd, _ = _fd_tangent(oracle, MR, PARAMS[MR], F, 0.05)
        b, J = F @ F.T, np.linalg.det(F)
        I1, I2 = np.trace(b), 0.5 * (np.trace(b) ** 2 - np.trace(b @ b))
        g = J ** (-5 / 3)
        sc2 = 2 * c2 * g * I1 * b - 2 * c2 * g * b @ b - 4 / 3 * c2 * g * I2 * np.eye(3)
        D = np.array([[2 / 3 * sc2[p % 3, p // 3] * _d(q % 3, q // 3) for q in range(9)] for p in range(9)])
        assert np.abs(C + D - Cfd).max() <= 1e-8 * np.abs(C).max()
        assert np.allclose(C, C.T, rtol=1e-12, atol=1e-12)


def _hex(seed):
    rng = np.random.default_rng(seed)
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float) * 0.5
    X += 0.03 * rng.standard_normal(X.shape)
    return X, 0.08 * rng.standard_normal(X.shape)


def _tet10(seed):
    rng = np.random.default_rng(seed)
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    edges = [(0, 1), (1, 2), (0, 2), (0, 3), (2, 3), (1, 3)]
    X = np.vstack([V] + [0.5 * (V[a] + V[b]) for a, b in edges]) + 0.02 * rng.standard_normal((10, 3))
    return X, 0.05 * rng.standard_normal((10, 3))


@pytest.mark.parametrize("mk", [_hex, _tet10])
@pytest.mark.parametrize("model,cons", [(GENT, False), (AB, True), (MR, False)])
def test_element_tangent_against_finite_differences(oracle, consistent, mk, model, cons):
    consistent(cons)
    X, u = mk(5)
    data = PARAMS[model] if model != MR else [0.4, 0.0]  # c2 = 0: no exponent quirk
    K, R, bad = oracle.elem_stiffness_residual_mat(X, u, model, data, 0.05)
    assert bad == 0
    n = u.size
    Kfd = np.zeros_like(K)
    h = 1e-6
    for j in range(n):
        up, um = u.ravel().copy(), u.ravel().copy()
        up[j] += h
        um[j] -= h
        _, Rp, _ = oracle.elem_stiffness_residual_mat(X, up.reshape(u.shape), model, data, 0.05)
        _, Rm, _ = oracle.elem_stiffness_residual_mat(X, um.reshape(u.shape), model, data, 0.05)
        Kfd[:, j] = -(Rp - Rm) / (2 * h)
    assert np.abs(K - Kfd).max() <= 1e-7 * np.abs(K).max()


def test_mooney_rivlin_without_c2_is_neo_hookean(oracle, consistent):
    consistent(True)
    X, u = _hex(7)
    K1, R1, _ = oracle.elem_stiffness_residual_mat(X, u, MR, [0.35, 0.0], 0.05)
    K0, R0, _ = oracle.elem_stiffness_residual(X, u, 0.7, 0.05)
    assert np.abs(K1 - K0).max() <= 1e-13 * np.abs(K0).max()
    assert np.abs(R1 - R0).max() <= 1e-13 * np.abs(R0).max()


@pytest.mark.parametrize("model", [MR, GENT, AB])
def test_zero_residual_and_rotation_invariance(oracle, model):
    X, u = _hex(9)
    _, R, _ = oracle.elem_stiffness_residual_mat(X, np.zeros_like(X), model, PARAMS[model], 0.05)
    assert np.abs(R).max() < 1e-14
    # rotate the deformed configuration: residual forces rotate with it
    th = 0.7
    Q = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    x = X + u
    ur = x @ Q.T - X
    _, R0, _ = oracle.elem_stiffness_residual_mat(X, u, model, PARAMS[model], 0.05)
    _, Rr, _ = oracle.elem_stiffness_residual_mat(X, ur, model, PARAMS[model], 0.05)
    assert np.abs(Rr.reshape(-1, 3) - R0.reshape(-1, 3) @ Q.T).max() <= 1e-12 * np.abs(R0).max()


def test_problem_material_models(oracle):
    from mphyfem_b200 import meshgen
    p = meshgen.hex8_cantilever(4, 2, 2)
    n = p.n_elem
    p.mat_id = (np.arange(n) % 3).astype(np.int32)
    p.mats = np.array([[0.4, 0.05, 3.0], [0.7, 0.05, 3.0], [0.7, 0.05, 3.0]])
    p.mat_model = np.array([MR, GENT, AB], np.int32)
    p.mat_data = np.array([[0.4, 0.15, 0, 0], [0.7, 12.0, 0, 0], [0.7, 5.0, 0, 0]])
    u = 0.01 * np.random.default_rng(2).standard_normal(p.n_dof)
    Ke, Re, bad = oracle.OracleProblem(p).elements(u)
    assert bad == -1
    for e in (0, 1, 2, 7):
        m = int(p.mat_id[e])
        X = p.coords[p.conn[e]]
        ue = u.reshape(-1, 3)[p.conn[e]]
        K, R, _ = oracle.elem_stiffness_residual_mat(X, ue, int(p.mat_model[m]), p.mat_data[m], 0.05)
        assert np.array_equal(K, Ke[e]) and np.array_equal(R, Re[e])
