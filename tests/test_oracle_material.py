"""Pins for the oracle's Neo-Hookean restatement
(src/material/utilitiesmaterialHyperelastic.cpp:45-140, 186-295)."""
import numpy as np
import pytest


def test_stress_free_at_identity(oracle):
    s, C = oracle.nh_stress_tangent(np.eye(3), 1.0, 0.1)
    assert np.abs(s).max() < 1e-15
    assert np.allclose(C, C.T, atol=1e-14)


def test_uniaxial_closed_form(oracle):
    # F = diag(l, 1, 1): sigma = mu J^{-5/3} (b - tr(b)/3 I) + K (J - 1) I
    mu, K, lam = 1.3, 7.0, 1.2
    s, _ = oracle.nh_stress_tangent(np.diag([lam, 1.0, 1.0]), mu, 1.0 / K)
    J = lam
    b = np.diag([lam * lam, 1.0, 1.0])
    ref = mu * J ** (-5.0 / 3.0) * (b - np.trace(b) / 3.0 * np.eye(3)) + K * (J - 1.0) * np.eye(3)
    # stre is the column-major 9-vector of sigma
    assert np.allclose(s, ref.T.ravel(), rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("utype", [1, 2, 3, 4, 5, 7, 8])
def test_volumetric_second_derivative_is_derivative_of_first(oracle, utype):
    K, h = 3.0, 1e-6
    for J in (0.8, 1.0, 1.3):
        fd = (oracle.lib().orc_vol_dU(utype, K, J + h) - oracle.lib().orc_vol_dU(utype, K, J - h)) / (2 * h)
        assert abs(fd - oracle.lib().orc_vol_d2U(utype, K, J)) < 1e-6 * max(1.0, abs(fd))


def test_tangent_major_symmetry_and_structure(oracle):
    rng = np.random.default_rng(3)
    F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
    mu, Kinv = 0.7, 0.05
    s, C = oracle.nh_stress_tangent(F, mu, Kinv)
    assert np.allclose(C, C.T, rtol=1e-13, atol=1e-13)
    # closed form of every entry with the 9-index (i, j) = (q % 3, q // 3)
    J = np.linalg.det(F)
    b = F @ F.T
    Ib = np.trace(b)
    K = 1.0 / Kinv
    dU, d2U = K * (J - 1.0), K
    a = mu * J ** (-5.0 / 3.0)
    d = np.eye(3)
    ref = np.zeros((9, 9))
    for p in range(9):
        i, j = p % 3, p // 3
        for q in range(9):
            k, l = q % 3, q // 3
            ref[p, q] = (a * Ib / 3.0 * d[i, l] * d[j, k] - 2.0 / 3.0 * a * (b[i, j] * d[k, l] + d[i, j] * b[k, l])
                         + 2.0 / 9.0 * a * Ib * d[i, j] * d[k, l] + a * b[j, l] * d[i, k]
                         + (J * d2U + dU) * d[i, j] * d[k, l] - dU * d[i, l] * d[j, k] - dU * d[j, l] * d[i, k])
    assert np.allclose(C, ref, rtol=1e-13, atol=1e-13)
