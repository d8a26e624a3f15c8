"""Pins for the oracle's arc-length restatement (femSolidmechanics2.cpp:855-1039,
SolverPetsc.cpp:671-757): the first step is a Newton solve at lambda = dt; every converged step
is in equilibrium at its own load factor (the state equals load control at that load factor);
failed attempts cut the arc length and retry; a first step that cannot converge is reported.
"""
import numpy as np
import pytest

from mphyfem_b200 import meshgen


@pytest.fixture
def consistent(oracle):
    oracle.set_consistent_tangent(True)
    yield
    oracle.set_consistent_tangent(False)


def _cantilever(dt=0.1, steps=6):
    p = meshgen.hex8_cantilever(8, 2, 2, traction=(0.0, 0.0, -0.05))
    p.dt, p.t_final, p.max_steps = dt, 2.0, steps
    return p


def _load_control(oracle, lam, n=8):
    q = _cantilever()
    q.t_final, q.dt, q.max_steps = lam, lam / n, 100
    u, _ = oracle.OracleProblem(q).newton(tol_abs=1e-11, tol_rel=0.0, cg_rtol=1e-12, max_newton=20)
    return u


def test_steps_are_equilibria(oracle, consistent):
    p = _cantilever()
    u, lam, hist = oracle.OracleProblem(p).arclength(tol_abs=1e-10, cg_rtol=1e-12, max_newton=10)
    assert len(lam) == 6 and lam[0] == p.dt
    assert np.all(np.diff(lam) > 0)
    # first step: a Newton solve at lambda = dt, the load factor does not move
    assert np.all(hist[hist[:, 0] == 1][:, 4] == p.dt)
    un = _load_control(oracle, lam[-1])
    assert np.linalg.norm(u - un) <= 1e-9 * np.linalg.norm(un)


def test_arc_length_is_constant_after_the_first_step(oracle, consistent):
    # Ds is set by the first step and capped there (doubling is bounded by Ds_max); with a
    # spherical constraint the load-displacement increments of steps 2..n have one length
    p = _cantilever(steps=5)
    op = oracle.OracleProblem(p)
    states, lams = [np.zeros(p.n_dof)], [0.0]
    for k in range(1, 6):
        q = _cantilever(steps=k)
        u, lam, _ = oracle.OracleProblem(q).arclength(tol_abs=1e-11, cg_rtol=1e-12, max_newton=10)
        states.append(u)
        lams.append(lam[-1])
    FtF = float(p.fnodal @ p.fnodal)
    ds = [np.sqrt(np.sum((states[k] - states[k - 1]) ** 2) + (lams[k] - lams[k - 1]) ** 2 * FtF)
          for k in range(1, 6)]
    ds1 = np.sqrt(np.sum(states[1] ** 2) + lams[1] ** 2 * FtF)
    assert ds[0] == pytest.approx(ds1, rel=1e-12)
    assert np.allclose(ds[1:], ds1, rtol=1e-6)
    del op


def test_failed_attempt_cuts_the_arc_length(oracle, consistent):
    # from an initial state off equilibrium, the first step's arc length is long; the second
    # step's first attempt folds an element, the retry at half the arc length converges, and two
    # converged steps in a row double it again (capped at the first step's)
    p = _cantilever(steps=5)
    x = p.coords
    u0 = np.zeros_like(x)
    s = x[:, 0] / x[:, 0].max()
    u0[:, 2] = 0.3 * s * s
    u, lam, hist = oracle.OracleProblem(p).arclength(tol_abs=1e-9, cg_rtol=1e-12, max_newton=12, disp=u0.ravel())
    attempts = [int(((hist[:, 0] == k) & (hist[:, 1] == 1)).sum()) for k in range(1, 6)]
    assert attempts == [1, 2, 1, 1, 1]
    assert len(lam) == 5 and np.all(np.diff(lam) > 0)
    assert (lam[3] - lam[2]) > 1.8 * (lam[2] - lam[1])  # doubled after steps 2 and 3 converged
    un = _load_control(oracle, lam[-1])
    assert np.linalg.norm(u - un) <= 1e-8 * np.linalg.norm(un)


def test_first_step_failure_is_reported(oracle, consistent):
    p = _cantilever()
    with pytest.raises(RuntimeError):
        oracle.OracleProblem(p).arclength(tol_abs=1e-10, cg_rtol=1e-12, max_newton=2)
