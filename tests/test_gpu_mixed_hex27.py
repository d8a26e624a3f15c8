"""GPU P2-P1 hex27 mixed element (Elem_Solid_3D_Mixed1 with 27 nodes: triquadratic displacement,
trilinear pressure on the 8 corners, the 3x3x3 rule) against the oracle's restatement: pressure
DOF numbering (bit-exact), element blocks (1e-12 of each element's largest entry), the assembled
two-field operator and right-hand side (1e-12), MINRES against a sparse LU (1e-8), Newton
histories and solutions (1e-8), and the homogeneous uniaxial patch."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu

NH, GENT = 0, 2
DATA = {NH: [0.8, 0, 0, 0], GENT: [0.7, 12.0, 0, 0]}


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return torch, api, _lib, api.Context(0)


@pytest.fixture
def consistent(oracle):
    yield oracle.set_consistent_tangent
    oracle.set_consistent_tangent(False)


def _problem(models=(NH,), kappa=20.0, jitter=0.15):
    p = meshgen.hex27_cantilever(3, 2, 2, lx=2.0, jitter=jitter, traction=(0.0, 0.0, -0.02))
    p.mat_id = (np.arange(p.n_elem) % len(models)).astype(np.int32)
    p.mat_data = np.array([DATA[m] for m in models], np.float64)
    p.mats = np.array([[d[0], 1.0 / kappa, 3.0] for d in p.mat_data])
    p.mat_model = np.array(models, np.int32)
    p.newton_rtol = 1e-9
    return p


def _state(p, seed=3):
    rng = np.random.default_rng(seed)
    x = p.coords
    s = x[:, 0] / x[:, 0].max()
    u = np.zeros_like(x)
    u[:, 2] = -0.05 * s * s
    u += 0.003 * rng.standard_normal(u.shape) * s[:, None]
    up = 0.6 * u
    pres = 0.05 * rng.standard_normal(p.n_node)
    return u.ravel(), up.ravel(), pres


def test_pressure_numbering_corner_nodes(env):
    torch, api, _lib, ctx = env
    from oracle.mixed_ref import pressure_dofs
    p = _problem()
    m = api.MixedSolidGpu(p, ctx)
    assert np.array_equal(m.pressure_nodes(), pressure_dofs(p)[0])
    assert m.n_pres == len(np.unique(p.conn[:, :8]))


@pytest.mark.parametrize("models", [(NH,), (GENT, NH)], ids=["nh", "gent_nh"])
@pytest.mark.parametrize("tangent", [0, 1])
def test_element_blocks_match_oracle(env, oracle, consistent, models, tangent):
    torch, api, _lib, ctx = env
    from oracle.mixed_ref import MixedProblem
    p = _problem(models)
    u, up, pres = _state(p)
    m = api.MixedSolidGpu(p, ctx, tangent=tangent)
    t = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    Kuu, FU, Kup, Kpp, FP, bad = (v.cpu().numpy() if hasattr(v, "cpu") else v
                                  for v in m.elements(t(u), t(up), t(pres)))
    assert bad == -1 and Kuu.shape == (p.n_elem, 81, 81) and Kup.shape == (p.n_elem, 81, 8)
    consistent(bool(tangent))
    oKuu, oKup, oKpp, oFU, oFP, obad = MixedProblem(p).elements(u, up, pres)
    assert obad == -1
    for g, o in ((Kuu, oKuu), (Kup, oKup), (Kpp, oKpp), (FU, oFU), (FP, oFP)):
        scale = np.abs(o).reshape(len(o), -1).max(axis=1) + 1e-300
        err = np.abs(g - o).reshape(len(o), -1).max(axis=1)
        assert np.all(err <= 1e-12 * scale)


def test_assembled_operator_matches_oracle(env, oracle, consistent):
    torch, api, _lib, ctx = env
    from oracle.mixed_ref import MixedProblem
    p = _problem((GENT, NH))
    u, up, pres = _state(p, 4)
    m = api.MixedSolidGpu(p, ctx, tangent=1)
    t = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    lam = 0.3
    nrm = m.assemble(t(u), t(up), t(pres), lam, t(p.fnodal))
    consistent(True)
    mp = MixedProblem(p)
    A, rhs, reac, bad = mp.assemble(u, up, pres)
    rhs[:mp.nu] += lam * p.fnodal[mp.afs]
    assert bad == -1
    assert nrm == pytest.approx(np.linalg.norm(rhs), rel=1e-12)
    g_rhs, g_reac, _ = (v.cpu().numpy() for v in m.vectors())
    nd = p.n_dof
    assert np.abs(g_rhs[mp.afs] - rhs[:mp.nu]).max() <= 1e-12 * np.abs(rhs).max()
    assert np.abs(g_rhs[nd:] - rhs[mp.nu:]).max() <= 1e-12 * np.abs(rhs).max()
    assert np.abs(g_reac - reac).max() <= 1e-12 * np.abs(reac).max()
    x = np.random.default_rng(9).standard_normal(m.n)
    y = m.apply(t(x)).cpu().numpy()
    yo = A @ np.concatenate([x[mp.afs], x[nd:]])
    scale = np.abs(yo).max()
    assert np.abs(y[mp.afs] - yo[:mp.nu]).max() <= 1e-12 * scale
    assert np.abs(y[nd:] - yo[mp.nu:]).max() <= 1e-12 * scale


def test_minres_matches_direct_solve(env, oracle, consistent):
    torch, api, _lib, ctx = env
    import scipy.sparse.linalg as spla
    from oracle.mixed_ref import MixedProblem
    p = _problem((NH,), kappa=1000.0)
    u, up, pres = _state(p, 5)
    m = api.MixedSolidGpu(p, ctx, tangent=1, rtol=1e-12)
    t = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    m.assemble(t(u), t(up), t(pres), 0.5, t(p.fnodal))
    rc, its, relres = m.solve()
    assert rc == 0 and relres <= 1e-10
    _, _, x = (v.cpu().numpy() for v in m.vectors())
    consistent(True)
    mp = MixedProblem(p)
    A, rhs, _, _ = mp.assemble(u, up, pres)
    rhs[:mp.nu] += 0.5 * p.fnodal[mp.afs]
    xo = spla.spsolve(A.tocsc(), rhs)
    xg = np.concatenate([x[mp.afs], x[p.n_dof:]])
    assert np.linalg.norm(xg - xo) <= 1e-8 * np.linalg.norm(xo)


@pytest.mark.parametrize("models,tangent", [((NH,), 1), ((GENT, NH), 1), ((NH,), 0)],
                         ids=["nh", "gent_nh", "nh_reference"])
def test_newton_matches_oracle(env, oracle, consistent, models, tangent):
    torch, api, _lib, ctx = env
    from oracle.mixed_ref import MixedProblem
    p = _problem(models, kappa=200.0)
    m = api.MixedSolidGpu(p, ctx, tangent=tangent, rtol=1e-12)
    res = m.solveWithNewtonRaphson(max_newton=15)
    assert res.status == 0
    consistent(bool(tangent))
    u, pres, hist = MixedProblem(p).newton(max_newton=15)
    assert np.array_equal(res.hist[:, :2], hist[:, :2])
    assert np.linalg.norm(res.disp - u) <= 1e-8 * np.linalg.norm(u)
    corners = np.unique(p.conn[:, :8])
    assert np.linalg.norm(res.pres[corners] - pres[corners]) <= 1e-8 * np.linalg.norm(pres[corners])


def test_uniaxial_patch(env, consistent):
    """Dead end load along x with symmetry supports: the homogeneous state u = (a x, b y, b z)
    with the uniform corner pressure K (J - 1)."""
    torch, api, _lib, ctx = env
    p = meshgen.hex27_cantilever(3, 2, 2, lx=2.0, traction=(0.05, 0.0, 0.0))
    X = p.coords
    fx = np.zeros((p.n_node, 3), np.uint8)
    fx[np.isclose(X[:, 0], 0.0), 0] = 1
    fx[np.isclose(X[:, 1], 0.0), 1] = 1
    fx[np.isclose(X[:, 2], 0.0), 2] = 1
    p.fixed = fx.ravel()
    p.mats = np.array([[1.0, 1.0 / 20.0, 3.0]])
    p.dt, p.t_final, p.max_steps = 0.25, 1.0, 4
    p.newton_rtol = 1e-10
    m = api.MixedSolidGpu(p, ctx, tangent=1, rtol=1e-13)
    res = m.solveWithNewtonRaphson(max_newton=15)
    assert res.status == 0
    U = res.disp.reshape(-1, 3)
    a = U[:, 0] @ X[:, 0] / (X[:, 0] @ X[:, 0])
    bb = U[:, 1] @ X[:, 1] / (X[:, 1] @ X[:, 1])
    assert np.abs(U[:, 0] - a * X[:, 0]).max() <= 1e-9 * abs(a)
    assert np.abs(U[:, 1] - bb * X[:, 1]).max() <= 1e-9 * abs(bb)
    J = (1 + a) * (1 + bb) ** 2
    corners = np.unique(p.conn[:, :8])
    assert np.allclose(res.pres[corners], 20.0 * (J - 1.0), rtol=1e-8)


def test_displacement_solver_refuses_hex27(env):
    torch, api, _lib, ctx = env
    p = _problem()
    mesh = api.Mesh(ctx, p)
    with pytest.raises(_lib.MphyError):
        api.SolverGpu(mesh, api.Pattern(mesh))
