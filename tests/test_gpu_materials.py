"""GPU parity of the hyperelastic material models (Neo-Hookean, Mooney-Rivlin, Gent, Arruda-Boyce)
against the CPU oracle, through the C ABI: the batched material call, element matrices (hex8 and
tet10), the assembled system, Newton solves (single problem, mixed precision, batched form).

Tolerances as in test_gpu_parity: FP64 stresses, tangents, element matrices and assembled values
to 1e-12 relative to the largest entry; Newton solutions to 1e-8 relative.
"""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu

NH, MR, GENT, AB = 0, 1, 2, 3
DATA = {NH: [0.8, 0, 0, 0], MR: [0.4, 0.15, 0, 0], GENT: [0.7, 12.0, 0, 0], AB: [0.7, 5.0, 0, 0]}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no GPU")
    return t


@pytest.fixture(scope="module")
def api(torch):
    from mphyfem_b200 import api as a, build
    build.build()
    return a


@pytest.fixture(scope="module")
def ctx(api):
    return api.Context(0)


@pytest.fixture
def consistent(oracle):
    yield oracle.set_consistent_tangent
    oracle.set_consistent_tangent(False)


def with_models(p, models, kappa=10.0, utype=3):
    """Material k of the list on elements e with e % len(models) == k."""
    p.mat_id = (np.arange(p.n_elem) % len(models)).astype(np.int32)
    p.mat_data = np.array([DATA[m] for m in models], np.float64)
    p.mats = np.array([[d[0], 1.0 / kappa, float(utype)] for d in p.mat_data])
    p.mat_model = np.array(models, np.int32)
    return p


@pytest.mark.parametrize("model", [NH, MR, GENT, AB])
@pytest.mark.parametrize("tangent", [0, 1])
def test_material_eval_matches_oracle(api, ctx, oracle, torch, consistent, model, tangent):
    rng = np.random.default_rng(3)
    F = np.eye(3)[None] + 0.15 * rng.standard_normal((64, 3, 3))
    for utype in (3, 5):
        consistent(bool(tangent))
        ref = [oracle.material_stress_tangent(model, DATA[model], f, 0.05, utype) for f in F]
        s, Cm = api.material_stress_and_tangent(ctx, torch.tensor(F, device="cuda"), model, DATA[model], 0.05,
                                                utype, tangent)
        s, Cm = s.cpu().numpy(), Cm.cpu().numpy()
        for k in range(len(F)):
            assert np.abs(s[k] - ref[k][0]).max() <= 1e-12 * max(1.0, np.abs(ref[k][0]).max())
            assert np.abs(Cm[k] - ref[k][1]).max() <= 1e-12 * max(1.0, np.abs(ref[k][1]).max())


def _tet10():
    return meshgen.tet10_kuhn(4, 2, 2, lx=2.0)


@pytest.mark.parametrize("mk", [lambda: meshgen.hex8_cantilever(8, 3, 3), _tet10], ids=["hex8", "tet10"])
@pytest.mark.parametrize("tangent", [0, 1])
def test_element_matrices_match_oracle(api, ctx, oracle, torch, consistent, mk, tangent):
    from tests.golden.make_golden import probe_displacement
    p = with_models(mk(), [MR, GENT, AB, NH])
    u = probe_displacement(p, amp=0.01)
    mesh = api.Mesh(ctx, p)
    Ke, Re, bad = api.calc_stiffness_and_residual(mesh, torch.tensor(u, device="cuda"), tangent=tangent)
    assert bad == -1
    Ke, Re = Ke.cpu().numpy(), Re.cpu().numpy()
    consistent(bool(tangent))
    Ko, Ro, bo = oracle.OracleProblem(p).elements(u)
    assert bo == -1
    kscale = np.abs(Ko).max(axis=(1, 2))
    rscale = np.abs(Ro).max(axis=1)
    assert np.all(np.abs(Ke - Ko).max(axis=(1, 2)) <= 1e-12 * kscale)
    assert np.all(np.abs(Re - Ro).max(axis=1) <= 1e-12 * rscale + 1e-18)


def test_dense_kernel_equals_structured_neo_hookean(api, ctx, torch):
    # Mooney-Rivlin with c2 = 0 is Neo-Hookean with mu = 2 c1 (consistent tangents): the dense-tangent
    # kernel against the closed-form Neo-Hookean kernel
    from tests.golden.make_golden import probe_displacement
    p = meshgen.hex8_cantilever(8, 3, 3, mu=0.8)
    u = torch.tensor(probe_displacement(p, amp=0.01), device="cuda")
    K0, R0, _ = api.calc_stiffness_and_residual(api.Mesh(ctx, p), u, tangent=1)
    q = meshgen.hex8_cantilever(8, 3, 3, mu=0.8)
    q.mat_model = np.array([MR], np.int32)
    q.mat_data = np.array([[0.4, 0.0, 0, 0]])
    K1, R1, _ = api.calc_stiffness_and_residual(api.Mesh(ctx, q), u, tangent=1)
    assert (K1 - K0).abs().max().item() <= 1e-12 * K0.abs().max().item()
    assert (R1 - R0).abs().max().item() <= 1e-12 * R0.abs().max().item()


def test_tensor_core_kernel_refuses_other_models(api, ctx, torch):
    from mphyfem_b200 import _lib
    p = with_models(meshgen.hex8_cantilever(4, 2, 2), [GENT])
    mesh = api.Mesh(ctx, p)
    with pytest.raises(_lib.MphyError) as ei:
        api.calc_stiffness_and_residual(mesh, torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"),
                                        tensor_cores=True)
    assert ei.value.status == _lib.ERR_UNSUPPORTED


def test_set_materials_validation(api, ctx):
    from mphyfem_b200 import _lib
    p = meshgen.hex8_cantilever(2, 1, 1)
    mesh = api.Mesh(ctx, p)
    for model, data in ((7, [1.0]), (GENT, [1.0, 0.0]), (AB, [1.0, -1.0])):
        with pytest.raises(_lib.MphyError) as ei:
            mesh.set_materials([model], [data])
        assert ei.value.status == _lib.ERR_INVALID_ARG
    with pytest.raises(_lib.MphyError):
        mesh.set_materials([GENT, GENT], [[1.0, 5.0], [1.0, 5.0]])  # the mesh has one material


def test_assembly_matches_oracle(api, ctx, oracle, torch):
    from tests.golden.make_golden import probe_displacement
    p = with_models(meshgen.hex8_cantilever(7, 3, 2), [AB, MR, GENT])
    p.fixed = p.fixed.copy()
    p.fixed[3 * (p.n_node - 1) + 1] = 1
    u = probe_displacement(p, amp=0.01)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh))
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    val, rhs, reac = sol.export()
    oval, orhs, oreac, bad = oracle.OracleProblem(p).assemble(u)
    assert bad == -1
    assert np.abs(val - oval).max() <= 1e-12 * np.abs(oval).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    assert np.abs(reac - oreac).max() <= 1e-12 * np.abs(oreac).max()


def _newton_problem(models):
    p = with_models(meshgen.hex8_cantilever(12, 3, 3, traction=(0.0, 0.0, -0.03)), models)
    p.newton_rtol = 1e-9
    return p


@pytest.mark.parametrize("models", [[GENT], [AB], [MR], [MR, GENT, AB, NH]], ids=["gent", "ab", "mr", "all"])
def test_newton_matches_oracle(api, ctx, oracle, consistent, models):
    from mphyfem_b200 import _lib
    p = _newton_problem(models)
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-12, tangent=_lib.TANGENT_CONSISTENT)
    res = fem.solveWithNewtonRaphson(max_newton=15)
    assert res.status == 0
    consistent(True)
    u_ref, hist = oracle.OracleProblem(p).newton(cg_rtol=1e-12, max_newton=15)
    assert np.linalg.norm(res.disp - u_ref) <= 1e-8 * np.linalg.norm(u_ref)
    assert np.array_equal(res.hist[:, :2], hist[:, :2])


def test_mixed_precision_newton(api, ctx, oracle, consistent):
    from mphyfem_b200 import _lib
    p = _newton_problem([MR, GENT, AB, NH])
    p.newton_rtol = 1e-8
    fem = api.FemSolidmechanicsGpu(p, ctx, rtol=1e-10, tangent=_lib.TANGENT_CONSISTENT, precision=_lib.PREC_MIXED,
                                   norm_type=1)
    res = fem.solveWithNewtonRaphson(max_newton=15)
    assert res.status == 0
    consistent(True)
    u_ref, _ = oracle.OracleProblem(p).newton(cg_rtol=1e-12, max_newton=15)
    assert np.linalg.norm(res.disp - u_ref) <= 1e-6 * np.linalg.norm(u_ref)


def test_batched_newton_with_models(api, ctx, oracle, consistent):
    from mphyfem_b200 import _lib
    probs = [with_models(meshgen.hex8_cantilever(nz, 2, 2, traction=(0.0, 0.0, -0.02)), ms)
             for nz, ms in ((6, [GENT]), (9, [AB, MR]), (4, [NH]), (7, [MR, GENT, AB]))]
    for q in probs:
        q.newton_rtol = 1e-8
    b = api.BatchGpu(probs, ctx, rtol=1e-12, norm_type=0, tangent=_lib.TANGENT_CONSISTENT)
    out = b.newton_run(max_newton=15)
    assert (out["status"] == 0).all(), out["status"]
    consistent(True)
    for i, q in enumerate(probs):
        u_ref, _ = oracle.OracleProblem(q).newton(cg_rtol=1e-12, max_newton=15)
        ui = out["disp"][b.instance_slice(i)]
        assert np.linalg.norm(ui - u_ref) <= 1e-8 * np.linalg.norm(u_ref), i
