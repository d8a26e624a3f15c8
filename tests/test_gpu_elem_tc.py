"""Tensor-core element kernel (MPHY_PREC_MIXED_TC): FP64 residual, tangent contraction with
split-BF16 mma and FP32 accumulation, against the FP64 kernel (itself checked against the
oracle to 1e-12).

Tolerances: residual 1e-12 of the largest entry (FP64 arithmetic in both); tangent entries
within 5e-5 of each element's largest entry (the split keeps about 16 bits of every operand,
FP32 accumulation); Newton to 1e-8 with that tangent ends within 1e-6 of the FP64 oracle's
displacements."""
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


def _deformed(q, scale, seed=3):
    rng = np.random.default_rng(seed)
    u = scale * rng.standard_normal(q.n_dof)
    u[q.fixed.astype(bool)] = 0.0
    return u


@pytest.mark.parametrize("kind", ["hex8", "tet10"])
@pytest.mark.parametrize("tangent", [0, 1])
def test_element_matrices_match_fp64_kernel(env, kind, tangent):
    torch, api, _lib, ctx = env
    q = meshgen.hex8_cantilever(6, 3, 2) if kind == "hex8" else meshgen.tet10_kuhn(4, 2, 2)
    q.mats = np.array([[1.7, 0.05, 3.0]])
    mesh = api.Mesh(ctx, q)
    u = torch.tensor(_deformed(q, 0.02), device="cuda")
    K64, R64, b64 = api.calc_stiffness_and_residual(mesh, u, tangent)
    Ktc, Rtc, btc = api.calc_stiffness_and_residual(mesh, u, tangent, tensor_cores=True)
    assert b64 == btc == -1
    R64, Rtc = R64.cpu().numpy(), Rtc.cpu().numpy()
    assert np.abs(Rtc - R64).max() <= 1e-12 * np.abs(R64).max()
    K64, Ktc = K64.cpu().numpy(), Ktc.cpu().numpy()
    scale = np.abs(K64).reshape(len(K64), -1).max(axis=1)[:, None, None]
    err = np.abs(Ktc - K64) / scale
    assert err.max() <= 5e-5, err.max()
    assert err.max() > 0.0  # the tensor-core path ran, in its own arithmetic


def test_assembled_operator_matches_mixed(env):
    torch, api, _lib, ctx = env
    q = meshgen.hex8_cantilever(16, 4, 4)
    mesh = api.Mesh(ctx, q)
    pat = api.Pattern(mesh)
    u = torch.tensor(_deformed(q, 0.01), device="cuda")
    vals = {}
    for prec in (_lib.PREC_MIXED, _lib.PREC_MIXED_TC):
        s = api.SolverGpu(mesh, pat, precision=prec)
        s.calcStiffnessAndResidual(u)
        vals[prec] = s.export(want_reac=False)
    (v1, r1, _), (v2, r2, _) = vals[_lib.PREC_MIXED], vals[_lib.PREC_MIXED_TC]
    assert np.abs(r2 - r1).max() <= 1e-12 * np.abs(r1).max()
    rp, _ = pat.export_csr()
    rowmax = np.maximum.reduceat(np.abs(v1), rp[:-1])
    err = np.abs(v2 - v1) / np.repeat(rowmax, np.diff(rp))
    assert err.max() <= 2e-4, err.max()


def test_newton_with_tensor_core_tangent(env):
    torch, api, _lib, ctx = env
    from oracle.binding import OracleProblem, set_consistent_tangent
    q = meshgen.cantilever_small()
    q.newton_rtol = 1e-8
    fem = api.FemSolidmechanicsGpu(q, ctx, tangent=1, precision=_lib.PREC_MIXED_TC, rtol=1e-10, norm_type=1,
                                   max_outer=4)
    res = fem.solveWithNewtonRaphson(max_newton=15)
    assert res.status == 0
    set_consistent_tangent(True)
    try:
        u_ref, hist = OracleProblem(q).newton(cg_rtol=1e-12, max_newton=15)
    finally:
        set_consistent_tangent(False)
    assert np.abs(res.disp - u_ref).max() <= 1e-6 * np.abs(u_ref).max()
    # the inexact tangent costs at most one extra Newton iteration per step
    for step in range(1, 6):
        n_gpu = int((res.hist[:, 0] == step).sum())
        n_ref = int((hist[:, 0] == step).sum())
        assert n_gpu <= n_ref + 1, (step, n_gpu, n_ref)
