"""Accuracy of the headline method beyond the parity case, at mid sizes of the three meshes the
workloads use: hex8 cantilever 128x32x32 (0.42 M DOFs), two-phase inclusions 64x16x16 and tet10
Kuhn 24x12x12 (kappa = 100).

For each, the first load step (lambda = dt from u = 0) is converged by Newton with the consistent
tangent, once by the plain FP64 GPU method (FP64 element kernel, FP64 matrix, Jacobi-PCG) and once
by the headline method (FP32 tangent and operator, FP64 residual and refinement, Jacobi + the
rigid-body coarse space). Bar: max|u - u64| <= 1e-6 max|u64|, both Newton runs converged.

The FP64 GPU Newton itself is checked against the oracle's Newton (orc_newton_run, the
restatement of femSolidmechanics2.cpp:730-851) on hex8 64x16x16: the same Newton iteration
count, residual norms within 1e-6 relative above 1e-9 ||R_0||, Krylov counts within 1 % while the
residual is above 1e-3 of its largest value, displacements within 1e-8.
"""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu

DISP_TOL = 1e-6  # max|u - u64| / max|u64|, the accuracy the headline method must keep


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return api, _lib, api.Context(0)


# (mesh, Newton relative tolerance, Krylov true-residual tolerance, coarse aggregates). The
# two-phase mesh's FP64 residual floor (the cancellation of a stiffness contrast of 1000 in
# ||b - A x||) lies near 1e-8 ||b||, so its solves stop at 5e-8 and Newton at 1e-7.
CASES = {
    "hex8_128x32x32": (lambda: meshgen.hex8_cantilever(128, 32, 32), 1e-8, 1e-8, 128),
    "two_phase_64x16x16": (lambda: meshgen.two_phase_inclusions(64, 16, 16, seed=23), 1e-7, 5e-8, 64),
    "tet10_kuhn_24x12x12": (lambda: meshgen.tet10_kuhn(24, 12, 12), 1e-8, 1e-8, 64),
}


def _first_step(api, _lib, ctx, p, newton_rtol, **opts):
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    s = api.SolverGpu(mesh, pat, tangent=_lib.TANGENT_CONSISTENT, **opts)
    r = api.newton_run(s, p, max_newton=12, tol_rel=newton_rtol, t_final=p.dt, max_steps=1)
    s.close()
    return r


@pytest.mark.parametrize("case", sorted(CASES))
def test_headline_method_matches_fp64_at_mid_size(env, case):
    api, _lib, ctx = env
    make, newton_rtol, krylov_rtol, coarse = CASES[case]
    p = make()
    common = dict(rtol=krylov_rtol, norm_type=1, max_outer=4, max_it=40000)
    r64 = _first_step(api, _lib, ctx, p, newton_rtol, precision=_lib.PREC_FP64, **common)
    rmx = _first_step(api, _lib, ctx, p, newton_rtol, precision=_lib.PREC_MIXED, coarse_aggregates=coarse, **common)
    for r in (r64, rmx):
        assert r.status == 0
        assert np.count_nonzero(r.hist[:, 1] == 1) == 1, r.hist[:, :5]  # converged without a cut
        assert r.hist[-1, 2] < newton_rtol * r.hist[0, 2], r.hist[:, :4]
    assert r64.hist[0, 2] == pytest.approx(rmx.hist[0, 2], rel=1e-12)  # the same load, the same R_0
    scale = np.abs(r64.disp).max()
    err = np.abs(rmx.disp - r64.disp).max() / scale
    assert err <= DISP_TOL, (case, err)


def test_fp64_gpu_newton_matches_oracle_newton(env, oracle):
    import os
    api, _lib, ctx = env
    p = meshgen.hex8_cantilever(64, 16, 16)
    p.t_final = p.dt
    p.max_steps = 1
    r = _first_step(api, _lib, ctx, p, 1e-8, precision=_lib.PREC_FP64, rtol=1e-10, max_it=20000)
    oracle.set_consistent_tangent(True)
    try:
        op = oracle.OracleProblem(p)
        uo, ho = op.newton(tol_rel=1e-8, cg_rtol=1e-10, cg_maxit=20000, max_newton=12, nthreads=os.cpu_count() or 1)
    finally:
        oracle.set_consistent_tangent(False)
    h = r.hist
    assert r.status == 0
    assert h.shape[0] == ho.shape[0], (h[:, :3], ho)
    big = ho[:, 2] > 1e-9 * ho[0, 2]
    assert np.allclose(h[big, 2], ho[big, 2], rtol=1e-6)
    # Krylov iterations per Newton iteration, while the right-hand side is well above round-off
    # (near convergence it is rounding noise and CG's path depends on its last bits)
    sig = ho[:, 2] > 1e-3 * ho[:, 2].max()
    assert np.all(np.abs(h[sig, 3] - ho[sig, 3]) <= np.maximum(2, 0.01 * ho[sig, 3])), (h[:, 3], ho[:, 3])
    assert np.abs(r.disp - uo).max() <= 1e-8 * np.abs(uo).max()
