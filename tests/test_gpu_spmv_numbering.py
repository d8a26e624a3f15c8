"""The solver's SpMV against the exported CSR operator, for the lexicographic numbering of a box
(every neighbour within a few hundred node ids) and for the same mesh under a seeded random node
permutation (neighbours anywhere in the 40,625 nodes, so the SELL slices gather from all over
the vector). The two numberings give the same operator up to the permutation.

Tolerances: FP64 storage to 1e-13 of the largest |y| (summation order only); FP32 storage to
1e-6 (FP32 values of the off-diagonal blocks, diagonal blocks formed in FP64).
"""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu


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


def _permuted(p, seed):
    """The same problem with its nodes renumbered by a seeded permutation: node n becomes perm[n]."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(p.n_node).astype(np.int64)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(p.n_node)
    q = meshgen.Problem(name=p.name + "_perm", coords=p.coords[inv], conn=perm[p.conn].astype(np.int32),
                        mat_id=p.mat_id, mats=p.mats,
                        fixed=p.fixed.reshape(-1, 3)[inv].ravel(), fnodal=p.fnodal.reshape(-1, 3)[inv].ravel())
    return q, perm


def _csr_apply(rp, col, val, x):
    y = np.zeros(len(rp) - 1)
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    np.add.at(y, rows, val * x[col])
    return y


def _check(api, ctx, torch, p, precision, seed):
    from mphyfem_b200 import _lib
    from tests.golden.make_golden import probe_displacement
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, precision=precision)
    u = probe_displacement(p, amp=0.001)
    sol.calcStiffnessAndResidual(torch.tensor(u, device="cuda"))
    assert sol.currentStatus == 3
    val, _, _ = sol.export()
    rp, col = pat.export_csr()
    free = np.flatnonzero(p.fixed == 0)
    rng = np.random.default_rng(seed)
    x = np.zeros(p.n_dof)
    x[free] = rng.standard_normal(free.size)
    y = torch.empty(p.n_dof, dtype=torch.float64, device="cuda")
    sol.spmv(torch.tensor(x, device="cuda"), y)
    torch.cuda.synchronize()
    yg = y.cpu().numpy()
    yo = _csr_apply(rp, col, val, x[free])
    tol = 1e-13 if precision == _lib.PREC_FP64 else 1e-6
    assert np.abs(yg[free] - yo).max() <= tol * np.abs(yo).max()
    sol.close()
    return yg


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_spmv_natural_and_permuted_numbering(api, ctx, torch, prec):
    from mphyfem_b200 import _lib
    precision = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
    p = meshgen.hex8_cantilever(64, 24, 24)  # 65 x 25 x 25 = 40,625 nodes
    y_nat = _check(api, ctx, torch, p, precision, 5)
    q, perm = _permuted(p, 17)
    # the same x in the permuted numbering gives the same y, permuted
    rng = np.random.default_rng(5)
    free = np.flatnonzero(p.fixed == 0)
    x = np.zeros(p.n_dof)
    x[free] = rng.standard_normal(free.size)
    from tests.golden.make_golden import probe_displacement
    _check(api, ctx, torch, q, precision, 5)
    mesh = api.Mesh(ctx, q)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, precision=precision)
    u = probe_displacement(p, amp=0.001).reshape(-1, 3)
    uq = np.empty_like(u)
    uq[perm] = u
    sol.calcStiffnessAndResidual(torch.tensor(uq.ravel(), device="cuda"))
    xq = np.empty((p.n_node, 3))
    xq[perm] = x.reshape(-1, 3)
    y = torch.empty(p.n_dof, dtype=torch.float64, device="cuda")
    sol.spmv(torch.tensor(xq.ravel(), device="cuda"), y)
    torch.cuda.synchronize()
    yq = y.cpu().numpy().reshape(-1, 3)[perm].ravel()
    tol = 1e-12 if prec == "fp64" else 1e-6
    assert np.abs(yq[free] - y_nat[free]).max() <= tol * np.abs(y_nat[free]).max()
    sol.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_spmv_dot_is_the_spmv_with_its_dot(api, ctx, torch, prec):
    """mphy_solver_spmv_dot (the CG iteration's SpMV kernel with the fused (x, Ax)) gives the same
    y as mphy_solver_spmv, bit for bit, and (x, y) to 1e-11 of torch's FP64 dot (both are FP64
    sums of ~10^5 terms in different orders)."""
    from mphyfem_b200 import _lib
    from tests.golden.make_golden import probe_displacement
    precision = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
    p = meshgen.hex8_cantilever(48, 12, 12)
    mesh = api.Mesh(ctx, p)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), precision=precision)
    sol.calcStiffnessAndResidual(torch.tensor(probe_displacement(p, amp=0.001), device="cuda"))
    x = torch.tensor(np.random.default_rng(3).standard_normal(p.n_dof), device="cuda")
    x[torch.tensor(p.fixed == 1, device="cuda")] = 0.0
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)
    sol.spmv(x, y1)
    xy = sol.spmv_dot(x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    ref = float(torch.dot(x, y2))
    assert abs(xy - ref) <= 1e-11 * abs(ref)
    sol.close()
