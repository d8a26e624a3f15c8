"""Oracle pattern (femSolidmechanics2.cpp:121-478), KSPCG restatement and Newton driver."""
import hashlib
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from mphyfem_b200 import meshgen

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cantilever_32x8x8.npz")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_config1_sizes_and_golden_pattern(oracle):
    p = meshgen.cantilever_small()
    assert (p.n_node, p.n_elem, p.n_dof) == (2673, 2048, 8019)
    op = oracle.OracleProblem(p)
    g = np.load(GOLD)
    assert op.n_free == 7776 == int(g["n_free"])
    assert op.nnz == 528750 == int(g["nnz"])
    afs, fav, rp, col = op.pattern()
    assert _sha(afs.astype(np.int32)) == str(g["assy_sha"])
    assert _sha(fav.astype(np.int32)) == str(g["fav_sha"])
    assert _sha(rp) == str(g["rowptr_sha"])
    assert _sha(col.astype(np.int32)) == str(g["col_sha"])


@pytest.mark.parametrize("mk", [lambda: meshgen.hex8_cantilever(6, 3, 2), lambda: meshgen.tet10_kuhn(3, 2, 2)])
def test_literal_and_per_node_patterns_agree(oracle, mk):
    p = mk()
    # mixed constraints: also prescribe single DOFs so rows of partly-free nodes appear
    p.fixed = p.fixed.copy()
    p.fixed[3 * (p.n_node - 1) + 1] = 1
    p.fixed[3 * (p.n_node // 2) + 2] = 1
    pats = []
    for mode in (1, 2):
        oracle.set_pattern_mode(mode)
        try:
            pats.append(oracle.OracleProblem(p).pattern())
        finally:
            oracle.set_pattern_mode(0)
    for a, b in zip(*pats):
        assert np.array_equal(a, b)
    afs, fav, rp, col = pats[0]
    # DOF numbering is node-major over free DOFs; rows sorted and unique; pattern symmetric
    assert np.all(np.diff(afs) > 0)
    assert np.array_equal(np.flatnonzero(p.fixed == 0), afs)
    for r in range(len(rp) - 1):
        assert np.all(np.diff(col[rp[r]:rp[r + 1]]) > 0)
    n = len(rp) - 1
    A = sp.csr_matrix((np.ones(len(col)), col, rp), shape=(n, n))
    assert (A != A.T).nnz == 0


def test_cg_matches_direct_solve(oracle):
    p = meshgen.cantilever_small()
    op = oracle.OracleProblem(p)
    val, rhs, _, _ = op.assemble(np.zeros(p.n_dof))
    _, _, rp, col = op.pattern()
    b = p.fnodal[np.flatnonzero(p.fixed == 0)] * 0.2
    x, its, fn, st = op.cg(val, b, rtol=1e-12)
    assert st == 0 and 100 < its < 2000
    A = sp.csr_matrix((val, col, rp), shape=(op.n_free, op.n_free))
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


def test_newton_golden_histories(oracle):
    g = np.load(GOLD)
    p = meshgen.cantilever_small()
    op = oracle.OracleProblem(p)
    oracle.set_consistent_tangent(True)
    try:
        uc, hc = op.newton(max_newton=15)
    finally:
        oracle.set_consistent_tangent(False)
    gh = g["newton_consistent_hist"]
    assert hc.shape == gh.shape
    assert np.array_equal(hc[:, :2], gh[:, :2])
    assert np.allclose(hc[:, 2], gh[:, 2], rtol=1e-6, atol=1e-12 * gh[0, 2])
    assert np.abs(uc - g["newton_consistent_u"]).max() < 1e-10
    # quadratic convergence in the last iterations of every step
    for s in np.unique(hc[:, 0]):
        r = hc[hc[:, 0] == s, 2]
        assert r[-1] < 1e-10 * r[0]


def test_reference_tangent_needs_step_cuts(oracle):
    """With the reference's own tangent the first 0.2 load step fails (indefinite tangent, then a
    negative Jacobian) and MyTime::cut halves dt, as femSolidmechanics2.cpp:827-845 does."""
    p = meshgen.cantilever_small()
    p.max_steps = 1
    op = oracle.OracleProblem(p)
    u, h = op.newton(max_newton=10)
    g = np.load(GOLD)["newton_reference_step_hist"]
    assert h[0, 2] == pytest.approx(1.171875e-3, rel=1e-12)
    assert h[2, 2] == pytest.approx(0.5 * 1.171875e-3, rel=1e-12)  # retried at dt = 0.1
    assert np.allclose(h[2:, 2], g[:, 2], rtol=1e-6, atol=1e-12 * g[0, 2])
