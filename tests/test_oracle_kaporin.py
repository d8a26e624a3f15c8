"""The learned preconditioner's training loss, restated on the CPU (oracle/gnn_ref.py), against
Kaporin's theorem: over a lower block pattern, exact block FSAI minimises the K-condition number
K(G A G^T) = (tr / N) / det^(1/N). So K(exact FSAI) <= K(block-Jacobi FSAI) <= K(point Jacobi),
and the zero-weight network (block-Jacobi FSAI by construction) has the block-Jacobi value."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen
from oracle import fsai_ref, gnn_ref
from oracle.binding import OracleProblem


def _log_k(A, lrow, lcol, blocks):
    """log K of G A G^T for G given by its lower blocks (dense, small problems)."""
    n_node = len(lrow) - 1
    N = 3 * n_node
    G = np.zeros((N, N))
    for n in range(n_node):
        for j in range(lrow[n], lrow[n + 1]):
            m = lcol[j]
            G[3 * n:3 * n + 3, 3 * m:3 * m + 3] = blocks[j]
    M = G @ A @ G.T
    sign, logdet = np.linalg.slogdet(M)
    assert sign > 0
    return np.log(np.trace(M) / N) - logdet / N


@pytest.fixture(scope="module")
def case():
    p = meshgen.two_phase_inclusions(8, 3, 3, seed=5, r_range=(0.3, 0.45))
    o = OracleProblem(p)
    val, _, _, _ = o.assemble(np.zeros(p.n_dof))
    _, _, rp, col = o.pattern()
    A = fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val).toarray()
    nbrs = fsai_ref.node_neighbours(p.conn, p.n_node)
    lrow, lcol, G = fsai_ref.block_fsai(fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val), nbrs)
    return p, A, nbrs, np.asarray(lrow), np.asarray(lcol), np.asarray(G)


def test_exact_fsai_minimises_kaporin(case):
    p, A, nbrs, lrow, lcol, G = case
    d = np.sqrt(np.abs(np.diag(A)))
    blocks_bj, blocks_pj = np.zeros_like(G), np.zeros_like(G)
    for n in range(p.n_node):
        j = lrow[n + 1] - 1          # the diagonal block is last in its lower row
        assert lcol[j] == n
        Ann = A[3 * n:3 * n + 3, 3 * n:3 * n + 3]
        blocks_bj[j] = np.linalg.cholesky(np.linalg.inv(Ann)).T
        blocks_pj[j] = np.diag(1.0 / d[3 * n:3 * n + 3])
    k_fsai, k_bj, k_pj = (_log_k(A, lrow, lcol, b) for b in (G, blocks_bj, blocks_pj))
    assert k_fsai < k_bj - 1e-3 < k_pj


def test_zero_network_is_block_jacobi_under_the_loss(case):
    p, A, nbrs, lrow, lcol, G = case
    import scipy.sparse as sp
    loss, grads, pred = gnn_ref.loss_and_grads(np.zeros(gnn_ref.layout()[1], np.float32),
                                               sp.csr_matrix(A), p.fixed, nbrs, lrow, lcol)
    # the loss is log K + (1/N) log det of the scaled operator
    d = np.sqrt(np.abs(np.diag(A)))
    As = A / np.outer(d, d)
    const = np.linalg.slogdet(As)[1] / A.shape[0]
    k_pred = _log_k(A, lrow, lcol, pred)
    assert abs((loss - const) - k_pred) < 1e-9
    blocks_bj = np.zeros_like(G)
    for n in range(p.n_node):
        j = lrow[n + 1] - 1
        blocks_bj[j] = np.linalg.cholesky(np.linalg.inv(A[3 * n:3 * n + 3, 3 * n:3 * n + 3])).T
    assert abs(k_pred - _log_k(A, lrow, lcol, blocks_bj)) < 1e-9
