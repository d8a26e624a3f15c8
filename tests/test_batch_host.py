"""Batched form, host side: the union mesh is the disjoint union of the instances, and its
sparsity pattern (oracle, CPU) is the block-diagonal stack of the instances' patterns."""
import numpy as np

from mphyfem_b200 import meshgen
from oracle.binding import OracleProblem


def test_batched_blocks_sizes_and_union_offsets():
    probs = meshgen.batched_blocks(512, seed=11)
    u = meshgen.batch_union(probs)
    npt = u.meta["inst_node_ptr"]
    assert len(npt) == 513 and npt[0] == 0 and npt[-1] == u.n_node
    assert u.n_elem == sum(q.n_elem for q in probs)
    assert 1.9e6 < u.n_elem < 2.2e6   # about 2.0 M elements at seed 11
    e = u.meta["inst_elem_ptr"]
    for i in (0, 17, 511):
        c = u.conn[e[i]:e[i + 1]]
        assert c.min() >= npt[i] and c.max() < npt[i + 1]
        assert (u.mat_id[e[i]:e[i + 1]] == i).all()
        np.testing.assert_array_equal(u.fixed[3 * npt[i]:3 * npt[i + 1]], probs[i].fixed)


def test_union_pattern_is_block_diagonal():
    probs = [meshgen.hex8_cantilever(3, 1, 1), meshgen.hex8_cantilever(5, 2, 1), meshgen.hex8_cantilever(2, 2, 2)]
    u = meshgen.batch_union(probs)
    _, _, rp_u, col_u = OracleProblem(u).pattern()
    rows, off = [], 0
    start = 0
    for q in probs:
        _, _, rp, col = OracleProblem(q).pattern()
        for r in range(len(rp) - 1):
            rows.append(col[rp[r]:rp[r + 1]] + off)
        off += int(q.n_free)
        start += q.n_node
    assert len(rows) == len(rp_u) - 1
    for r, ref in enumerate(rows):
        np.testing.assert_array_equal(col_u[rp_u[r]:rp_u[r + 1]], ref)
