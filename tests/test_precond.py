"""Block-Jacobi preconditioner (host side, no GPU): the diagonal blocks
assembled from the leaves equal the same blocks of the dense matrix, and the
preconditioner's leaves are their inverses."""
import numpy as np

import hlr_b200 as hlr
from hlr_b200.solve import block_jacobi_leaves, diagonal_blocks


def _random_h(n=10, seed=0):
    """A 2 x 2 block matrix with dense diagonal leaves and low-rank
    off-diagonal leaves, made symmetric positive definite, and its dense form."""
    rng = np.random.default_rng(seed)
    h = n // 2
    U = rng.standard_normal((h, 2))
    V = rng.standard_normal((n - h, 2))
    D0 = rng.standard_normal((h, h))
    D1 = rng.standard_normal((n - h, n - h))
    D0 = D0 @ D0.T + n * np.eye(h)
    D1 = D1 @ D1.T + n * np.eye(n - h)
    ll = hlr.LeafList(n, n)
    ll.add_dense(0, 0, D0)
    ll.add_lowrank(0, h, U, V)
    ll.add_lowrank(h, 0, V, U)
    ll.add_dense(h, h, D1)
    A = np.zeros((n, n))
    A[:h, :h], A[h:, h:] = D0, D1
    A[:h, h:] = U @ V.T
    A[h:, :h] = V @ U.T
    return ll, A


def test_diagonal_blocks_match_dense_matrix():
    ll, A = _random_h(10)
    for block in (3, 4, 5, 10):
        for i0, B in diagonal_blocks(ll, block):
            i1 = min(i0 + block, 10)
            assert np.allclose(B, A[i0:i1, i0:i1], atol=1e-12), (block, i0)


def test_block_jacobi_leaves_are_inverses():
    ll, A = _random_h(12, seed=3)
    W = block_jacobi_leaves(ll, 4)
    d = W.h_desc()
    dense = [d.blocks[k] for k in range(d.nblocks) if d.blocks[k].kind == hlr.LEAF_DENSE]
    assert len(dense) == 3
    for b in dense:
        Wk = np.ctypeslib.as_array(b.D, shape=(b.ldd * b.ncols,)).reshape(b.ncols, b.ldd).T[:b.nrows]
        i0 = int(b.row0)
        assert np.allclose(Wk @ A[i0:i0 + 4, i0:i0 + 4], np.eye(4), atol=1e-10)
    # the other leaves have rank 0 and, with the dense ones, cover the matrix
    # exactly once (the planner rejects gaps and overlaps)
    cover = np.zeros((12, 12), dtype=int)
    for k in range(d.nblocks):
        b = d.blocks[k]
        assert b.kind == hlr.LEAF_DENSE or b.rank == 0
        cover[b.row0:b.row0 + b.nrows, b.col0:b.col0 + b.ncols] += 1
    assert (cover == 1).all()
    assert hlr.plan_info(W)["matrix_bytes"] == 3 * 16 * 8
