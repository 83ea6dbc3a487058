"""The batched solver's block-diagonal matrix (host side, no GPU): each
system's lower triangle, permuted by its own ordering, as one diagonal
block, exactly as tril(P A P^T) of each system would give."""
import numpy as np
import scipy.sparse as sp

from ma57_b200 import OrderingType, SymLDLT
from ma57_b200 import matrices as M
from ma57_b200.batch import BatchedSolver


def test_block_diagonal_equals_permuted_systems():
    systems = [M.config4_system(i)[0] for i in range(12)]
    bs = BatchedSolver(systems)
    blocks = []
    for A, perm in zip(systems, bs.perms):
        s = SymLDLT()
        s.setOrdering(OrderingType.AMD)
        s.analyzePattern(A)
        np.testing.assert_array_equal(perm, s.symbolicFactor().perm)
        full = M.sym_full(A).tocsr()
        blocks.append(sp.tril(full[perm][:, perm]).tocsc())
    ref = sp.block_diag(blocks, format="csc")
    ref.sort_indices()
    np.testing.assert_array_equal(bs.A.indptr, ref.indptr)
    np.testing.assert_array_equal(bs.A.indices, ref.indices)
    np.testing.assert_array_equal(bs.A.data, ref.data)
    assert bs.offsets[-1] == sum(A.shape[0] for A in systems)
