"""Many independent sparse symmetric systems, factorized and solved together.

Each system is ordered on its own (AMD by default), and the permuted systems
are placed as the diagonal blocks of one block-diagonal matrix, factorized
with the natural order: its elimination tree is the forest of the systems'
trees, so every level launch of the factorization and of the solve covers
the fronts of all systems at once (one small-front launch for all their
leaves, one panel launch per iteration for all their large fronts). With
graph launch on, the whole static factorization pass is one CUDA graph.
Results per system are those of factorizing it alone (the fronts and their
pivots are the same); only the launches are shared.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import matrices as M
from .solver import OrderingType, SymLDLT


class BatchedSolver:
    def __init__(self, systems, ordering=OrderingType.AMD, device: int = 0, graph: bool = True):
        """systems: lower triangles (CSC) of the symmetric matrices."""
        self.perms, blocks, self.offsets = [], [], [0]
        for A in systems:
            s = SymLDLT(device)
            s.setOrdering(ordering)
            s.analyzePattern(A)
            perm = np.asarray(s.symbolicFactor().perm)
            full = M.sym_full(A).tocsr()
            blocks.append(sp.tril(full[perm][:, perm]).tocsc())
            self.perms.append(perm)
            self.offsets.append(self.offsets[-1] + A.shape[0])
        self.A = sp.block_diag(blocks, format="csc")
        self.A.sort_indices()
        self.n = self.A.shape[0]
        self.solver = SymLDLT(device)
        self.solver.setOrdering(OrderingType.Natural)
        self.solver.setGraphLaunch(graph)
        self.solver.analyzePattern(self.A)

    def factorize(self):
        self.solver.factorize(self.A)

    def stack(self, Bs):
        """Right-hand sides of every system (n_i x nrhs) into the batch order."""
        nrhs = Bs[0].shape[1] if Bs[0].ndim == 2 else 1
        out = np.zeros((self.n, nrhs), order="F")
        for perm, o, B in zip(self.perms, self.offsets, Bs):
            out[o:o + len(perm)] = np.asarray(B).reshape(len(perm), nrhs)[perm]
        return out

    def unstack(self, X):
        xs = []
        for perm, o in zip(self.perms, self.offsets):
            x = np.zeros((len(perm), X.shape[1]))
            x[perm] = X[o:o + len(perm)]
            xs.append(x)
        return xs

    def solve(self, Bs):
        return self.unstack(self.solver.solve(self.stack(Bs)))
