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

from .solver import OrderingType, SymLDLT


class BatchedSolver:
    def __init__(self, systems, ordering=OrderingType.AMD, device: int = 0, graph: bool = True):
        """systems: lower triangles (CSC) of the symmetric matrices."""
        self.perms, self.offsets = [], [0]
        rows, cols, vals = [], [], []
        for A in systems:
            s = SymLDLT(device)
            s.setOrdering(ordering)
            s.analyzePattern(A)
            perm = np.asarray(s._analysis.perm())
            # the permuted lower triangle: every stored entry (r >= c) moves to
            # (max, min) of its new positions, shifted to the system's block
            C = sp.tril(sp.csc_matrix(A)).tocoo()
            inv = np.empty_like(perm)
            inv[perm] = np.arange(len(perm), dtype=perm.dtype)
            r, c = inv[C.row], inv[C.col]
            o = self.offsets[-1]
            rows.append(np.maximum(r, c) + o)
            cols.append(np.minimum(r, c) + o)
            vals.append(C.data)
            self.perms.append(perm)
            self.offsets.append(o + A.shape[0])
        n = self.offsets[-1]
        self.A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
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
