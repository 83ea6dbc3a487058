"""Matrix Market (coordinate) files: the format of the SuiteSparse Matrix
Collection, which the reference's real-matrix suite reads with
Eigen::loadMarket (test/correctness/real_matrix_test.cpp:84,
bench/fetch_matrices.py:54-86).

``load_market`` returns the stored entries as a CSC matrix, exactly as the
file lists them: for a ``symmetric`` file (one triangle stored, the lower one
in the Collection) that is the triangle alone, which is what SymLDLT reads
(only the lower triangle of the values is used; multifrontal.hpp:190-216).
``real``, ``integer`` and ``pattern`` fields are accepted (pattern entries
read as 1.0); ``complex`` is rejected. Duplicate entries are summed.
"""
from __future__ import annotations

import gzip
import io
import os

import numpy as np
import scipy.sparse as sp


class MatrixMarketError(ValueError):
    pass


def _open(path):
    if str(path).endswith(".gz"):
        return io.TextIOWrapper(gzip.open(path, "rb"), encoding="ascii", errors="replace")
    return open(path, "r", encoding="ascii", errors="replace")


def load_market(path) -> sp.csc_matrix:
    """Read a coordinate Matrix Market file (optionally .gz) into CSC."""
    with _open(path) as f:
        header = f.readline().split()
        if len(header) < 5 or header[0].lower() != "%%matrixmarket":
            raise MatrixMarketError(f"{path}: not a Matrix Market file")
        obj, fmt, field, symm = (h.lower() for h in header[1:5])
        if obj != "matrix" or fmt != "coordinate":
            raise MatrixMarketError(f"{path}: only coordinate matrices are supported ({obj} {fmt})")
        if field not in ("real", "integer", "pattern", "double"):
            raise MatrixMarketError(f"{path}: unsupported field '{field}'")
        if symm not in ("general", "symmetric", "skew-symmetric"):
            raise MatrixMarketError(f"{path}: unsupported symmetry '{symm}'")
        line = f.readline()
        while line and (line.startswith("%") or not line.strip()):
            line = f.readline()
        dims = line.split()
        if len(dims) != 3:
            raise MatrixMarketError(f"{path}: bad size line")
        nr, nc, nnz = (int(x) for x in dims)
        ncol = 2 if field == "pattern" else 3
        data = np.loadtxt(f, ndmin=2, max_rows=nnz, usecols=range(ncol)) if nnz > 0 else np.zeros((0, ncol))
    if data.shape[0] != nnz:
        raise MatrixMarketError(f"{path}: expected {nnz} entries, found {data.shape[0]}")
    rows = data[:, 0].astype(np.int64) - 1
    cols = data[:, 1].astype(np.int64) - 1
    vals = np.ones(nnz) if field == "pattern" else data[:, 2].astype(np.float64)
    if nnz and (rows.min() < 0 or cols.min() < 0 or rows.max() >= nr or cols.max() >= nc):
        raise MatrixMarketError(f"{path}: index out of range")
    A = sp.coo_matrix((vals, (rows, cols)), shape=(nr, nc)).tocsc()
    A.sum_duplicates()
    A.sort_indices()
    return A


def save_market(path, A, symmetric: bool = False, comment: str | None = None) -> None:
    """Write A in coordinate real format; with ``symmetric`` only its lower
    triangle is written under a ``symmetric`` header."""
    A = sp.coo_matrix(A)
    if symmetric:
        keep = A.row >= A.col
        A = sp.coo_matrix((A.data[keep], (A.row[keep], A.col[keep])), shape=A.shape)
    order = np.lexsort((A.row, A.col))
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if symmetric else 'general'}\n")
        if comment:
            for c in comment.splitlines():
                f.write(f"% {c}\n")
        f.write(f"{A.shape[0]} {A.shape[1]} {A.nnz}\n")
        for k in order:
            f.write(f"{A.row[k] + 1} {A.col[k] + 1} {A.data[k]:.17g}\n")


def collection_path(root, group: str, name: str):
    """<root>/<group>/<name>/<name>.mtx, the layout bench/fetch_matrices.py
    unpacks the Collection's tarballs into."""
    return os.path.join(root, group, name, f"{name}.mtx")
