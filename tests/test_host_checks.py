"""Host-side pattern checks of the drop-in call on inputs large enough for
their parallel passes (>= 2^17 stored entries), against the oracle and the
reference's rules (src/speigs_core.c:363-401 and :445-466).  No device work
is needed: a non-symmetric input is rejected before any, and the component
labels come from speigs_components()."""
import numpy as np
import scipy.sparse as sp

from conftest import import_oracle

NOTSYM = -6


def _call(pkg, lib, A):
    s = pkg.speigs
    o = s.default_opts(lib, tol=1e-10)
    rc, *_ = s.speigs(A, 1, s.SM, o, vectors=False, lib=lib)
    return rc


def test_components_match_oracle(pkg, lib):
    w = pkg.workloads
    blocks = [w.lap3d(20), w.lap3d(20), w.lap3d(24), w.lap3d(20)]
    A = sp.block_diag(blocks, format="coo")
    n = A.shape[0]
    # explicit zeros between the blocks do not connect them
    rows = np.concatenate([A.row, [5, 8005]])
    cols = np.concatenate([A.col, [8005, 5]])
    vals = np.concatenate([A.data, [0.0, 0.0]])
    A = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    assert A.nnz >= 1 << 17
    nc, lab = pkg.speigs.components(A, lib=lib)
    onc, olab = import_oracle().find_components(A)
    assert nc == onc == 4
    assert np.array_equal(lab, olab)


def test_components_random_graph(pkg, lib):
    rng = np.random.default_rng(11)
    n = 60000
    m = 80000                                    # below the connectivity threshold
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    A = sp.coo_matrix((np.ones(m), (r, c)), shape=(n, n))
    A = (A + A.T + sp.eye(n)).tocsc()
    assert A.nnz >= 1 << 17
    nc, lab = pkg.speigs.components(A, lib=lib)
    onc, olab = import_oracle().find_components(A)
    assert nc == onc
    assert np.array_equal(lab, olab)


def test_symmetry_verdicts(pkg, lib):
    ora = import_oracle()
    A = pkg.workloads.lap3d(40).tocsc()
    A.sort_indices()
    assert A.nnz >= 1 << 17
    assert ora.check_symmetry(A) == 1
    assert _call(pkg, lib, A) != NOTSYM

    # one upper entry off by 1e-10 relative: not symmetric
    B = A.copy()
    col = 1000
    q = B.indptr[col]
    assert B.indices[q] < col
    B.data[q] *= 1.0 + 1e-10
    assert ora.check_symmetry(B) == 0
    assert _call(pkg, lib, B) == NOTSYM

    # upper-triangle storage is accepted
    U = sp.triu(A, format="csc")
    assert ora.check_symmetry(U) == 2
    assert _call(pkg, lib, U) != NOTSYM

    # row indices out of order in one column: the reference compares the
    # transpose entry by entry, so this symmetric matrix is rejected
    Ap, Ai, Ax = A.indptr.astype(np.int64), A.indices.astype(np.int64).copy(), A.data.copy()
    a, b = Ap[col], Ap[col + 1]
    Ai[a:b] = Ai[a:b][::-1].copy()
    Ax[a:b] = Ax[a:b][::-1].copy()
    assert _call(pkg, lib, (A.shape[0], Ap, Ai, Ax)) == NOTSYM
