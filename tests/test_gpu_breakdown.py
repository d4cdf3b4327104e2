"""Lanczos breakdown (an invariant Krylov subspace) through the C ABI, against
the reference's solver compiled on the CPU (oracle/_ref), on identical CSC
bytes.

The reference restarts the recurrence with a random vector orthogonalised
against the basis when beta_j <= 1e-13 ||A||_1 (src/speigs_core.c:205-216),
and shortens the basis when three such vectors fail.  The device library
checks beta_j one step late (the next step is already queued); these cases
make that path run: a diagonal matrix with four distinct eigenvalues (every
Krylov space of it has dimension <= 4, so the basis breaks down every few
steps) and a matrix smaller than the basis (the space is exhausted).
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _both(pkg, lib, ref_lib, A, k, which):
    s = pkg.speigs
    out = []
    for L in (lib, ref_lib):
        o = s.default_opts(L, tol=1e-10, detect=0, dense_max=0)
        out.append(s.speigs(A, k, which, o, vectors=True, lib=L))
    return out


@pytest.mark.parametrize("which", [0, 1])
def test_repeated_eigenvalues_breakdown(pkg, lib, ref_lib, which):
    n = 2000
    d = np.repeat([1.0, 2.0, 3.0, 4.0], n // 4)
    A = sp.diags(d).tocsc()
    (rc, lam, V, res, info), (rr, rlam, rV, rres, rinfo) = _both(pkg, lib, ref_lib, A, 3, which)
    assert rc == 0 and rr == 0
    want = 1.0 if which == 0 else 4.0
    assert np.max(np.abs(lam - want)) <= 1e-12
    assert np.max(np.abs(lam - rlam)) <= 1e-12
    assert info["flag"] == rinfo["flag"] == 0
    assert info["nops"] == rinfo["nops"]
    assert info["restarts"] == rinfo["restarts"]
    r = np.linalg.norm(A @ V - V * lam, axis=0)
    assert r.max() <= 1e-10 * info["anorm"]


@pytest.mark.parametrize("which", [0, 1])
def test_space_exhausted(pkg, lib, ref_lib, which):
    n = 16
    A = sp.diags([-np.ones(n - 1), 2.0 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsc()
    (rc, lam, V, res, info), (rr, rlam, rV, rres, rinfo) = _both(pkg, lib, ref_lib, A, 2, which)
    assert rc == 0 and rr == 0
    ex = 2.0 - 2.0 * np.cos(np.arange(1, n + 1) * np.pi / (n + 1))
    ex = ex[:2] if which == 0 else ex[::-1][:2]
    assert np.max(np.abs(lam - ex) / ex) <= 1e-12
    assert np.max(np.abs(lam - rlam) / np.abs(rlam)) <= 1e-12
    assert info["flag"] == rinfo["flag"] == 0
    assert info["nops"] == rinfo["nops"]
