"""Batched components: k eigenpairs of every connected component
(speigs_batched), checked per component against a dense CPU eigensolver; the
components on the Krylov route go through the segmented lockstep Lanczos, and
a forest that needs a shift falls back to one solve per component.  The
drop-in blocks route (components solved concurrently, one per host thread)
is checked against the compiled reference."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def test_batched_per_component_eigenpairs(lib, pkg):
    s, w = pkg.speigs, pkg.workloads
    A = w.rgg_blocks(10, seed=7, nmin=50, nmax=900)      # + isolated vertices
    k = 4
    ncomp, comp = s.components(A, lib)
    assert ncomp >= 10
    o = s.default_opts(lib, tol=1e-10)
    rc, lam, V, res, nv, info = s.speigs_batched(A, k, s.SM, o, comp=comp, vectors=True, lib=lib)
    assert rc == 0, (rc, s.last_error(lib))
    assert info["ncomp"] == ncomp and info["flag"] == 0
    Ad = A.tocsr()
    for c in range(ncomp):
        rows = np.flatnonzero(comp == c)
        kc = min(k, len(rows))
        assert nv[c] == kc
        Ac = Ad[rows][:, rows].toarray()
        ex = np.sort(np.linalg.eigvalsh(Ac))[:kc]
        got = lam[c, :kc]
        assert np.all(np.abs(got - ex) <= 1e-10 * np.maximum(np.abs(ex), 1e-3)), (c, got, ex)
        assert np.all(lam[c, kc:] == 0.0)
        Vc = V[rows][:, :kc]
        r = np.linalg.norm(Ac @ Vc - Vc * got, axis=0)
        anorm = np.abs(Ac).sum(axis=0).max()
        assert r.max() <= 1e-10 * max(anorm, 1.0) * 1.0001
        # V's column t holds the t-th eigenvector of every component on that
        # component's rows, so a component's vectors cannot be told apart from
        # its neighbours' in V; what a leak would break is checked instead:
        # the residual above uses only this component's rows, and columns past
        # its own min(k, n_c) are zero on them
        assert np.all(V[rows][:, kc:] == 0.0)


def test_blocks_route_matches_reference(lib, pkg, ref_lib):
    s, w = pkg.speigs, pkg.workloads
    A = w.rgg_blocks(6, seed=11, nmin=200, nmax=1500)
    k = 6
    o = s.default_opts(lib, tol=1e-10)
    rc, lam, V, res, info = s.speigs(A, k, s.SM, o, lib=lib)
    rr, rlam, rV, rres, rinfo = s.speigs(A, k, s.SM, s.default_opts(ref_lib, tol=1e-10), lib=ref_lib)
    assert rc == 0 and rr == 0
    assert info["path"] == rinfo["path"] == s.PATH_BLOCKS and info["ncomp"] == rinfo["ncomp"]
    # 1e-12 relative, down to the rounding floor of a Rayleigh quotient
    # (16 eps ||A||_1): these blocks' smallest eigenvalue is 1e-3, a
    # thousandth of their norm
    floor = 16 * np.finfo(float).eps * max(info["anorm"], rinfo["anorm"], 1.0)
    assert np.all(np.abs(lam - rlam) <= 1e-12 * np.abs(rlam) + floor)
    r = np.linalg.norm(A @ V - V * lam, axis=0)
    assert r.max() <= 1e-10 * max(info["anorm"], rinfo["anorm"], 1.0) * 1.0001
    # each merged eigenvector lives on one component's rows
    ncomp, comp = s.components(A, lib)
    for t in range(k):
        on = np.unique(comp[np.abs(V[:, t]) > 0])
        assert len(on) == 1, (t, on)


def test_batched_rejects_bad_labels(lib, pkg):
    s, w = pkg.speigs, pkg.workloads
    A = w.rgg_blocks(2, seed=3, nmin=50, nmax=80)
    n = A.shape[0]
    comp = np.zeros(n, dtype=np.int64)
    comp[0] = 5      # a label past ncomp - 1 leaves components empty
    rc, *_ = s.speigs_batched(A, 2, s.SM, comp=comp, lib=lib)
    assert rc == s.ERR_ARG


def test_batched_singular_component_falls_back(lib, pkg):
    """A singular PSD component (a Neumann Laplacian) needs its own shift, as
    in the reference's per-component call: the answer is the per-component
    one, zero eigenvalue included."""
    s, w = pkg.speigs, pkg.workloads
    A1, A2 = w.lap3d(7, dirichlet=False), w.lap3d(6)
    A = w.block_diag(A1, A2)
    k = 4
    o = s.default_opts(lib, tol=1e-10)
    rc, lam, V, res, nv, info = s.speigs_batched(A, k, s.SM, o, vectors=True, lib=lib)
    assert rc == 0 and info["flag"] == 0 and info["ncomp"] == 2
    ex1 = w.spectrum3d(7, dirichlet=False)[:k]
    ex2 = w.spectrum3d(6)[:k]
    assert abs(lam[0, 0]) <= 1e-9
    assert np.all(np.abs(lam[0, 1:] - ex1[1:]) <= 1e-9 * ex1[1:])
    assert np.all(np.abs(lam[1] - ex2) <= 1e-12 * ex2)


def test_batched_matches_one_call_per_component(lib, pkg):
    """The segmented lockstep Lanczos against the per-component drop-in
    (speigs() on each component alone): the same eigenvalues to 1e-12 and
    the residual bound on every component."""
    s, w = pkg.speigs, pkg.workloads
    A = w.rgg_blocks(4096, seed=4, first=24)
    k = 4
    o = s.default_opts(lib, tol=1e-10)
    ncomp, comp = s.components(A, lib)
    rc, lam, V, res, nv, info = s.speigs_batched(A, k, s.SM, o, comp=comp, vectors=True, lib=lib)
    assert rc == 0 and info["flag"] == 0
    Ad = A.tocsr()
    for c in range(ncomp):
        rows = np.flatnonzero(comp == c)
        if len(rows) <= 64:
            continue
        Ac = Ad[rows][:, rows].tocsc()
        r1, l1, V1, re1, i1 = s.speigs(Ac, k, s.SM, o, lib=lib)
        assert r1 == 0
        floor = 16 * np.finfo(float).eps * max(i1["anorm"], 1.0)
        assert np.all(np.abs(lam[c] - l1) <= 1e-12 * np.abs(l1) + floor)
        Vc = V[rows][:, :k]
        r = np.linalg.norm(Ac @ Vc - Vc * lam[c], axis=0)
        assert r.max() <= 1e-10 * max(i1["anorm"], 1.0) * 1.0001


def test_batched_straggler_handed_off(lib, pkg):
    """A forest of quickly converging components plus one slow one (a path
    graph Laplacian + 1e-3 I, whose smallest eigenvalues are clustered to
    1e-6 of each other): once the live components hold at most 1/8 of the
    rows, the lockstep loop hands the straggler to the per-component
    executor.  Every component must still agree with speigs() on it alone."""
    s, w = pkg.speigs, pkg.workloads
    n1 = 1500
    path = sp.diags([-np.ones(n1 - 1), 2.0 * np.ones(n1) + 1e-3, -np.ones(n1 - 1)], [-1, 0, 1])
    path = sp.csc_matrix(path)
    path[0, 0] -= 1.0
    path[n1 - 1, n1 - 1] -= 1.0
    quick = w.rgg_blocks(4096, seed=4, first=40)
    A = sp.block_diag([quick, path], format="csc")
    A.sort_indices()
    k = 4
    o = s.default_opts(lib, tol=1e-10)
    ncomp, comp = s.components(A, lib)
    assert np.sum(comp == comp[-1]) * 8 <= A.shape[0]
    rc, lam, V, res, nv, info = s.speigs_batched(A, k, s.SM, o, comp=comp, vectors=True, lib=lib)
    assert rc == 0
    Ad = A.tocsr()
    for c in range(ncomp):
        rows = np.flatnonzero(comp == c)
        if len(rows) <= 64:
            continue
        Ac = Ad[rows][:, rows].tocsc()
        r1, l1, V1, re1, i1 = s.speigs(Ac, k, s.SM, o, lib=lib)
        assert r1 == 0
        floor = 16 * np.finfo(float).eps * max(i1["anorm"], 1.0)
        assert np.all(np.abs(lam[c] - l1) <= 1e-12 * np.abs(l1) + floor), c
        Vc = V[rows][:, :k]
        r = np.linalg.norm(Ac @ Vc - Vc * lam[c], axis=0)
        if i1["flag"] == 0:
            assert r.max() <= 1e-10 * max(i1["anorm"], 1.0) * 1.0001
