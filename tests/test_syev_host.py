"""The host solver of the Lanczos loops' projected eigenproblem
(speigs_b200_syev_small_host, the reference's LAPACK dsyev("V", "U") at
src/speigs_core.c:180, :236): eigenvalues against numpy's LAPACK to a few
ulps of ||H||, residuals and orthogonality of the vectors, the ordering
contract (theta ascending, ord by |theta| descending, ties in ascending
order), the upper triangle as the only input, and degenerate spectra --
multiple eigenvalues, a diagonal matrix, the zero matrix, order 1 and 2, and
the arrowhead form of a thick-restarted Lanczos matrix.  No GPU needed."""
import ctypes

import numpy as np
import pytest

DP = ctypes.POINTER(ctypes.c_double)
IP = ctypes.POINTER(ctypes.c_int)
EPS = np.finfo(float).eps


def syev_host(lib, H, ldh=None):
    m = H.shape[0]
    ldh = ldh or m
    Hb = np.zeros((m, ldh))                  # row c of Hb = column c of H, ld = ldh
    Hb[:, :m] = H.T
    th = np.zeros(m)
    S = np.zeros((m, m))                      # row c = eigenvector c
    od = np.zeros(m, dtype=np.int32)
    rc = lib.speigs_b200_syev_small_host(m, Hb.ctypes.data_as(DP), ldh, th.ctypes.data_as(DP),
                                         S.ctypes.data_as(DP), od.ctypes.data_as(IP))
    return rc, th, S.T.copy(), od


def check(H, th, S, od):
    m = H.shape[0]
    scale = max(np.abs(np.linalg.eigvalsh(H)).max(), 1e-300)
    ev = np.linalg.eigvalsh(H)
    assert np.max(np.abs(th - ev)) <= 64 * m * EPS * scale
    assert np.all(np.diff(th) >= 0)
    assert np.max(np.abs(H @ S - S * th)) <= 64 * m * EPS * scale
    assert np.max(np.abs(S.T @ S - np.eye(m))) <= 64 * m * EPS
    assert np.array_equal(od, np.argsort(-np.abs(th), kind="stable"))


@pytest.mark.parametrize("m", [1, 2, 3, 8, 33, 61, 93, 128, 200])
def test_random_symmetric(lib, m):
    rng = np.random.default_rng(m)
    A = rng.standard_normal((m, m))
    H = A + A.T
    rc, th, S, od = syev_host(lib, H)
    assert rc == 0
    check(H, th, S, od)


def test_reads_upper_triangle_only(lib):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((40, 40))
    H = A + A.T
    junk = np.triu(H) + np.tril(rng.standard_normal((40, 40)), -1) * 1e6
    rc, th, S, od = syev_host(lib, junk, ldh=47)
    assert rc == 0
    check(H, th, S, od)


def test_multiple_eigenvalues(lib):
    rng = np.random.default_rng(9)
    Q, _ = np.linalg.qr(rng.standard_normal((30, 30)))
    lam = np.repeat([1.0, 2.0, 2.0 + 1e-14, 5.0, -5.0], 6)
    H = (Q * lam) @ Q.T
    H = 0.5 * (H + H.T)
    rc, th, S, od = syev_host(lib, H)
    assert rc == 0
    check(H, th, S, od)


@pytest.mark.parametrize("kind", ["zero", "diagonal", "identity"])
def test_trivial(lib, kind):
    m = 17
    H = {"zero": np.zeros((m, m)), "identity": np.eye(m),
         "diagonal": np.diag(np.arange(m, 0, -1.0) * (-1.0) ** np.arange(m))}[kind]
    rc, th, S, od = syev_host(lib, H)
    assert rc == 0
    assert np.array_equal(th, np.sort(np.diag(H)))
    assert np.max(np.abs(H @ S - S * th)) == 0.0
    assert np.array_equal(od, np.argsort(-np.abs(th), kind="stable"))


def test_thick_restart_arrowhead(lib):
    """The projected matrix after a thick restart: the l kept Ritz values on
    the diagonal, their couplings to the next Lanczos vector in one row and
    column, then a tridiagonal tail."""
    rng = np.random.default_rng(3)
    m, l = 33, 21
    H = np.zeros((m, m))
    H[np.arange(l), np.arange(l)] = np.sort(rng.uniform(1, 100, l))[::-1]
    H[l, :l] = H[:l, l] = rng.standard_normal(l) * 1e-6
    d = rng.uniform(0, 1, m - l)
    e = rng.uniform(0.1, 1, m - l - 1)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    H[l:, l:] = T
    rc, th, S, od = syev_host(lib, H)
    assert rc == 0
    check(H, th, S, od)


def test_bad_arguments(lib):
    H = np.eye(3)
    th, S, od = np.zeros(3), np.zeros(9), np.zeros(3, dtype=np.int32)
    f = lib.speigs_b200_syev_small_host
    assert f(0, H.ctypes.data_as(DP), 3, th.ctypes.data_as(DP), S.ctypes.data_as(DP),
             od.ctypes.data_as(IP)) == -1
    assert f(3, H.ctypes.data_as(DP), 2, th.ctypes.data_as(DP), S.ctypes.data_as(DP),
             od.ctypes.data_as(IP)) == -1


def syev_select(lib, H, nvec, ldh=None):
    m = H.shape[0]
    ldh = ldh or m
    Hb = np.zeros((m, ldh))
    Hb[:, :m] = H.T
    th = np.zeros(m)
    S = np.full((m, m), np.nan)
    od = np.zeros(m, dtype=np.int32)
    rc = lib.speigs_b200_syev_select_host(m, Hb.ctypes.data_as(DP), ldh, nvec,
                                          th.ctypes.data_as(DP), S.ctypes.data_as(DP),
                                          od.ctypes.data_as(IP))
    return rc, th, S.T.copy(), od


def check_select(lib, H, nvec):
    """Eigenvalues within a few ulps of ||H|| of the full solver's (both
    ascending), the order by |theta| descending; the selected vectors are
    eigenvectors to a few ulps of ||H|| and orthonormal; every other column
    is zero."""
    m = H.shape[0]
    rc0, th0, S0, od0 = syev_host(lib, H)
    rc, th, S, od = syev_select(lib, H, nvec)
    assert rc == 0 and rc0 == 0
    scale = max(np.abs(th).max(), 1e-300)
    assert np.max(np.abs(th - th0)) <= 16 * m * EPS * scale
    assert np.all(np.diff(th) >= 0)
    assert np.array_equal(od, np.argsort(-np.abs(th), kind="stable"))
    sel = od[:nvec]
    Ss = S[:, sel]
    if nvec:
        assert np.max(np.abs(H @ Ss - Ss * th[sel])) <= 64 * m * EPS * scale
        assert np.max(np.abs(Ss.T @ Ss - np.eye(nvec))) <= 64 * m * EPS
    rest = np.setdiff1d(np.arange(m), sel)
    assert np.all(S[:, rest] == 0.0)
    return S


@pytest.mark.parametrize("m,nvec", [(2, 1), (3, 2), (33, 21), (96, 21), (128, 40), (61, 0)])
def test_select_random_symmetric(lib, m, nvec):
    rng = np.random.default_rng(100 + m)
    A = rng.standard_normal((m, m))
    check_select(lib, A + A.T, nvec)


def test_select_multiple_and_clustered_eigenvalues(lib):
    """Exact multiplicities (the cube Laplacian's threefold modes), a pair
    1e-14 apart and a tight cluster: inverse iteration with Gram-Schmidt
    inside each cluster still returns an orthonormal eigenbasis."""
    rng = np.random.default_rng(21)
    m = 48
    Q, _ = np.linalg.qr(rng.standard_normal((m, m)))
    lam = np.concatenate([[9.0] * 3, [8.0, 8.0 + 1e-14], 7.0 + 1e-9 * np.arange(4),
                          rng.uniform(-1, 1, m - 9)])
    H = (Q * lam) @ Q.T
    check_select(lib, 0.5 * (H + H.T), 12)


def test_select_thick_restart_arrowhead(lib):
    rng = np.random.default_rng(4)
    m, l = 96, 21
    H = np.zeros((m, m))
    H[np.arange(l), np.arange(l)] = np.sort(rng.uniform(1, 100, l))[::-1]
    H[l, :l] = H[:l, l] = rng.standard_normal(l) * 1e-6
    d = rng.uniform(0, 1, m - l)
    e = rng.uniform(0.1, 1, m - l - 1)
    H[l:, l:] = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    check_select(lib, H, l)


def test_select_full_width_is_the_full_solver(lib):
    rng = np.random.default_rng(8)
    A = rng.standard_normal((20, 20))
    H = A + A.T
    _, th0, S0, od0 = syev_host(lib, H)
    rc, th, S, od = syev_select(lib, H, 20)
    assert rc == 0 and np.array_equal(th, th0) and np.array_equal(S, S0)


def test_select_bad_arguments(lib):
    H = np.eye(3)
    th, S, od = np.zeros(3), np.zeros(9), np.zeros(3, dtype=np.int32)
    f = lib.speigs_b200_syev_select_host
    args = (th.ctypes.data_as(DP), S.ctypes.data_as(DP), od.ctypes.data_as(IP))
    assert f(3, H.ctypes.data_as(DP), 3, -1, *args) == -1
    assert f(3, H.ctypes.data_as(DP), 2, 1, *args) == -1
