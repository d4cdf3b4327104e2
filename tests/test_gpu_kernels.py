"""Kernel-level parity on the GPU through the C ABI: the start vector, the
projected eigenproblem and the two operators, each against a CPU statement
of the same operation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rand_vec_bit_exact(lib, pkg, oracle):
    """Device xorshift64* with jump-ahead == the sequential stream (:49-54)."""
    for n, seed in [(1, 88172645463325252), (1000, 88172645463325252), (4097, 12345),
                    (100003, 2**63 + 11)]:
        v = pkg.speigs.rand_vec(n, seed, lib)
        m = min(n, 5000)
        _, ref = oracle.rand_vec(seed, m)
        assert np.array_equal(v[:m], ref), f"n={n} seed={seed}"
    # the tail of a long draw: advance the oracle state, then compare
    n = 100003
    v = pkg.speigs.rand_vec(n, 7, lib)
    s = 7
    for _ in range(n - 64):
        s, _ = oracle.rng_next(s)
    _, tail = oracle.rand_vec(s, 64)
    assert np.array_equal(v[-64:], tail)


@pytest.mark.parametrize("m", [2, 3, 20, 41, 64, 101])
def test_syev_small_random(lib, pkg, m):
    rng = np.random.default_rng(m)
    B = rng.standard_normal((m, m))
    H = np.triu(B + B.T)                      # only the upper triangle is read
    th, S, ordv = pkg.speigs.syev_small(H, lib)
    Hs = np.triu(H) + np.triu(H, 1).T
    ref = np.linalg.eigvalsh(Hs)
    assert np.allclose(th, ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    assert np.all(np.diff(th) >= 0)
    assert np.allclose(S.T @ S, np.eye(m), atol=1e-13)
    assert np.allclose(Hs @ S, S * th, atol=1e-12 * np.abs(ref).max())
    key = np.abs(th[ordv])
    assert np.all(np.diff(key) <= 0)
    assert sorted(ordv.tolist()) == list(range(m))


def test_syev_small_graded(lib, pkg):
    """Thick-restart arrowhead with a huge range (shift-invert near a null
    space): small eigenvalues must stay relatively accurate."""
    m = 20
    d = np.concatenate([[8.3e4], np.linspace(1.0, 26.0, m - 1)])
    H = np.diag(d)
    H[:-1, -1] = 1e-3 * np.arange(1, m)
    th, S, _ = pkg.speigs.syev_small(H, lib)
    Hs = np.triu(H) + np.triu(H, 1).T
    ref = np.linalg.eigvalsh(Hs)
    assert np.max(np.abs(th - ref) / np.abs(ref)) < 1e-13


def test_spmv_operator(lib, pkg):
    torch = pytest.importorskip("torch")
    A = pkg.workloads.lap2d(200)
    P = pkg.Plan(A, which=pkg.speigs.LM, lib=lib)
    x = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    assert P.apply_device(x.data_ptr(), y.data_ptr()) == 0
    ref = A @ x.cpu().numpy()
    assert np.allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    P.close()


@pytest.mark.parametrize("N,coef", [(12, False), (20, False), (16, True), (30, True)])
def test_cholesky_solve_operator(lib, pkg, N, coef):
    """(A + shift I)^{-1} b from the device multifrontal factor vs scipy."""
    torch = pytest.importorskip("torch")
    import scipy.sparse.linalg as spla
    A = pkg.workloads.varcoef3d(N, seed=N) if coef else pkg.workloads.lap3d(N)
    P = pkg.Plan(A, which=pkg.speigs.SM, lib=lib)
    rc, shift = P.factor()
    assert rc == 0 and shift == 0.0
    b = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    assert P.apply_device(b.data_ptr(), x.data_ptr()) == 0
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    ref = spla.spsolve(A.tocsc(), bh)
    assert np.linalg.norm(xh - ref) / np.linalg.norm(ref) < 1e-11
    assert np.linalg.norm(A @ xh - bh) / np.linalg.norm(bh) < 1e-12
    P.close()


@pytest.mark.parametrize("n", [65, 333, 1000])
def test_cholesky_solve_dense_front(lib, pkg, n):
    """A dense SPD matrix is one front with n pivots: many 64-column panel
    steps, ragged edge tiles, and the tile-level inversion of L11."""
    torch = pytest.importorskip("torch")
    import scipy.sparse as sp
    rng = np.random.default_rng(n)
    B = rng.standard_normal((n, n))
    Ad = B @ B.T / n + np.eye(n)
    A = sp.csc_matrix(Ad)
    P = pkg.Plan(A, which=pkg.speigs.SM, lib=lib)
    rc, shift = P.factor()
    assert rc == 0 and shift == 0.0
    b = torch.randn(n, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    assert P.apply_device(b.data_ptr(), x.data_ptr()) == 0
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    ref = np.linalg.solve(Ad, bh)
    assert np.linalg.norm(xh - ref) / np.linalg.norm(ref) < 1e-11
    P.close()


def test_cholesky_solve_large_separators(lib, pkg):
    """3-D Laplacian 40^3: separators of ~1,600 columns (25 panel steps)."""
    torch = pytest.importorskip("torch")
    import scipy.sparse.linalg as spla
    A = pkg.workloads.lap3d(40)
    P = pkg.Plan(A, which=pkg.speigs.SM, lib=lib)
    rc, shift = P.factor()
    assert rc == 0 and shift == 0.0
    b = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    assert P.apply_device(b.data_ptr(), x.data_ptr()) == 0
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    assert np.linalg.norm(A @ xh - bh) / np.linalg.norm(bh) < 1e-12
    P.close()


def test_cholesky_not_pd_escalates(lib, pkg):
    """Singular PSD (Neumann) input: the first factorization fails on device,
    the capped escalation finds delta = 1e-6 ||A||_1 (reference :953-970)."""
    A = pkg.workloads.lap3d(10, dirichlet=False)
    P = pkg.Plan(A, which=pkg.speigs.SM, lib=lib)
    rc, shift = P.factor()
    assert rc == 0
    assert shift == pytest.approx(1e-6 * 12.0, rel=1e-12)
    P.close()
