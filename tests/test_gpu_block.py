"""The block path: the multi-right-hand-side shift-invert solve and the block
thick-restart Lanczos built on it (speigs_ext_opts.block).

* A block solve of nr columns equals nr single solves column by column
  (1e-13 relative; the sums are ordered differently) and solves
  (A + shift I) X = B to a small backward error, for every block width the
  kernel has (rows of 8, 16, 24 or 32 doubles, narrower blocks padded) and
  for the FP32 factor with FP64 refinement; buffers sized for a wide block
  serve narrower ones.
* The block Lanczos returns the eigenpairs of the single-vector method
  (1e-12 relative in FP64, 1e-10 for the mixed form) with the residual bound
  met, for several block sizes, and uses every column of an exact start
  subspace.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _plan(pkg, lib, A, mixed=False):
    s = pkg.speigs
    ext = s.ext_opts(lib, precision=s.MIXED if mixed else s.FP64)
    return s.Plan(A, s.SM, s.default_opts(lib, tol=1e-10), lib=lib, ext=ext)


@pytest.mark.parametrize("nr", [1, 5, 8, 13, 16, 24, 32])
def test_block_solve_matches_single_solves(pkg, lib, nr):
    torch = pytest.importorskip("torch")
    A = pkg.workloads.varcoef3d(20, seed=4)
    n = A.shape[0]
    plan = _plan(pkg, lib, A)
    rc, shift = plan.factor()
    assert rc == 0
    ld = n + 7                                   # a leading dimension other than n
    rng = np.random.default_rng(nr)
    Bh = rng.standard_normal((nr, ld))           # column-major n x nr, ld rows per column
    B = torch.tensor(Bh, dtype=torch.float64, device="cuda")
    X = torch.zeros((nr, ld), dtype=torch.float64, device="cuda")
    rc = plan.apply_block_device(B.data_ptr(), ld, X.data_ptr(), ld, nr)
    assert rc == 0, pkg.speigs.last_error(lib)
    Xb = X.cpu().numpy()[:, :n]
    assert np.all(X.cpu().numpy()[:, n:] == 0.0)    # rows past n untouched
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    for c in range(nr):
        x = torch.tensor(Bh[c, :n], dtype=torch.float64, device="cuda")
        assert plan.apply_device(x.data_ptr(), y.data_ptr()) == 0
        ys = y.cpu().numpy()
        assert np.max(np.abs(Xb[c] - ys)) <= 1e-13 * np.max(np.abs(ys)), c
    M = (A + shift * sp.identity(n)).tocsr()
    R = Bh[:, :n].T - M @ Xb.T
    anorm = abs(A).sum(axis=0).max()
    assert np.max(np.linalg.norm(R, axis=0) /
                  (anorm * np.linalg.norm(Xb, axis=1) + np.linalg.norm(Bh[:, :n], axis=1))) <= 1e-14
    plan.close()


def test_block_solve_narrower_after_wider(pkg, lib):
    """Buffers sized for 32 columns serve later solves of 8 and 24 columns
    (each at its own width) with the same results as on a fresh plan."""
    torch = pytest.importorskip("torch")
    A = pkg.workloads.varcoef3d(20, seed=4)
    n = A.shape[0]
    rng = np.random.default_rng(7)
    Bh = rng.standard_normal((32, n))
    B = torch.tensor(Bh, dtype=torch.float64, device="cuda")

    def solve(plan, nr):
        X = torch.zeros((nr, n), dtype=torch.float64, device="cuda")
        assert plan.apply_block_device(B.data_ptr(), n, X.data_ptr(), n, nr) == 0
        return X.cpu().numpy()

    plan = _plan(pkg, lib, A)
    assert plan.factor()[0] == 0
    wide = solve(plan, 32)
    narrow = {nr: solve(plan, nr) for nr in (8, 24, 5)}
    plan.close()
    for nr, Xn in narrow.items():
        fresh = _plan(pkg, lib, A)
        assert fresh.factor()[0] == 0
        assert np.array_equal(Xn, solve(fresh, nr))
        fresh.close()
        assert np.max(np.abs(Xn - wide[:nr])) <= 1e-13 * np.max(np.abs(wide[:nr]))


@pytest.mark.parametrize("nr", [3, 24])
def test_block_solve_mixed_refined(pkg, lib, nr):
    torch = pytest.importorskip("torch")
    A = pkg.workloads.varcoef3d(20, seed=4)
    n = A.shape[0]
    plan = _plan(pkg, lib, A, mixed=True)
    rc, shift = plan.factor()
    assert rc == 0
    rng = np.random.default_rng(100 + nr)
    Bh = rng.standard_normal((nr, n))
    B = torch.tensor(Bh, dtype=torch.float64, device="cuda")
    X = torch.zeros((nr, n), dtype=torch.float64, device="cuda")
    assert plan.apply_block_device(B.data_ptr(), n, X.data_ptr(), n, nr) == 0
    Xb = X.cpu().numpy()
    M = (A + shift * sp.identity(n)).tocsr()
    R = Bh.T - M @ Xb.T
    anorm = abs(A).sum(axis=0).max()
    back = np.linalg.norm(R, axis=0) / (anorm * np.linalg.norm(Xb, axis=1) +
                                         np.linalg.norm(Bh, axis=1))
    assert back.max() <= 1e-14, back.max()
    plan.close()


def _solve(pkg, lib, A, k, block=0, warm=None, mixed=False):
    s = pkg.speigs
    o = s.default_opts(lib, tol=1e-10)
    e = s.ext_opts(lib, precision=s.MIXED if mixed else s.FP64, block=block)
    rc, lam, V, res, info, ei = s.speigs_ex(A, k, s.SM, o, e, lib=lib, warm=warm)
    assert rc == 0, (rc, s.last_error(lib))
    return lam, V, res, info, ei


@pytest.mark.parametrize("block,mixed", [(4, False), (8, False), (16, False), (24, False),
                                         (32, False), (16, True)])
def test_block_lanczos_matches_single_vector(pkg, lib, block, mixed):
    A = pkg.workloads.varcoef3d(24, seed=3)
    k = 8
    lam0, V0, res0, info0, _ = _solve(pkg, lib, A, k, block=-1)
    lam, V, res, info, ei = _solve(pkg, lib, A, k, block=block, mixed=mixed)
    assert info["flag"] == 0 and ei["block"] == block and ei["block_solves"] > 0
    err = np.abs(lam - lam0) / np.abs(lam0)
    print(f"block {block} mixed {mixed}: {info['nops']} vectors in {ei['block_solves']} block "
          f"solves, {info['restarts']} restarts (single vector: {info0['nops']}); err {err.max():.1e}")
    assert err.max() <= (1e-10 if mixed else 1e-12)
    r = np.linalg.norm(A @ V - V * lam, axis=0)
    assert r.max() <= 1e-10 * info["anorm"] * 1.0001
    assert np.max(np.abs(res - r)) <= 1e-9 * info["anorm"]


def test_block_lanczos_exact_start_block(pkg, lib):
    """A start block that spans the wanted eigenvectors converges at the
    first check: one block application."""
    A = pkg.workloads.varcoef3d(20, seed=9)
    k = 8
    lam0, V0, _, info0, _ = _solve(pkg, lib, A, k, block=-1)
    Y = V0 + 1e-12 * np.random.default_rng(2).standard_normal(V0.shape)
    lam, V, res, info, ei = _solve(pkg, lib, A, k, warm=Y)
    assert ei["block"] == k and ei["warm_cols"] == k
    assert info["flag"] == 0 and ei["block_solves"] == 1 and info["nops"] == k
    assert np.max(np.abs(lam - lam0) / np.abs(lam0)) <= 1e-12


def test_block_lanczos_dependent_start_columns(pkg, lib):
    """Dependent and zero start columns are replaced from the random stream."""
    A = pkg.workloads.lap3d(12)
    k = 4
    Y = pkg.workloads.laplace_modes(12, 6)
    Y = np.concatenate([Y, Y[:, :2] * 3.0, np.zeros((A.shape[0], 1))], axis=1)
    lam, V, res, info, ei = _solve(pkg, lib, A, k, warm=Y)
    assert info["flag"] == 0 and ei["block"] == 9 and ei["warm_cols"] == 6
    ex = pkg.workloads.spectrum3d(12)[:k]
    assert np.max(np.abs(lam - ex) / ex) <= 1e-12
