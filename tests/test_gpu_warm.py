"""Start subspace for the thick-restart Lanczos (speigs_ext_opts.warm), in
both of its uses: as the first block of the block method (block = 0, the
default with a start subspace) and folded into the single-vector method's
start vector (block = -1: the normalised sum of an orthonormal basis of the
subspace plus a small share of the reference's random start).  The answer
must not depend on the start (same eigenpairs as the random start, residual
bound met); a start that already contains the wanted eigenvectors must need
far fewer operator applications."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(pkg, lib, A, k, warm=None, mixed=False, block=0):
    s = pkg.speigs
    o = s.default_opts(lib, tol=1e-10)
    e = s.ext_opts(lib, precision=s.MIXED if mixed else s.FP64, block=block)
    return s.speigs_ex(A, k, s.SM, o, e, lib=lib, warm=warm)


@pytest.mark.parametrize("block", [0, -1])
def test_exact_subspace_converges_at_once(lib, pkg, block):
    A = pkg.workloads.varcoef3d(20, seed=9)
    k = 8
    rc, lam, V, res, info, ei = _solve(pkg, lib, A, k)
    assert rc == 0 and info["flag"] == 0 and ei["warm_cols"] == 0
    rng = np.random.default_rng(1)
    Y = V + 1e-9 * rng.standard_normal(V.shape)
    rc2, lam2, V2, res2, info2, ei2 = _solve(pkg, lib, A, k, warm=Y, block=block)
    assert ei2["block"] == (k if block == 0 else 0)
    assert rc2 == 0 and info2["flag"] == 0
    assert ei2["warm_cols"] == k
    assert info2["restarts"] <= 1
    assert info2["nops"] < info["nops"]
    assert np.max(np.abs(lam2 - lam) / np.abs(lam)) <= 1e-10
    r = np.linalg.norm(A @ V2 - V2 * lam2, axis=0)
    assert r.max() <= 1e-10 * info2["anorm"] * 1.0001


@pytest.mark.parametrize("mixed,block", [(False, 0), (True, 0), (False, -1), (True, -1)])
def test_laplace_mode_start_same_answer(lib, pkg, mixed, block):
    N, k = 16, 8
    w = pkg.workloads
    A = w.grf3d(N, seed=1001)
    rc, lam, V, res, info, _ = _solve(pkg, lib, A, k, mixed=mixed)
    Y = w.laplace_modes(N, k + 6)
    rc2, lam2, V2, res2, info2, ei2 = _solve(pkg, lib, A, k, warm=Y, mixed=mixed, block=block)
    assert rc == 0 and rc2 == 0 and info2["flag"] == 0
    assert ei2["warm_cols"] == k + 6
    assert np.max(np.abs(lam2 - lam) / np.abs(lam)) <= 1e-10
    r = np.linalg.norm(A @ V2 - V2 * lam2, axis=0)
    assert r.max() <= 1e-10 * info2["anorm"] * 1.0001


@pytest.mark.parametrize("block", [0, -1])
def test_dependent_columns_are_dropped(lib, pkg, block):
    A = pkg.workloads.lap3d(12)
    k = 4
    Y = pkg.workloads.laplace_modes(12, 6)
    Y = np.concatenate([Y, Y[:, :2] * 3.0, np.zeros((A.shape[0], 1))], axis=1)
    rc, lam, V, res, info, ei = _solve(pkg, lib, A, k, warm=Y, block=block)
    assert rc == 0 and info["flag"] == 0
    assert ei["warm_cols"] == 6
    ex = pkg.workloads.spectrum3d(12)[:k]
    assert np.max(np.abs(lam - ex) / ex) <= 1e-10


def test_wide_start_subspace_reduced_to_its_best_block(lib, pkg):
    """A start subspace wider than the block is reduced to the block's width
    by Rayleigh-Ritz with A: given the 8 wanted eigenvectors hidden among 16
    unwanted ones (the wanted ones last), blocks of 8 start from the wanted
    directions and finish in one restart cycle, where the first 8 columns
    alone would start from unwanted ones."""
    A = pkg.workloads.varcoef3d(20, seed=9)
    k = 8
    rc, lam, V, res, info, ei = _solve(pkg, lib, A, 24)
    assert rc == 0 and info["flag"] == 0
    order = np.argsort(np.abs(lam))
    rng = np.random.default_rng(3)
    Y = V[:, order[::-1]] + 1e-9 * rng.standard_normal(V.shape)      # wanted columns last
    rc0, lam0, *_ = _solve(pkg, lib, A, k)
    rc2, lam2, V2, res2, info2, ei2 = _solve(pkg, lib, A, k, warm=Y, block=8)
    assert rc0 == 0 and rc2 == 0 and info2["flag"] == 0
    assert ei2["block"] == 8 and ei2["warm_cols"] == 8
    assert info2["restarts"] <= 1
    assert np.max(np.abs(lam2 - lam0) / np.abs(lam0)) <= 1e-10
    r = np.linalg.norm(A @ V2 - V2 * lam2, axis=0)
    assert r.max() <= 1e-10 * info2["anorm"] * 1.0001


def test_device_subspace_equals_host_subspace(lib, pkg):
    """speigs_ext_opts.warm may point to device memory (a proposal computed
    on the GPU): the eigenpairs are bit for bit those of the same subspace
    given from host memory, and its bytes are not counted as host-to-device
    traffic."""
    torch = pytest.importorskip("torch")
    s = pkg.speigs
    A = pkg.workloads.varcoef3d(18, seed=4)
    n, k, p = A.shape[0], 6, 8
    rng = np.random.default_rng(3)
    Y = np.asfortranarray(rng.standard_normal((n, p)))
    o = s.default_opts(lib, tol=1e-10)
    c0 = s.counters(lib)
    rc, lam, V, res, info, ei = s.speigs_ex(A, k, s.SM, o, s.ext_opts(lib, block=8), lib=lib,
                                            warm=Y)
    c1 = s.counters(lib)
    Yd = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()      # (p, n): column-major n x p
    torch.cuda.synchronize()
    e = s.ext_opts(lib, block=8)
    e.warm = Yd.data_ptr()
    e.warm_cols = p
    rc2, lam2, V2, res2, info2, ei2 = s.speigs_ex(A, k, s.SM, o, e, lib=lib)
    c2 = s.counters(lib)
    assert rc == 0 and rc2 == 0 and ei2["warm_cols"] == ei["warm_cols"] == p
    assert np.array_equal(lam, lam2) and np.array_equal(V, V2)
    assert (c1[1] - c0[1]) - (c2[1] - c1[1]) == Y.nbytes
