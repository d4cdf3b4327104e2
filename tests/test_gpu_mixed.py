"""Mixed precision (FP32 factor on the TF32 tensor cores + FP64 refinement of
every solve) against the plain FP64 path and the CPU reference.

The refined operator must agree with an FP64 solve to the refinement target,
and the eigenpairs with the FP64 path's to 1e-10 relative, every pair meeting
||Av - lambda v|| <= 1e-10 ||A||_1 (the per-eigenpair error is the quantity
the mixed-precision form reports).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed_plan(pkg, lib, A, **kw):
    s = pkg.speigs
    ext = s.ext_opts(lib, precision=s.MIXED, **kw)
    return pkg.Plan(A, which=s.SM, lib=lib, ext=ext)


@pytest.mark.parametrize("case", ["lap16", "var16", "lap40", "dense333"])
def test_mixed_operator_matches_fp64_solve(lib, pkg, case):
    torch = pytest.importorskip("torch")
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    w = pkg.workloads
    if case == "dense333":
        rng = np.random.default_rng(5)
        B = rng.standard_normal((333, 333))
        A = sp.csc_matrix(B @ B.T / 333 + np.eye(333))
    else:
        A = {"lap16": lambda: w.lap3d(16), "var16": lambda: w.varcoef3d(16, seed=16),
             "lap40": lambda: w.lap3d(40)}[case]()
    P = _mixed_plan(pkg, lib, A)
    rc, shift = P.factor()
    assert rc == 0 and shift == 0.0
    b = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    assert P.apply_device(b.data_ptr(), x.data_ptr()) == 0
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    # backward error at the FP64 level after refinement
    r = bh - A @ xh
    anorm = abs(A).sum(axis=0).max()
    assert np.linalg.norm(r) <= 1e-13 * (anorm * np.linalg.norm(xh) + np.linalg.norm(bh))
    ref = spla.spsolve(A.tocsc(), bh) if A.shape[0] > 400 else np.linalg.solve(A.toarray(), bh)
    assert np.linalg.norm(xh - ref) / np.linalg.norm(ref) < 1e-10
    P.close()


@pytest.mark.parametrize("case", ["lap20", "var24"])
def test_mixed_eigenpairs_match_fp64(lib, pkg, case):
    w = pkg.workloads
    s = pkg.speigs
    A, k = {"lap20": (w.lap3d(20), 6), "var24": (w.varcoef3d(24, seed=3), 8)}[case]
    o = s.default_opts(lib, tol=1e-10)
    rc0, lam0, V0, res0, info0 = s.speigs(A, k, s.SM, o, lib=lib)
    rc1, lam1, V1, res1, info1, e1 = s.speigs_ex(A, k, s.SM, o, s.ext_opts(lib, precision=s.MIXED),
                                                 lib=lib)
    assert rc0 == 0 and rc1 == 0
    assert e1["precision"] == s.MIXED and e1["refine_steps"] > 0
    assert info1["flag"] == 0 and info1["path"] == s.PATH_SHIFTINV
    rel = np.abs(lam1 - lam0) / np.abs(lam0)
    assert rel.max() <= 1e-10, rel
    anorm = info1["anorm"]
    r = np.linalg.norm(A @ V1 - V1 * lam1, axis=0)
    assert r.max() <= 1e-10 * anorm * 1.0001
    if case == "lap20":
        ex = w.spectrum3d(20)[:k]
        assert np.max(np.abs(lam1 - ex) / ex) <= 1e-10


def test_mixed_singular_takes_shift(lib, pkg):
    """Neumann Laplacian: the FP32 factor also meets the zero pivot and the
    capped shift escalation applies."""
    A = pkg.workloads.lap3d(10, dirichlet=False)
    P = _mixed_plan(pkg, lib, A)
    rc, shift = P.factor()
    assert rc == 0 and shift > 0.0
    P.close()


@pytest.mark.parametrize("case", ["lap40", "var24", "dense333"])
def test_fp32_factor_is_fp32_accurate(lib, pkg, case):
    """One solve with the FP32 factor alone (refine_tol = 1 accepts it
    without a correction): its backward error is at the FP32 level.  The
    trailing updates take three TF32 products (hi.hi + hi.lo + lo.hi) on the
    tensor cores; with the head alone the factor would carry TF32 errors
    (~1e-3), far above this bound."""
    torch = pytest.importorskip("torch")
    import scipy.sparse as sp
    w = pkg.workloads
    if case == "dense333":
        rng = np.random.default_rng(7)
        B = rng.standard_normal((333, 333))
        A = sp.csc_matrix(B @ B.T / 333 + np.eye(333))
    else:
        A = {"lap40": lambda: w.lap3d(40), "var24": lambda: w.varcoef3d(24, seed=24)}[case]()
    P = _mixed_plan(pkg, lib, A, refine_tol=1.0)
    rc, shift = P.factor()
    assert rc == 0 and shift == 0.0
    b = torch.randn(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    assert P.apply_device(b.data_ptr(), x.data_ptr()) == 0
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    anorm = abs(A).sum(axis=0).max()
    be = np.linalg.norm(bh - A @ xh) / (anorm * np.linalg.norm(xh) + np.linalg.norm(bh))
    assert be < 1e-5, be
    P.close()
