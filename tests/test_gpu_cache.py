"""The opt-in factorization cache (speigs_b200_factor_cache): a repeated
speigs() on the same operator skips the analysis and the factorization and
returns the same eigenpairs bit for bit; a changed value is a different
operator; the least recently used plan is released past capacity; 0 frees
everything."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_factor_cache_reuse_and_eviction(pkg, lib):
    s, w = pkg.speigs, pkg.workloads
    assert lib.speigs_b200_factor_cache(2) == 0
    try:
        A = w.varcoef3d(24, seed=3)
        o = s.default_opts(lib, tol=1e-10)
        rc, lam1, V1, r1, i1 = s.speigs(A, 6, s.SM, o, lib=lib)
        assert rc == 0 and i1["t_factor"] > 0 and lib.speigs_b200_factor_cache_size() == 1
        rc, lam2, V2, r2, i2 = s.speigs(A, 6, s.SM, o, lib=lib)
        assert rc == 0 and i2["t_analyze"] == 0.0
        assert i2["t_factor"] < 0.1 * i1["t_factor"]
        assert np.array_equal(lam1, lam2) and np.array_equal(V1, V2)
        # other Lanczos options on the cached factor
        rc, lam3, V3, r3, i3 = s.speigs(A, 8, s.SM, s.default_opts(lib, tol=1e-12), lib=lib)
        assert rc == 0 and i3["t_analyze"] == 0.0
        assert np.max(np.abs(lam3[:6] - lam1) / lam1) <= 1e-12
        # a changed value is another operator
        B = A.copy()
        B.data = B.data * 2.0
        rc, lamb, *_ = s.speigs(B, 6, s.SM, o, vectors=False, lib=lib)
        assert rc == 0 and np.max(np.abs(lamb - 2 * lam1) / lam1) <= 1e-12
        assert lib.speigs_b200_factor_cache_size() == 2
        C = w.varcoef3d(20, seed=5)
        rc, *_ = s.speigs(C, 4, s.SM, o, vectors=False, lib=lib)
        assert rc == 0 and lib.speigs_b200_factor_cache_size() == 2
        # A was the least recently used: it was released, so it is analysed again
        rc, lam4, _, _, i4 = s.speigs(A, 6, s.SM, o, vectors=False, lib=lib)
        assert rc == 0 and i4["t_analyze"] > 0.0
    finally:
        assert lib.speigs_b200_factor_cache(0) == 0
    assert lib.speigs_b200_factor_cache_size() == 0
