"""The FP64 restatement of the warm-start network (oracle/mpnn_oracle.py)
is checked against central finite differences before it is used to check
the device kernels."""
import numpy as np
import scipy.sparse as sp

from conftest import import_package


def _setup(seed=0, N=3, F=5, H=64, L=2, P=4, k=3):
    pkg = import_package()
    rng = np.random.default_rng(seed)
    kap = np.exp(rng.standard_normal((N, N, N)))
    rowptr, col, w = pkg.learned.grid_graph(N, kap)
    n = N ** 3
    A = sp.csr_matrix((w.astype(np.float64), col, rowptr), shape=(n, n))
    X = rng.standard_normal((n, F))
    U, _ = np.linalg.qr(rng.standard_normal((n, k)))
    from mpnn_oracle import layer_shapes
    cnt = sum(o * i + o for o, i in layer_shapes(F, H, L, P))
    params = 0.2 * rng.standard_normal(cnt)
    return A, X, U, params, (F, H, L, P)


def test_adjacency_is_symmetric_normalised():
    pkg = import_package()
    rng = np.random.default_rng(1)
    N = 4
    kap = np.exp(rng.standard_normal((N, N, N)))
    rowptr, col, w = pkg.learned.grid_graph(N, kap)
    A = sp.csr_matrix((w, col, rowptr), shape=(N ** 3,) * 2).toarray()
    assert np.allclose(A, A.T, atol=1e-7)
    # D^{-1/2} T D^{-1/2}: spectral radius 1
    assert abs(np.max(np.abs(np.linalg.eigvalsh(A))) - 1.0) < 1e-5


def test_oracle_gradient_matches_finite_differences(oracle):
    import mpnn_oracle as mo
    A, X, U, params, dims = _setup()
    Y, cache = mo.forward(params, A, X, *dims)
    loss, dY = mo.loss_and_dY(Y, U)
    g = mo.backward(params, A, cache, dY, *dims)
    rng = np.random.default_rng(3)
    idx = rng.choice(params.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        l1 = mo.loss_and_dY(mo.forward(p1, A, X, *dims)[0], U)[0]
        l2 = mo.loss_and_dY(mo.forward(p2, A, X, *dims)[0], U)[0]
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
