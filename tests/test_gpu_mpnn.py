"""Device kernels of the warm-start network (BF16 weights and activations,
FP32 accumulation) against the FP64 oracle: forward output and the
gradient of the subspace loss.  Tolerances reflect BF16 storage."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _device_case(pkg, N=6, seed=0, P=6, k=4, L=4):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(seed)
    kap = np.exp(rng.standard_normal((N, N, N)))
    rowptr, col, w = pkg.learned.grid_graph(N, kap)
    X = pkg.learned.features(N, kap)
    n = N ** 3
    U, _ = np.linalg.qr(rng.standard_normal((n, k)))
    net = pkg.learned.WarmStartNet(nout=P, layers=L, seed=11)
    dev = torch.device("cuda")
    t = {name: torch.from_numpy(np.ascontiguousarray(a)).to(dev) for name, a in
         [("rp", rowptr), ("ci", col), ("w", w), ("X", X), ("U", U.astype(np.float32))]}
    A = sp.csr_matrix((w.astype(np.float64), col, rowptr), shape=(n, n))
    return torch, net, t, A, X.astype(np.float64), U, n, (X.shape[1], 64, L, P), k


def test_forward_matches_oracle(pkg, oracle):
    import mpnn_oracle as mo
    torch, net, t, A, X, U, n, dims, k = _device_case(pkg)
    Y = torch.empty((n, dims[3]), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = net.forward_device(n, t["rp"].data_ptr(), t["ci"].data_ptr(), t["w"].data_ptr(),
                            t["X"].data_ptr(), Y.data_ptr(), 0)
    assert rc == 0
    torch.cuda.synchronize()
    Yd = Y.double().cpu().numpy()
    Yo, _ = mo.forward(net.get_params().astype(np.float64), A, X, *dims)
    err = np.linalg.norm(Yd - Yo) / np.linalg.norm(Yo)
    assert err < 2e-2, err


def test_gradient_matches_oracle(pkg, oracle):
    import mpnn_oracle as mo
    torch, net, t, A, X, U, n, dims, k = _device_case(pkg)
    torch.cuda.synchronize()
    loss_d = net.train_step_device(n, t["rp"].data_ptr(), t["ci"].data_ptr(), t["w"].data_ptr(),
                                   t["X"].data_ptr(), t["U"].data_ptr(), k, 0.0, 0)
    gd = net.grads().astype(np.float64)
    params = net.get_params().astype(np.float64)
    Yo, cache = mo.forward(params, A, X, *dims)
    loss_o, dY = mo.loss_and_dY(Yo, U)
    go = mo.backward(params, A, cache, dY, *dims)
    assert abs(loss_d - loss_o) < 2e-2 * max(abs(loss_o), 1e-3)
    cos = gd @ go / (np.linalg.norm(gd) * np.linalg.norm(go))
    assert cos > 0.995, cos
    assert np.linalg.norm(gd - go) / np.linalg.norm(go) < 0.1


def test_training_reduces_loss(pkg):
    torch, net, t, A, X, U, n, dims, k = _device_case(pkg, N=8, seed=2)
    args = (n, t["rp"].data_ptr(), t["ci"].data_ptr(), t["w"].data_ptr(), t["X"].data_ptr(),
            t["U"].data_ptr(), k)
    first = net.train_step_device(*args, 3e-3, 0)
    for _ in range(60):
        last = net.train_step_device(*args, 3e-3, 0)
    assert last < 0.8 * first, (first, last)


@pytest.mark.parametrize("N,P", [(48, 24), (7, 8), (6, 6)])
def test_tensor_core_layers_match_fma_layers(pkg, N, P):
    """The dense layers on the tensor cores (tcgen05, FP32 accumulation in
    TMEM) against the FP32-FMA kernels on the same BF16 operands: the
    48^3 proposal workload (hidden and output layers on the tensor cores),
    a ragged last tile (343 rows) and an output width the tensor-core
    kernel does not take (6: that layer stays on FMA).  The two differ in
    the order of the FP32 sums only, so BF16 activations agree except for
    an occasional last-bit flip."""
    torch, net, t, A, X, U, n, dims, k = _device_case(pkg, N=N, P=P)
    Y = {}
    for on in (0, 1):
        net.tensor_cores(on)
        Y[on] = torch.empty((n, P), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc = net.forward_device(n, t["rp"].data_ptr(), t["ci"].data_ptr(), t["w"].data_ptr(),
                                t["X"].data_ptr(), Y[on].data_ptr(), 0)
        assert rc == 0
    torch.cuda.synchronize()
    assert net.tensor_cores(-1) == 1
    a, b = Y[1].double().cpu().numpy(), Y[0].double().cpu().numpy()
    assert np.all(np.isfinite(a))
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert err < 1e-2, err


@pytest.mark.parametrize("N", [1, 2, 6, 48])
def test_device_grid_graph_is_host_grid_graph(pkg, N):
    """The network's input graph built on the device from the conductivities
    equals the host construction bit for bit (row pointers, columns and
    FP32 weights), including the smallest grids."""
    torch = pytest.importorskip("torch")
    L = pkg.learned
    rng = np.random.default_rng(N)
    kap = np.exp(rng.standard_normal((N, N, N)))
    rp, ci, w = L.grid_graph(N, kap)
    net = L.WarmStartNet(nout=8, layers=1, seed=3)
    n, nnz = N ** 3, 6 * N * N * (N - 1)
    t_kap = torch.from_numpy(kap.ravel()).cuda()
    t_rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    t_ci = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    t_w = torch.empty(max(nnz, 1), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    assert net.grid_graph_device(N, t_kap.data_ptr(), t_rp.data_ptr(), t_ci.data_ptr(),
                                 t_w.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    assert np.array_equal(t_rp.cpu().numpy(), rp) and rp[-1] == nnz
    assert np.array_equal(t_ci.cpu().numpy()[:nnz], ci)
    assert np.array_equal(t_w.cpu().numpy()[:nnz], w)
