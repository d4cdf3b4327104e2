"""The trained warm-start network on a held-out operator of its family
(48^3, conductivity exp(GRF), seed outside the training range): what its
proposal captures of the wanted eigenvectors, against the closed-form
Laplace modes it reads as input, and what it changes in the solve."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _captured(Y, U):
    Q, _ = np.linalg.qr(Y)
    return float(np.sum((Q.T @ U) ** 2) / U.shape[1])


def test_trained_network_on_held_out_operator(lib, pkg):
    L, s, w = pkg.learned, pkg.speigs, pkg.workloads
    if not os.path.exists(L.CHECKPOINT):
        pytest.skip("no trained checkpoint")
    N, k, seed = 48, 16, 3300
    kap = w.grf_conductivity(N, seed)
    A = w.FVPattern(N).matrix(kap)
    o = s.default_opts(lib, tol=1e-10)
    rc, lam, U, res, info, _ = s.speigs_ex(A, k, s.SM, o, lib=lib)
    assert rc == 0 and info["flag"] == 0
    net = L.WarmStartNet.load(L.CHECKPOINT, lib=lib)
    Y = L.propose(net, N, kap)
    got = _captured(Y, U)
    base = _captured(w.laplace_modes(N, Y.shape[1]), U)
    print(f"share of the 16 eigenvectors in span: learned {got:.3f}, Laplace modes {base:.3f}")
    assert got > 0.6 and got > base + 0.05
    rc2, lam2, V2, res2, info2, ei2 = s.speigs_ex(A, k, s.SM, o, lib=lib, warm=Y)
    assert rc2 == 0 and info2["flag"] == 0 and ei2["warm_cols"] == Y.shape[1]
    assert np.max(np.abs(lam2 - lam) / np.abs(lam)) <= 1e-10
    r = np.linalg.norm(A @ V2 - V2 * lam2, axis=0)
    assert r.max() <= 1e-10 * info2["anorm"] * 1.0001
    print(f"operator applications: random start {info['nops']}, learned start {info2['nops']}")
    assert info2["nops"] <= info["nops"] + 12
