"""The allocation-free eigensolver entry point agrees with the allocating one.

speigs_b200_syev_small_noalloc serves callers that cannot call cudaMalloc
where they need the projected eigenproblem solved (code under CUDA stream
capture, real-time loops, hosts whose device memory belongs to another
allocator); its workspace is an array compiled into the library and shared
by every call.  Checked through the C ABI against speigs_b200_syev_small on
two calls in a row, so a call that finds the previous call's leftovers in the
shared workspace is covered.  This file sorts last so that a run stopping at
the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, H, stream, with_status=True):
    m = H.shape[0]
    dH = torch.tensor(np.asfortranarray(H).ravel(order="F"), dtype=torch.float64, device="cuda")
    th = torch.empty(m, dtype=torch.float64, device="cuda")
    S = torch.empty(m * m, dtype=torch.float64, device="cuda")
    od = torch.empty(m, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.speigs_b200_syev_small_noalloc(m, dH.data_ptr(), th.data_ptr(), S.data_ptr(),
                                            od.data_ptr(), st.data_ptr() if with_status else None,
                                            stream)
    assert rc == 0
    torch.cuda.synchronize()
    return (th.cpu().numpy(), S.cpu().numpy().reshape(m, m, order="F"), od.cpu().numpy(),
            int(st.item()) if with_status else 1)


@pytest.mark.parametrize("m", [20, 41, 130, 256])
def test_noalloc_matches_allocating_entry_point(lib, pkg, m):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(100 + m)
    for call in range(2):
        B = rng.standard_normal((m, m))
        H = np.triu(B + B.T) * (1.0 + call)
        th0, S0, od0 = pkg.speigs.syev_small(H, lib)
        # the second call leaves the status to the library's own shared word
        th1, S1, od1, sweeps = _noalloc(lib, torch, H, stream, with_status=(call == 0))
        assert sweeps > 0
        scale = np.abs(th0).max()
        assert np.allclose(th1, th0, rtol=0, atol=1e-13 * scale)
        assert np.array_equal(od1, od0)
        # eigenvectors agree up to sign
        dots = np.abs(np.sum(S0 * S1, axis=0))
        assert np.all(dots > 1 - 1e-10)
        assert np.allclose(S1.T @ S1, np.eye(m), atol=1e-13)


def test_noalloc_rejects_oversized(lib, pkg):
    rc = lib.speigs_b200_syev_small_noalloc(257, 1, 1, 1, 1, None, None)
    assert rc == pkg.speigs.ERR_ARG
    assert "257" in pkg.speigs.last_error(lib)
    rc = lib.speigs_b200_syev_small_noalloc(0, 1, 1, 1, 1, None, None)
    assert rc == pkg.speigs.ERR_ARG
