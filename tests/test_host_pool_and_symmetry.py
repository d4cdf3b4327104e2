"""Host logic of the drop-in call that needs no GPU.

* The component worker pool runs its per-thread set-up before any item, which
  is how every worker adopts the caller's CUDA device (a new thread starts on
  device 0).  Checked by a small C++ harness compiled against the pool.
* The symmetry verdict agrees with the reference's check_symmetry
  (src/speigs_core.c:363-401, called through oracle/_ref/libspeigs_probe.so)
  on randomised small inputs, including the unusual layouts the reference's
  transpose comparison decides: repeated row indices, unsorted columns,
  upper-only and lower-only storage, and values off by more or less than
  1e-12 relative.  The verdict is read from speigs(): SPEIGS_ERR_NOTSYM
  exactly when the reference's verdict is 0.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ORACLE_DIR, PKG_DIR

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(ORACLE_DIR, "_ref", "libspeigs_probe.so")


def test_worker_pool_runs_enter_on_every_thread(tmp_path):
    exe = tmp_path / "pool_check"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-pthread",
                           "-I", os.path.join(PKG_DIR, "csrc", "host"),
                           os.path.join(HERE, "host", "pool_check.cpp"), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"


def _variants(rng):
    """Small CSC arrays (n, Ap, Ai, Ax) in the layouts the reference's check decides."""
    out = []
    for t in range(60):
        n = int(rng.integers(3, 14))
        dense = rng.random((n, n)) < 0.35
        M = np.where(dense, rng.standard_normal((n, n)), 0.0)
        S = np.triu(M) + np.triu(M, 1).T
        np.fill_diagonal(S, 1.0 + np.abs(np.diag(S)))
        kind = t % 10
        cols = []
        for c in range(n):
            rows = [r for r in range(n) if S[r, c] != 0.0]
            if kind == 1:
                rows = [r for r in rows if r <= c]                      # upper only
            elif kind == 2:
                rows = [r for r in rows if r >= c]                      # lower only
            cols.append([(r, S[r, c]) for r in rows])
        c = int(rng.integers(0, n))
        offd = [i for i, (r, _) in enumerate(cols[c]) if r != c]
        if kind == 3 and offd:                                          # value off by 1e-10
            i = offd[0]
            cols[c][i] = (cols[c][i][0], cols[c][i][1] * (1 + 1e-10))
        elif kind == 4 and offd:                                        # value off by 1e-14
            i = offd[0]
            cols[c][i] = (cols[c][i][0], cols[c][i][1] * (1 + 1e-14))
        elif kind == 5 and len(cols[c]) >= 2:                           # one column reversed
            cols[c] = cols[c][::-1]
        elif kind == 6 and offd:                                        # mirrored duplicate
            r, v = cols[c][offd[0]]
            cols[c].insert(offd[0], (r, v))
            j = [i for i, (rr, _) in enumerate(cols[r]) if rr == c][0]
            cols[r].insert(j, (c, v))
        elif kind == 7 and offd:                                        # unmirrored duplicate
            r, v = cols[c][offd[0]]
            cols[c].insert(offd[0], (r, v))
        elif kind == 8 and offd:                                        # duplicates, values swapped
            r, v = cols[c][offd[0]]
            cols[c][offd[0]:offd[0] + 1] = [(r, v), (r, 2 * v)]
            j = [i for i, (rr, _) in enumerate(cols[r]) if rr == c][0]
            cols[r][j:j + 1] = [(c, 2 * v), (c, v)]
        elif kind == 9:                                                 # a repeated diagonal
            cols[c].insert([i for i, (r, _) in enumerate(cols[c]) if r >= c][0], (c, 0.5))
        Ap = np.zeros(n + 1, dtype=np.int64)
        Ai, Ax = [], []
        for j in range(n):
            Ai += [r for r, _ in cols[j]]
            Ax += [v for _, v in cols[j]]
            Ap[j + 1] = len(Ai)
        out.append((n, Ap, np.array(Ai, dtype=np.int64), np.array(Ax, dtype=np.float64)))
    return out


def test_symmetry_verdict_matches_reference(pkg, lib):
    if not os.path.exists(PROBE):
        if not os.path.isdir("/root/reference"):
            pytest.skip("oracle/_ref not built and the reference tree is absent")
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    probe = ctypes.CDLL(PROBE)
    ip = ctypes.POINTER(ctypes.c_int64)
    dp = ctypes.POINTER(ctypes.c_double)
    s = pkg.speigs
    verdicts = {0: 0, 1: 0, 2: 0, 3: 0}
    for n, Ap, Ai, Ax in _variants(np.random.default_rng(21)):
        ref = probe.probe_check_symmetry(ctypes.c_int64(n), Ap.ctypes.data_as(ip),
                                         Ai.ctypes.data_as(ip), Ax.ctypes.data_as(dp))
        verdicts[ref] += 1
        rc, *_ = s.speigs((n, Ap, Ai, Ax), 1, s.SM, s.default_opts(lib), vectors=False, lib=lib)
        assert (rc == s.ERR_NOTSYM) == (ref == 0), (ref, rc, Ap, Ai, Ax)
    assert all(v > 0 for v in verdicts.values()), verdicts
