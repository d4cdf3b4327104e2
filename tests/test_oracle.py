"""The oracle, pinned before it is trusted (CPU only).

* The reference's solver compiled from its sources against this project's
  CHOLMOD/UMFPACK stand-in passes the reference's own validation suite
  (test/test_speigs.c, 73 checks) apart from checks known to depend on
  rounding.
* The numpy restatement (oracle/speigs_oracle.py) reproduces the reference's
  static helpers bit for bit (golden vectors from oracle/_ref/libspeigs_probe)
  and the reference solver's eigenpairs and operator counts.
"""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ORACLE_DIR, ROOT

GOLD = os.path.join(ROOT, "tests", "golden")
TEST_BIN = os.path.join(ORACLE_DIR, "_ref", "test_speigs")
PROBE = os.path.join(ORACLE_DIR, "_ref", "libspeigs_probe.so")


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(GOLD, "golden.npz"))
    meta = json.load(open(os.path.join(GOLD, "golden.json")))
    return z, meta


def _need_ref_build(path):
    if not os.path.exists(path):
        if not os.path.isdir("/root/reference"):
            pytest.skip("oracle/_ref not built here")
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])


def test_reference_validation_suite():
    _need_ref_build(TEST_BIN)
    # single-threaded BLAS: the singular case [2] (shift 1.2e-5 on a PSD
    # matrix with a null space, tol 1e-14) converges or not depending on the
    # summation order of the threaded BLAS kernels on some CPUs; one thread
    # gives the serial order the reference's own runs use
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    out = subprocess.run([TEST_BIN, "16"], capture_output=True, text=True, env=env,
                         timeout=600).stdout
    m = re.search(r"(\d+) checks, (\d+) failures", out)
    assert m, out[-2000:]
    checks, fails = int(m.group(1)), int(m.group(2))
    assert checks == 73
    failed = [ln for ln in out.splitlines() if ln.strip().startswith("FAIL")]
    # the third copy of the top triple in 'lm' mode is found or missed by
    # rounding (single-vector Lanczos); nothing else may fail
    assert all("largest[3]" in ln for ln in failed), failed
    assert fails <= 1


def test_restated_rng_matches_reference(golden, oracle):
    z, meta = golden
    for i, r in enumerate(meta["rng"]):
        seed_after, v = oracle.rand_vec(int(r["seed"]), r["n"])
        assert np.array_equal(v, z[f"rng{i}"])
        assert seed_after == int(r["seed_after"])


def test_restated_orth_block_matches_reference(golden, oracle):
    z, _ = golden
    h = np.zeros(z["orth_B"].shape[1])
    w = oracle.orth_block(z["orth_B"], z["orth_w0"].copy(), h)
    assert np.allclose(w, z["orth_w"], rtol=0, atol=1e-15)
    assert np.allclose(h, z["orth_h"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("name", ["lap3d12_sm_k5", "neumann10_sm_k4", "varcoef12_sm_k6",
                                  "varcoef10_lm_k4"])
def test_restated_solver_matches_reference(golden, oracle, pkg, name):
    z, meta = golden
    w = pkg.workloads
    build = {"lap3d12_sm_k5": (lambda: w.lap3d(12), 5, "sm"),
             "neumann10_sm_k4": (lambda: w.lap3d(10, dirichlet=False), 4, "sm"),
             "varcoef12_sm_k6": (lambda: w.varcoef3d(12, seed=3), 6, "sm"),
             "varcoef10_lm_k4": (lambda: w.varcoef3d(10, seed=5), 4, "lm")}[name]
    A = build[0]()
    out = oracle.speigs(A, build[1], build[2], tol=1e-10)
    ref = z[f"{name}_lam"]
    assert np.max(np.abs(out["lam"] - ref) / np.abs(ref).clip(1e-300)) <= 1e-10 or \
        np.max(np.abs(out["lam"] - ref)) <= 1e-12
    if name != "neumann10_sm_k4":
        # the reference factors this one with its banded route and a larger
        # shift, so only its eigenvalues are comparable
        assert out["nops"] == meta["cases"][name]["nops"]


def test_restated_symmetry_and_components_match_reference(oracle, pkg):
    _need_ref_build(PROBE)
    import scipy.sparse as sp
    probe = ctypes.CDLL(PROBE)
    ip = ctypes.POINTER(ctypes.c_int64)
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(3)
    cases = []
    for t in range(6):
        n = 40 + 10 * t
        R = sp.random(n, n, density=0.04, random_state=rng, format="csc")
        S = (R + R.T).tocsc()
        cases += [S, sp.triu(S, format="csc"), sp.tril(S, format="csc"), R.tocsc()]
    for A in cases:
        A = A.tocsc()
        A.sort_indices()
        n = A.shape[0]
        Ap = A.indptr.astype(np.int64)
        Ai = A.indices.astype(np.int64)
        Ax = A.data.astype(np.float64)
        got = probe.probe_check_symmetry(ctypes.c_int64(n), Ap.ctypes.data_as(ip),
                                         Ai.ctypes.data_as(ip), Ax.ctypes.data_as(dp))
        assert got == oracle.check_symmetry(A)
        comp = np.zeros(n, dtype=np.int64)
        probe.probe_find_components.restype = ctypes.c_int64
        nc = probe.probe_find_components(ctypes.c_int64(n), Ap.ctypes.data_as(ip),
                                         Ai.ctypes.data_as(ip), Ax.ctypes.data_as(dp),
                                         comp.ctypes.data_as(ip))
        nc2, comp2 = oracle.find_components(A)
        assert nc == nc2 and np.array_equal(comp, comp2)
