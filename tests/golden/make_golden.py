"""Regenerate tests/golden/ from the reference's own code compiled on the CPU.

    make -C oracle && python tests/golden/make_golden.py

Sources: oracle/_ref/libspeigs_probe.so (static helpers of the reference's
src/speigs_core.c: rand_vec, orth_block) and oracle/_ref/libspeigs_ref.so
(the reference's speigs() over the CHOLMOD stand-in).  The fixtures pin the
CPU restatement and the device library to the reference's behaviour.
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import REF_LIB, import_package  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "libspeigs_probe.so")

CASES = {
    # name: (builder, k, which)
    "lap3d12_sm_k5": (lambda w: w.lap3d(12), 5, 0),
    "neumann10_sm_k4": (lambda w: w.lap3d(10, dirichlet=False), 4, 0),
    "varcoef12_sm_k6": (lambda w: w.varcoef3d(12, seed=3), 6, 0),
    "varcoef10_lm_k4": (lambda w: w.varcoef3d(10, seed=5), 4, 1),
    "blocks12_10_sm_k6": (lambda w: w.block_diag(w.lap3d(12), w.lap3d(10)), 6, 0),
}
RNG = [(88172645463325252, 4096), (12345, 1000), (2**63 + 11, 777)]


def main():
    pkg = import_package()
    s, w = pkg.speigs, pkg.workloads
    probe = ctypes.CDLL(PROBE)
    arrays, meta = {}, {"rng": [], "cases": {}}
    for i, (seed, n) in enumerate(RNG):
        v = np.zeros(n)
        after = ctypes.c_uint64()
        probe.probe_rand_vec(ctypes.c_uint64(seed), ctypes.c_int64(n),
                             v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(after))
        arrays[f"rng{i}"] = v
        meta["rng"].append({"seed": str(seed), "n": n, "seed_after": str(after.value)})
    rng = np.random.default_rng(7)
    n, m = 500, 7
    B, _ = np.linalg.qr(rng.standard_normal((n, m)))
    B = np.asfortranarray(B)
    w0 = rng.standard_normal(n)
    wv = w0.copy()
    h = np.zeros(m)
    dp = ctypes.POINTER(ctypes.c_double)
    probe.probe_orth_block(ctypes.c_int64(n), ctypes.c_int64(m), B.ctypes.data_as(dp),
                           wv.ctypes.data_as(dp), h.ctypes.data_as(dp))
    arrays.update(orth_B=B, orth_w0=w0, orth_w=wv, orth_h=h)
    ref = s.load(REF_LIB)
    for name, (build, k, which) in CASES.items():
        A = build(w)
        o = s.default_opts(ref, tol=1e-10)
        rc, lam, V, res, info = s.speigs(A, k, which, o, lib=ref)
        assert rc == 0, name
        arrays[f"{name}_lam"] = lam
        arrays[f"{name}_resid"] = res
        meta["cases"][name] = {k2: info[k2] for k2 in ("flag", "nconv", "restarts", "nops",
                                                        "shift", "anorm", "path", "ncomp")}
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", sorted(arrays))


if __name__ == "__main__":
    main()
