"""Reference results at the workloads' full sizes, for the device parity tests.

    make -C oracle && python tests/golden/make_config_golden.py [name ...]

Runs the reference's own solver (oracle/_ref/libspeigs_ref.so: the
reference's src/speigs_core.c compiled unmodified over this project's
CHOLMOD/UMFPACK stand-ins) once per workload on the CPU and writes
tests/golden/configs.json: eigenvalues, residuals, operator applications,
restarts, flag, route and shift.  Every workload is a seeded synthetic
operator from sparse-eigs-mex_b200/workloads.py, built the same way by the
tests; the CSC bytes are fingerprinted (sha256) so a test can tell that it
rebuilt the same input.  The reference runs with its default options except
tol = 1e-10.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import REF_LIB, import_package  # noqa: E402

OUT = os.path.join(HERE, "configs.json")
TOL = 1e-10


def workloads(w):
    """name: (builder, k, which, description) -- the same builders the tests use."""
    return {
        "lap2d1000_lm_k6": (lambda: w.lap2d(1000), 6, 1,
                            "2-D 5-point Dirichlet Laplacian 1000^2 (n=1,000,000), k=6 'lm'"),
        "varcoef64_sm_k20": (lambda: w.varcoef3d(64, seed=3), 20, 0,
                             "3-D FV, log-normal conductivity (sigma 1, seed 3), 64^3, k=20 'sm'"),
        "grf48_s3200_sm_k16": (lambda: w.grf3d(48, 3200), 16, 0,
                               "3-D FV, conductivity exp(GRF) seed 3200, 48^3, k=16 'sm'"),
        "rgg_sample_sm_k4": (lambda: w.rgg_sample(), 4, 0,
                             "120 components of the 4,096-component RGG generator (seed 4), "
                             "k=4 'sm' per component"),
    }


def fingerprint(A):
    A = A.tocsc()
    h = hashlib.sha256()
    for a in (A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data.astype(np.float64)):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def run_one(s, ref, A, k, which):
    o = s.default_opts(ref, tol=TOL)
    t0 = time.perf_counter()
    rc, lam, V, res, info = s.speigs(A, k, which, o, vectors=False, lib=ref)
    dt = time.perf_counter() - t0
    assert rc == 0, rc
    return {"lam": lam.tolist(), "resid": res.tolist(), "nops": int(info["nops"]),
            "restarts": int(info["restarts"]), "flag": int(info["flag"]),
            "nconv": int(info["nconv"]), "path": int(info["path"]), "shift": info["shift"],
            "anorm": info["anorm"], "cpu_s": dt}


def main(names):
    pkg = import_package()
    s, w = pkg.speigs, pkg.workloads
    ref = s.load(REF_LIB)
    meta = json.load(open(OUT)) if os.path.exists(OUT) else {}
    meta.setdefault("_source", "oracle/_ref/libspeigs_ref.so (reference src/speigs_core.c "
                               "over the CHOLMOD stand-in), tol 1e-10, default options")
    meta.setdefault("_threads", os.environ.get("OPENBLAS_NUM_THREADS", "default"))
    for name, (build, k, which, desc) in workloads(w).items():
        if names and name not in names:
            continue
        A = build()
        entry = {"desc": desc, "n": int(A.shape[0]), "nnz": int(A.nnz), "k": k, "which": which,
                 "sha256_32": fingerprint(A)}
        if name.startswith("rgg_sample"):
            # per component, as speigs_batched returns them: the reference
            # solves each component with its own speigs() call
            ncomp, comp = w.components_of(A)
            Ad = A.tocsr()
            comps = []
            for c in range(ncomp):
                rows = np.flatnonzero(comp == c)
                kc = min(k, len(rows))
                if len(rows) == 1:
                    comps.append({"n": 1, "lam": [float(Ad[rows[0], rows[0]])], "nops": 0,
                                  "flag": 0, "path": 0})
                    continue
                r = run_one(s, ref, Ad[rows][:, rows].tocsc(), kc, which)
                comps.append({"n": int(len(rows)), "lam": r["lam"], "nops": r["nops"],
                              "flag": r["flag"], "path": r["path"], "resid": r["resid"],
                              "anorm": r["anorm"]})
            entry["ncomp"] = int(ncomp)
            entry["components"] = comps
        else:
            entry.update(run_one(s, ref, A, k, which))
        meta[name] = entry
        print(name, {kk: entry[kk] for kk in entry if kk not in ("components", "lam", "resid")},
              flush=True)
        json.dump(meta, open(OUT, "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
