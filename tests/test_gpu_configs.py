"""Parity with the reference at the workloads' full sizes.

Each workload is rebuilt from its seeded generator and fingerprinted against
the input the reference solved (tests/golden/configs.json, written by
tests/golden/make_config_golden.py from oracle/_ref, the reference's own
src/speigs_core.c compiled on the CPU).  Tolerances: eigenvalues within
1e-12 relative for the FP64 forms and 1e-10 for the mixed-precision forms,
and ||A v - lambda v|| <= 1e-10 ||A||_1 for every returned pair, recomputed
here from the returned vectors.
"""
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLD_DIR = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLD_DIR)
from make_config_golden import fingerprint, workloads  # noqa: E402

TOL = 1e-10
GOLD = json.load(open(os.path.join(GOLD_DIR, "configs.json"))) \
    if os.path.exists(os.path.join(GOLD_DIR, "configs.json")) else {}


def _case(pkg, name):
    if name not in GOLD:
        pytest.skip(f"no reference result for {name}")
    build, k, which, _ = workloads(pkg.workloads)[name]
    A = build()
    g = GOLD[name]
    assert fingerprint(A) == g["sha256_32"], "the generator no longer builds the reference's input"
    return A, k, which, g


def _check_pairs(A, lam, V, anorm, nconv_expect=None):
    r = np.linalg.norm(A @ V - V * lam, axis=0)
    assert r.max() <= TOL * anorm * 1.0001, r.max() / anorm


def _solve(pkg, lib, A, k, which, precision="fp64", warm=None):
    s = pkg.speigs
    o = s.default_opts(lib, tol=TOL)
    e = s.ext_opts(lib, precision=s.MIXED if precision == "mixed" else s.FP64)
    rc, lam, V, res, info, ei = s.speigs_ex(A, k, which, o, e, vectors=True, lib=lib, warm=warm)
    assert rc == 0, (rc, s.last_error(lib))
    return lam, V, res, info, ei


def test_c3_varcoef64_fp64(pkg, lib):
    """64^3 variable-coefficient FV operator (n=262,144), k=20 'sm'."""
    A, k, which, g = _case(pkg, "varcoef64_sm_k20")
    lam, V, res, info, _ = _solve(pkg, lib, A, k, which)
    assert info["path"] == g["path"] and info["flag"] == g["flag"] == 0
    rl = np.array(g["lam"])
    assert np.max(np.abs(lam - rl) / np.abs(rl)) <= 1e-12
    _check_pairs(A, lam, V, info["anorm"])
    print(f"nops {info['nops']} (reference {g['nops']}), restarts {info['restarts']} "
          f"({g['restarts']})")
    assert info["nops"] == g["nops"] and info["restarts"] == g["restarts"]


def test_c3_varcoef64_mixed(pkg, lib):
    A, k, which, g = _case(pkg, "varcoef64_sm_k20")
    lam, V, res, info, ei = _solve(pkg, lib, A, k, which, "mixed")
    assert info["flag"] == 0 and ei["precision"] == pkg.speigs.MIXED
    rl = np.array(g["lam"])
    err = np.abs(lam - rl) / np.abs(rl)
    print("per-eigenpair relative error, mixed vs reference:", err)
    assert err.max() <= 1e-10
    _check_pairs(A, lam, V, info["anorm"])


@pytest.mark.parametrize("form", ["fp64", "fp64+learned", "mixed", "mixed+learned"])
def test_c5_grf48_forms(pkg, lib, form):
    """48^3 exp(GRF) operator, held-out seed 3200 (n=110,592), k=16 'sm', every form."""
    A, k, which, g = _case(pkg, "grf48_s3200_sm_k16")
    warm = None
    if "learned" in form:
        L, w = pkg.learned, pkg.workloads
        if not os.path.exists(L.CHECKPOINT):
            pytest.skip("no trained checkpoint")
        net = L.WarmStartNet.load(L.CHECKPOINT, lib=lib)
        warm = L.propose(net, 48, w.grf_conductivity(48, 3200))
    lam, V, res, info, ei = _solve(pkg, lib, A, k, which, form.split("+")[0], warm)
    assert info["flag"] == 0 and info["nconv"] >= k
    rl = np.array(g["lam"])
    err = np.abs(lam - rl) / np.abs(rl)
    print(f"{form}: nops {info['nops']} (reference {g['nops']}), max rel err {err.max():.2e}")
    assert err.max() <= (1e-10 if form.startswith("mixed") else 1e-12)
    _check_pairs(A, lam, V, info["anorm"])
    if form == "fp64":
        assert info["nops"] == g["nops"] and info["restarts"] == g["restarts"]


def test_c2b_lap2d1000_lm(pkg, lib):
    """2-D Laplacian 1000^2 (n=1,000,000), k=6 'lm': the reference stops at
    maxit with a partial flag (near-degenerate top eigenvalues); the device
    library must take the same number of steps to the same verdict, and the
    pairs either side certifies must agree."""
    A, k, which, g = _case(pkg, "lap2d1000_lm_k6")
    s = pkg.speigs
    lam, V, res, info, _ = _solve(pkg, lib, A, k, which)
    assert info["path"] == g["path"] == s.PATH_DIRECT
    assert info["flag"] == g["flag"]
    assert info["nops"] == g["nops"] and info["restarts"] == g["restarts"]
    rtol = TOL * max(g["anorm"], 1.0)
    rl, rres = np.array(g["lam"]), np.array(g["resid"])
    conv = (res <= rtol) | (rres <= rtol)
    print(f"converged pairs: device {int((res <= rtol).sum())}, reference "
          f"{int((rres <= rtol).sum())}")
    if conv.any():
        assert np.max(np.abs(lam[conv] - rl[conv]) / np.abs(rl[conv])) <= 1e-12
    ex = pkg.workloads.spectrum2d_extreme(1000, k, True)
    assert np.max(np.abs(lam - ex) / ex) <= 1e-4


def test_c4_rgg_sample_batched(pkg, lib):
    """The first 120 blocks of the 4,096-block RGG workload through
    speigs_batched, every component against the reference's own speigs()."""
    A, k, which, g = _case(pkg, "rgg_sample_sm_k4")
    s = pkg.speigs
    ncomp, comp = s.components(A, lib)
    assert ncomp == g["ncomp"]
    o = s.default_opts(lib, tol=TOL)
    rc, lam, V, res, nv, info = s.speigs_batched(A, k, which, o, comp=comp, vectors=True,
                                                 lib=lib)
    assert rc == 0 and info["flag"] == 0
    Ad = A.tocsr()
    worst = 0.0
    for c, gc in enumerate(g["components"]):
        kc = len(gc["lam"])
        assert nv[c] == kc
        rl = np.array(gc["lam"])
        err = np.abs(lam[c, :kc] - rl) / np.abs(rl)
        worst = max(worst, float(err.max()))
        rows = np.flatnonzero(comp == c)
        Ac = Ad[rows][:, rows]
        anorm_c = float(abs(Ac).sum(axis=0).max())
        # 1e-12 relative, down to the rounding floor of a Rayleigh quotient
        # (16 eps ||A_c||_1): every block's smallest eigenvalue is 1e-3, and
        # the reference solves components of up to 800 rows with the dense
        # LAPACK eigensolver, whose backward error is also O(eps ||A_c||)
        floor = 16 * np.finfo(float).eps * max(anorm_c, 1.0)
        assert np.all(np.abs(lam[c, :kc] - rl) <= 1e-12 * np.abs(rl) + floor), (c, lam[c, :kc], rl)
        if gc["n"] > 1:
            Vc = V[rows][:, :kc]
            r = np.linalg.norm(Ac @ Vc - Vc * lam[c, :kc], axis=0)
            assert r.max() <= TOL * max(anorm_c, 1.0) * 1.0001
    print(f"{ncomp} components, worst eigenvalue relative error {worst:.2e}; total operator "
          f"applications {info['nops']} (reference {sum(gc['nops'] for gc in g['components'])})")
