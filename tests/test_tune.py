"""The autotuner's cache (sparse-eigs-mex_b200/tune.py): workload
signatures, storing and looking up entries in a JSON file, on the CPU; and,
on the GPU, a tuning run over a few block and basis sizes whose winner
converged, agrees with the reference method's eigenvalues and is found
again by tuned()."""
import json

import numpy as np
import pytest


def test_signature_and_cache_roundtrip(pkg, tmp_path):
    t, w = pkg.tune, pkg.workloads
    A = w.lap3d(8)
    B = A.copy()
    B.data = B.data * 2.0                      # same family: same pattern, other values
    cache = str(tmp_path / "tune.json")
    key = t.signature(A, 6)
    assert key == t.signature(B, 6)
    assert key != t.signature(A, 7) and key != t.signature(A, 6, precision=1)
    assert key != t.signature(A, 6, warm_cols=24) and key != t.signature(A, 6, kind="batched")
    assert t.tuned(A, 6, cache=cache) is None
    t.store(key, {"best": {"block": 8, "ncv": 96, "ms": 1.0}, "results": []}, cache)
    t.store(t.signature(A, 6, kind="batched"), {"best": {"handoff": 4, "s": 2.0}}, cache)
    assert t.tuned(B, 6, cache=cache) == (8, 96)
    assert t.tuned_handoff(A, 6, cache=cache) == 4
    data = json.load(open(cache))
    assert set(data) == {key, t.signature(A, 6, kind="batched")}


def test_cache_path_from_environment(pkg, tmp_path, monkeypatch):
    monkeypatch.setenv("SPEIGS_B200_TUNE_CACHE", str(tmp_path / "x.json"))
    assert pkg.tune.cache_path() == str(tmp_path / "x.json")
    assert pkg.tune.cache_path(str(tmp_path / "y.json")) == str(tmp_path / "y.json")


@pytest.mark.gpu
def test_tune_operator_picks_a_converged_candidate(pkg, lib, tmp_path):
    t, s, w = pkg.tune, pkg.speigs, pkg.workloads
    A = w.varcoef3d(20, seed=4)
    cache = str(tmp_path / "tune.json")
    e = t.tune_operator(A, 8, blocks=(-1, 8, 16), ncvs=(0, 64), reps=1, cache=cache, lib=lib)
    assert e["results"][0]["block"] == -1 and e["results"][0]["ok"]
    best = e["best"]
    assert any(r["ok"] and r["block"] == best["block"] and r["ncv"] == best["ncv"]
               for r in e["results"])
    assert best["ms"] == min(r["ms"] for r in e["results"] if r["ok"])
    assert t.tuned(A, 8, cache=cache) == (best["block"], best["ncv"])
    # the tuned configuration through the drop-in extension call
    o = s.default_opts(lib, tol=1e-10, ncv=best["ncv"])
    x = s.ext_opts(lib, block=best["block"])
    rc, lam, V, res, info, ei = s.speigs_ex(A, 8, s.SM, o, x, lib=lib)
    rc0, lam0, *_ = s.speigs(A, 8, s.SM, s.default_opts(lib, tol=1e-10), lib=lib)
    assert rc == 0 and rc0 == 0 and info["flag"] == 0
    assert np.all(np.abs(lam - lam0) <= 1e-10 * np.abs(lam0) + 64 * np.finfo(float).eps *
                  info["anorm"])
