"""Autotuner of the Krylov method's free parameters, with a JSON cache.

The 'sm' route's block size b (speigs_ext_opts.block) and basis size m
(speigs_opts.ncv) do not change what is computed -- the k wanted eigenpairs
under the same residual test, ||A x - lambda x|| <= tol max(||A||_1, 1) --
only how fast it is computed.  A wider block reads the factor once for more
vectors but builds a Krylov space of lower degree per restart cycle; a
larger basis restarts less often but pays more Gram-Schmidt and a larger
projected problem.  Which pair wins depends on the operator's spectrum and
its factor's tree, so it is measured:

* tune_operator() runs every candidate (b, m) on the caller's operator on
  the GPU -- whole solves on a resident plan, CUDA events on the plan's
  stream, after a warm-up solve -- drops the candidates that did not
  converge or whose eigenvalues differ from the first candidate's by more
  than the tolerance allows, and records the fastest;
* tune_batched() does the same for speigs_batched's hand-off fraction
  (speigs_ext_opts.handoff) on a batch of components, timing the call end to
  end.

Results are stored in a JSON file under a workload signature -- device
name, order, stored entries, k, which, precision, start-subspace width and
tolerance -- so operators of one family (the same grid, other coefficients)
share an entry: tune once on a training instance, then look the entry up
with tuned() for every later solve.  The cache file is the `cache` argument,
else $SPEIGS_B200_TUNE_CACHE, else ~/.cache/speigs_b200/tune.json.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import speigs as s

DEFAULT_BLOCKS = (-1, 8, 16, 24)
DEFAULT_NCVS = (0, 64, 96, 128)
DEFAULT_HANDOFFS = (2, 4, 8, 16, -1)


def cache_path(cache: str | None = None) -> str:
    if cache:
        return cache
    env = os.environ.get("SPEIGS_B200_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "speigs_b200", "tune.json")


def _device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        pass
    return "unknown"


def signature(A, k, which=s.SM, precision=s.FP64, warm_cols=0, tol=1e-10, kind="operator") -> str:
    """Cache key of a workload (see the module docstring)."""
    n = A.shape[0]
    return (f"{kind}|{_device_name()}|n={n}|nnz={A.nnz}|k={k}|which={int(which)}|"
            f"prec={int(precision)}|warm={int(warm_cols)}|tol={tol:.3g}")


def load_cache(cache: str | None = None) -> dict:
    path = cache_path(cache)
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def store(key: str, entry: dict, cache: str | None = None) -> None:
    path = cache_path(cache)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    data = load_cache(path)
    data[key] = entry
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned(A, k, which=s.SM, precision=s.FP64, warm_cols=0, tol=1e-10, cache=None):
    """The cached best (block, ncv) of this workload's signature, or None."""
    e = load_cache(cache).get(signature(A, k, which, precision, warm_cols, tol))
    return None if e is None else (int(e["best"]["block"]), int(e["best"]["ncv"]))


def _time_plan(A, k, which, opts, ext, reps, lib):
    """(best ms over reps after one warm-up, info, ext_info, eigenvalues) of
    one configuration's whole solve on a resident plan."""
    import torch
    n = A.shape[0]
    plan = s.Plan(A, which, opts, lib=lib, ext=ext)
    try:
        st = torch.cuda.ExternalStream(plan.stream())
        lam = torch.zeros(k, dtype=torch.float64, device="cuda")
        V = torch.zeros((k, n), dtype=torch.float64, device="cuda")
        res = torch.zeros(k, dtype=torch.float64, device="cuda")
        ms, info = [], None
        for rep in range(reps + 1):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            rc, info = plan.solve_device(k, lam.data_ptr(), V.data_ptr(), res.data_ptr())
            e1.record(st)
            e1.synchronize()
            if rc != 0:
                return None, info, None, None
            if rep > 0:
                ms.append(e0.elapsed_time(e1))
        return min(ms), info, plan.ext_info(), lam.cpu().numpy()
    finally:
        plan.close()


def tune_operator(A, k, which=s.SM, precision=s.FP64, warm_ptr=None, warm_cols=0, tol=1e-10,
                  blocks=DEFAULT_BLOCKS, ncvs=DEFAULT_NCVS, reps=2, cache=None, lib=None,
                  save=True) -> dict:
    """Time every (block, ncv) candidate on A and cache the fastest.

    block -1 is the reference's single-vector Lanczos (ncv 0 only: its basis
    is the reference's default); b > 0 the block method.  warm_ptr/warm_cols:
    a start subspace for the plans (as speigs_ext_opts.warm).  Candidates
    that fail, do not converge, or whose eigenvalues differ from the first
    candidate's by more than 1e-10 relative (plus the rounding floor of the
    Rayleigh quotient, 64 eps ||A||_1) are dropped.  Returns the cache entry:
    {"best": {...}, "results": [...], "tuned_at": ...}."""
    lib = lib or s.load()
    results, ref = [], None
    for b in blocks:
        for ncv in (ncvs if b > 0 else (0,)):
            opts = s.default_opts(lib, tol=tol, ncv=ncv)
            ext = s.ext_opts(lib, precision=precision, block=b)
            if warm_ptr is not None and warm_cols > 0:
                ext.warm = warm_ptr
                ext.warm_cols = warm_cols
            ms, info, ei, lam = _time_plan(A, k, which, opts, ext, reps, lib)
            r = {"block": b, "ncv": ncv, "ms": None if ms is None else round(ms, 3)}
            if ms is not None:
                r.update(flag=int(info["flag"]), nops=int(info["nops"]),
                         restarts=int(info["restarts"]), block_solves=int(ei["block_solves"]))
                ok = info["flag"] == 0
                if ok and ref is None:
                    ref = (lam, info["anorm"])
                elif ok:
                    floor = 64 * np.finfo(float).eps * max(ref[1], 1.0)
                    ok = bool(np.all(np.abs(np.sort(lam) - np.sort(ref[0])) <=
                                     1e-10 * np.abs(np.sort(ref[0])) + floor))
                r["ok"] = ok
            else:
                r["ok"] = False
            results.append(r)
    good = [r for r in results if r["ok"]]
    if not good:
        raise RuntimeError("tune_operator: no candidate converged")
    best = min(good, key=lambda r: r["ms"])
    entry = {"best": {"block": best["block"], "ncv": best["ncv"], "ms": best["ms"]},
             "results": results, "tuned_at": time.strftime("%Y-%m-%dT%H:%M:%S")}
    if save:
        store(signature(A, k, which, precision, warm_cols, tol), entry, cache)
    return entry


def tune_batched(A, k, comp=None, which=s.SM, tol=1e-10, handoffs=DEFAULT_HANDOFFS, reps=1,
                 cache=None, lib=None, save=True) -> dict:
    """Time speigs_batched end to end for each hand-off fraction and cache
    the fastest.  All candidates compute the same per-component results (a
    handed-off component is solved alone, as the reference solves it)."""
    lib = lib or s.load()
    if comp is None:
        _, comp = s.components(A, lib)
    opts = s.default_opts(lib, tol=tol)
    results = []
    for h in handoffs:
        ext = s.ext_opts(lib, handoff=h)
        ts = []
        for _ in range(reps + 1):
            t0 = time.perf_counter()
            rc, *_ = s.speigs_batched(A, k, which, opts, ext, comp=comp, lib=lib)
            ts.append(time.perf_counter() - t0)
            if rc != 0:
                break
        r = {"handoff": h, "ok": rc == 0, "s": round(min(ts[1:] or ts), 4),
             "stats": s.batched_stats(lib)}
        results.append(r)
    good = [r for r in results if r["ok"]]
    if not good:
        raise RuntimeError("tune_batched: every candidate failed")
    best = min(good, key=lambda r: r["s"])
    entry = {"best": {"handoff": best["handoff"], "s": best["s"]}, "results": results,
             "tuned_at": time.strftime("%Y-%m-%dT%H:%M:%S")}
    if save:
        store(signature(A, k, which, s.FP64, 0, tol, kind="batched"), entry, cache)
    return entry


def tuned_handoff(A, k, which=s.SM, tol=1e-10, cache=None):
    """The cached best hand-off fraction of a batch's signature, or None."""
    e = load_cache(cache).get(signature(A, k, which, s.FP64, 0, tol, kind="batched"))
    return None if e is None else int(e["best"]["handoff"])
