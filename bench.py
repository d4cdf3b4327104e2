#!/usr/bin/env python
"""Time to k eigenpairs at residual <= 1e-10 ||A||_1 on B200.

Default workload: the metric's own configuration -- the held-out 48^3
finite-volume operator with conductivity exp(GRF) (seed 3200), k=16 'sm' --
timed in every form on the same B200: the plain FP64 drop-in, mixed
precision, the learned block start, and both together (the line's `value`).
Other workloads (--workload lap46, lap20, lap2d1000, varcoef64, rgg) time
one form of the drop-in path.

A step is one complete solve of the workload: numeric factorization ('sm')
plus thick-restart Lanczos to convergence, with the k eigenpairs left in
device memory.  `value` times steps with the matrix and its symbolic
analysis already resident on the GPU (speigs_plan_solve_device); `e2e` times
the drop-in call speigs() from host CSC arrays to host results, so the host
analysis and every host<->device copy are inside.  N GPUs run N independent
replicas (the single-operator path does not shard), so scaling is weak.

--impl reference times the reference's own CPU solver (compiled from its
sources into oracle/_ref, CHOLMOD stand-in and OpenBLAS) on the same
workload with every host thread, on rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "sparse-eigs-mex_b200")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libspeigs_ref.so")
METRIC = "time to k eigenpairs @ resid 1e-10: mixed/learned vs plain FP64, same B200"
TOL = 1e-10
TUNE_SEED = 1000          # a training operator of the 48^3 GRF family (the tuner's input)


def import_pkg():
    import importlib.util
    if "speigs_b200" in sys.modules:
        return sys.modules["speigs_b200"]
    spec = importlib.util.spec_from_file_location(
        "speigs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["speigs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workloads(w, s):
    return {
        "lap46": dict(desc="3-D 7-point Dirichlet Laplacian 46^3 (n=97,336), k=6 smallest ('sm', "
                           "shift-invert), FP64 CSR, tol 1e-10",
                      build=lambda: w.lap3d(46), k=6, which=s.SM,
                      exact=lambda: w.spectrum3d(46)[:6]),
        "lap20": dict(desc="3-D 7-point Dirichlet Laplacian 20^3 (n=8,000), k=6 'sm', tol 1e-10",
                      build=lambda: w.lap3d(20), k=6, which=s.SM,
                      exact=lambda: w.spectrum3d(20)[:6]),
        "lap2d1000": dict(desc="2-D 5-point Dirichlet Laplacian 1000^2 (n=1,000,000), k=6 largest "
                               "('lm', direct Lanczos), tol 1e-10",
                          build=lambda: w.lap2d(1000), k=6, which=s.LM,
                          exact=lambda: w.spectrum2d_extreme(1000, 6, True)),
        "varcoef64": dict(desc="3-D variable-coefficient FV diffusion 64^3 (n=262,144), log-normal "
                               "conductivity (sigma=1, seed 3), k=20 'sm', tol 1e-10",
                          build=lambda: w.varcoef3d(64, seed=3), k=20, which=s.SM, exact=None),
        "grf48": dict(desc="3-D FV diffusion 48^3 (n=110,592), conductivity exp(GRF) (SE "
                           "covariance, length 0.1, variance 1), held-out seed 3200, k=16 'sm', "
                           "tol 1e-10",
                      build=lambda: w.grf3d(48, 3200), k=16, which=s.SM, exact=None),
        "rgg": dict(desc="block-diagonal SPD: 4,096 random-geometric-graph Laplacians (+1e-3 I), "
                         "sizes U[50, 5000] (seed 4), mean degree 8, k=4 'sm' per component, "
                         "tol 1e-10",
                    build=lambda: w.rgg_blocks(4096, seed=4), k=4, which=s.SM, exact=None),
        "rgg256": dict(desc="block-diagonal SPD: the first 256 blocks of the 4,096-block "
                            "random-geometric-graph workload, k=4 'sm' per component, tol 1e-10",
                       build=lambda: w.rgg_blocks(4096, seed=4, first=256), k=4, which=s.SM,
                       exact=None),
    }


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def _wait_line(self, timeout):
        t0 = time.time()
        while not self.lines and time.time() - t0 < timeout and self.proc.poll() is None:
            time.sleep(0.005)

    def ready(self, timeout=5.0):
        """Wait until nvidia-smi reports, then drop what it sampled before the
        timed region (a short region would otherwise see no sample at all)."""
        if self.proc:
            self._wait_line(timeout)
            self.lines.clear()

    def stop(self, gpu_index=None):
        if not self.proc:
            return None
        # a region shorter than the sampling interval: take the next sample
        self._wait_line(0.5)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            if gpu_index is not None and p[0] != str(gpu_index):
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_times(pkg, A, wl, steps, warmup, budget_s=None):
    """Wall time of the reference's CPU solver (oracle/_ref) per full solve."""
    s = pkg.speigs
    ref = s.load(REF_LIB)
    o = s.default_opts(ref, tol=TOL)
    out = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        rc, lam, V, res, info = s.speigs(A, wl["k"], wl["which"], o, vectors=True, lib=ref)
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"reference solver rc={rc}")
        if i >= warmup:
            out.append(dt)
        if budget_s is not None and sum(out) > budget_s and len(out) >= 1:
            break
    return out, lam, info


def run_reference(args, pkg, wl, rank):
    if rank != 0:
        return 0
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libspeigs_ref.so not built (needs the reference tree)"}))
        return 0
    A = wl["build"]()
    times, lam, info = cpu_reference_times(pkg, A, wl, args.steps, args.warmup)
    v = statistics.mean(times)
    cores = os.cpu_count()
    line = {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": wl["desc"], "n": int(A.shape[0]), "nnz": int(A.nnz), "k": wl["k"],
                   "tol": TOL, "nops": int(info["nops"]), "restarts": int(info["restarts"])},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "reference",
                         "sample": "full solves of the same workload by the reference's "
                                   "src/speigs_core.c (CHOLMOD stand-in + OpenBLAS, all host "
                                   "threads)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _dev_time(torch, fn, steps, warmup, stream):
    for _ in range(warmup):
        fn()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ms = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.mean(ms), out, ms


def block_solve_bytes(op_bytes_single, n, b):
    """Algorithmic bytes of one block solve of b columns: the panels and row
    lists once forward and once backward (the single solve's figure), plus
    three n-vectors per column (right-hand side in, intermediate, result)."""
    return op_bytes_single + 24.0 * n * (b - 1)


def run_metric(args, pkg, wl, ctx):
    """The headline: time to k=16 eigenpairs of the held-out 48^3 GRF operator
    at residual <= 1e-10 ||A||_1, mixed precision with the learned block start
    (`value`) against the plain FP64 drop-in and the other forms, same B200.

    Device timing (`value`, `forms[*].value_s`): one solve per step on a plan
    whose matrix and symbolic analysis are resident -- numeric factor, the
    network's proposal on the device (learned forms), the Lanczos to
    convergence -- on the plan's stream with CUDA events, a 256 MiB buffer
    written between steps to flush L2.  End to end (`e2e`): host CSC and host
    conductivity in, host eigenpairs out: the proposal (graph and features
    built on the host, uploaded, network forward, result downloaded) and
    speigs_ex() with every copy inside."""
    import torch
    s, w, L = pkg.speigs, pkg.workloads, pkg.learned
    lib = ctx["lib"]
    dev = ctx["dev"]
    N, seed = 48, 3200
    A = wl["build"]()
    n, k, nnz = A.shape[0], wl["k"], A.nnz
    kap = w.grf_conductivity(N, seed)
    opts = s.default_opts(lib, tol=TOL)
    have_net = os.path.exists(L.CHECKPOINT)
    net = L.WarmStartNet.load(L.CHECKPOINT, lib=lib) if have_net else None
    P = net.nout if net is not None else 24
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peak, peak_kind = measured_peaks()

    # the proposal's inputs on the device (the learned forms read them
    # there): the conductivities and the node features; the network's graph
    # is built from the conductivities on the device in every step
    X = L.features(N, kap)
    t_kap = torch.from_numpy(np.ascontiguousarray(kap, dtype=np.float64).ravel()).to(dev)
    gnnz = 6 * N * N * (N - 1)
    t_rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    t_ci = torch.empty(gnnz, dtype=torch.int32, device=dev)
    t_w = torch.empty(gnnz, dtype=torch.float32, device=dev)
    t_X = torch.from_numpy(X).to(dev)
    Y32 = torch.empty((n, P), dtype=torch.float32, device=dev)
    Yw = torch.zeros((P, n), dtype=torch.float64, device=dev)      # column-major n x P

    def propose_device(stream):
        rc = net.grid_graph_device(N, t_kap.data_ptr(), t_rp.data_ptr(), t_ci.data_ptr(),
                                   t_w.data_ptr(), stream.cuda_stream)
        if rc != 0:
            raise RuntimeError(f"mpnn grid graph rc={rc}")
        rc = net.forward_device(n, t_rp.data_ptr(), t_ci.data_ptr(), t_w.data_ptr(),
                                t_X.data_ptr(), Y32.data_ptr(), stream.cuda_stream)
        if rc != 0:
            raise RuntimeError(f"mpnn forward rc={rc}")
        with torch.cuda.stream(stream):
            Yw.copy_(Y32.t())

    # the proposal's forward pass alone (CUDA events, median of 20 after 3
    # warm-up runs), with the dense layers on the tensor cores (the default)
    # and on the FP32-FMA kernels, before any timed region
    proposal_ms = None
    if net is not None:
        proposal_ms = {}
        pst = torch.cuda.current_stream()
        for label, on in (("fma_dense_layers", 0), ("tensor_core_dense_layers", 1)):
            net.tensor_cores(on)
            for _ in range(3):
                propose_device(pst)
            tms = []
            for _ in range(20):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(pst)
                propose_device(pst)
                e1.record(pst)
                e1.synchronize()
                tms.append(e0.elapsed_time(e1))
            proposal_ms[label] = round(statistics.median(tms), 4)
        net.tensor_cores(1)

    # ---- autotuning (before any timed region): the block size and basis
    # size of the learned forms, chosen by pkg.tune on a TRAINING operator
    # of the same family (seed 1000, one the network was trained on), with
    # that operator's own proposal; the held-out operator is not seen
    tuning = {}
    if net is not None and not args.no_tune:
        kap_t = w.grf_conductivity(N, TUNE_SEED)
        A_t = w.grf3d(N, TUNE_SEED)
        rp_t, ci_t, w_t = L.grid_graph(N, kap_t)
        X_t = L.features(N, kap_t)
        tt = [torch.from_numpy(a).to(dev) for a in (rp_t, ci_t, w_t, X_t)]
        Y_t = torch.zeros((P, n), dtype=torch.float64, device=dev)
        rc = net.forward_device(n, tt[0].data_ptr(), tt[1].data_ptr(), tt[2].data_ptr(),
                                tt[3].data_ptr(), Y32.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise RuntimeError(f"mpnn forward rc={rc}")
        Y_t.copy_(Y32.t())
        torch.cuda.synchronize()
        cache = os.path.join(ROOT, "gpurun_out", "tune_cache.json") \
            if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else None
        t_tune = time.perf_counter()
        for pname, prec in (("fp64", s.FP64), ("mixed", s.MIXED)):
            e = pkg.tune.tune_operator(A_t, k, s.SM, prec, warm_ptr=Y_t.data_ptr(), warm_cols=P,
                                       tol=TOL, blocks=(-1, 8, 16, 24), ncvs=(64, 96, 128),
                                       reps=1, cache=cache, lib=lib)
            tuning[pname] = e["best"]
            tuning[pname + "_candidates"] = [
                {kk: r.get(kk) for kk in ("block", "ncv", "ms", "ok", "block_solves")}
                for r in e["results"]]
        tuning["seconds"] = round(time.perf_counter() - t_tune, 2)
        del Y_t, tt
    fb, fn = (tuning["fp64"]["block"], tuning["fp64"]["ncv"]) if tuning else (0, 0)
    mb, mn = (tuning["mixed"]["block"], tuning["mixed"]["ncv"]) if tuning else (0, 0)

    forms_spec = [("fp64", s.FP64, False, -1, 0), ("mixed", s.MIXED, False, -1, 0)]
    if net is not None:
        forms_spec += [("fp64+learned", s.FP64, True, fb, fn),
                       ("mixed+learned", s.MIXED, True, mb, mn)]
    forms_spec += [("fp64+block(random)", s.FP64, False, fb if fb > 0 else P, fn),
                   ("mixed+block(random)", s.MIXED, False, mb if mb > 0 else P, mn)]
    target = "mixed+learned" if net is not None else "mixed"
    form_params = {name: {"block": b, "ncv": c} for name, _, _, b, c in forms_spec}
    forms, keep = {}, {}
    for name, prec, learned, block, ncv in forms_spec:
        ext = s.ext_opts(lib, precision=prec, block=block)
        if learned:
            ext.warm = Yw.data_ptr()
            ext.warm_cols = P
        fopts = s.default_opts(lib, tol=TOL, ncv=ncv)
        plan = s.Plan(A, s.SM, fopts, lib=lib, ext=ext)
        pstream = torch.cuda.ExternalStream(plan.stream(), device=dev)
        lam = torch.zeros(k, dtype=torch.float64, device=dev)
        V = torch.zeros((k, n), dtype=torch.float64, device=dev)
        res = torch.zeros(k, dtype=torch.float64, device=dev)

        def step():
            if learned:
                propose_device(pstream)
            rc, info = plan.solve_device(k, lam.data_ptr(), V.data_ptr(), res.data_ptr())
            if rc != 0:
                raise RuntimeError(f"{name}: rc={rc} {s.last_error(lib)}")
            return info
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            info = step()
        is_target = name == target
        steps = args.steps if is_target or name == "fp64" else max(2, min(args.steps, 3))
        sampler = ClockSampler()
        if is_target:
            sampler.start()
            sampler.ready()
        ctx["barrier"]()
        torch.cuda.synchronize()
        l0 = s.counters(lib)[0]
        step_ms, t_op, t_all = [], 0.0, []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(pstream)
            info = step()
            e1.record(pstream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            t_op += info["t_op"]
            t_all.append({kk: round(info[kk], 5) for kk in ("t_factor", "t_op", "t_ortho",
                                                               "t_resid", "t_ritz")})
        torch.cuda.synchronize()
        launches = (s.counters(lib)[0] - l0) // max(steps, 1)
        ctx["barrier"]()
        clocks = sampler.stop() if is_target else None
        ei = plan.ext_info()
        costs = plan.costs()
        lam_h = lam.cpu().numpy()
        Vh = np.ascontiguousarray(V.cpu().numpy().T)
        r = np.linalg.norm(A @ Vh - Vh * lam_h[None, :], axis=0)
        plan.close()
        forms[name] = {"value_s": statistics.mean(step_ms) * 1e-3,
                       "step_ms": [round(x, 3) for x in step_ms],
                       "nops": int(info["nops"]), "restarts": int(info["restarts"]),
                       "flag": int(info["flag"]), "block": int(ei["block"]),
                       "ncv_opt": int(ncv),
                       "block_solves": int(ei["block_solves"]),
                       "refine_steps": int(ei["refine_steps"]), "warm_cols": int(ei["warm_cols"]),
                       "max_resid_over_anorm": float(r.max() / info["anorm"]),
                       "phases_s": t_all[-1]}
        keep[name] = dict(lam=lam_h, info=info, ei=ei, costs=costs, launches=launches,
                          clocks=clocks, t_op=t_op / steps, steps=steps)

    # ---- end to end through the public API: host in, host out
    def e2e_run(name):
        prec = s.MIXED if name.startswith("mixed") else s.FP64
        learned = "learned" in name
        c0 = s.counters(lib)
        t0 = time.perf_counter()
        extra_h2d = extra_d2h = 0
        if learned:
            # the proposal stays on the device: its graph and features go up,
            # the network runs, and speigs_ex takes the device subspace
            Yd = L.propose(net, N, kap, on_device=True)
            extra_h2d = kap.nbytes + X.nbytes
            fp = form_params[name]
            ext = s.ext_opts(lib, precision=prec, block=fp["block"])
            ext.warm = Yd.data_ptr()
            ext.warm_cols = Yd.shape[0]
            eopts = s.default_opts(lib, tol=TOL, ncv=fp["ncv"])
            rc, *_ = s.speigs_ex(A, k, s.SM, eopts, ext, vectors=True, lib=lib)
            del Yd
        else:
            ext = s.ext_opts(lib, precision=prec, block=-1)
            rc, *_ = s.speigs_ex(A, k, s.SM, opts, ext, vectors=True, lib=lib)
        dt = time.perf_counter() - t0
        c1 = s.counters(lib)
        if rc != 0:
            raise RuntimeError(f"e2e {name}: rc={rc} {s.last_error(lib)}")
        return dt, c1[1] - c0[1] + extra_h2d, c1[2] - c0[2] + extra_d2h
    e2e = {}
    for name in (target, "fp64"):
        for _ in range(max(1, min(args.warmup, 2))):
            e2e_run(name)
        ts, h2d, d2h = [], 0, 0
        for _ in range(max(2, min(args.steps, 3))):
            dt, h2d, d2h = e2e_run(name)
            ts.append(dt)
        e2e[name] = {"value": statistics.mean(ts), "unit": "s", "h2d_bytes_per_step": int(h2d),
                     "d2h_bytes_per_step": int(d2h), "steps_s": [round(x, 4) for x in ts]}

    # ---- roofline of the dominant kernel of the timed form.  For a block
    # form that is the block solve mf_bsolve (FP32 panels in the mixed
    # form): algorithmic bytes of one launch (the plan's solve-pair bytes
    # with rows of b values) over its average device time, measured by the
    # library with CUDA events around every block solve of the timed solve
    # (t_block_solve over the solves that ran; corrections that returned at
    # once on the device add a few microseconds each).  For the
    # single-vector forms it is the solve pair mf_solve_sf, timed the same
    # way through the operator phase.
    kt = keep[target]
    ei, info = kt["ei"], kt["info"]
    bsz = max(1, int(ei["block"]))
    if bsz > 1:
        launches = max(1, int(ei["block_solves"]))
        per_launch = block_solve_bytes(kt["costs"]["op_bytes"], n, bsz)
        avg_s = float(ei["t_block_solve"]) / launches
        kname = f"mf_bsolve<{(bsz + 7) // 8 * 8}>"
    else:
        launches = max(1, int(info["nops"]) + int(ei["refine_steps"]))
        per_launch = kt["costs"]["op_bytes"]
        avg_s = kt["t_op"] / launches
        kname = "mf_solve_sf"
    achieved = per_launch / avg_s / 1e9 if avg_s > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"grf48:{target}:{kname}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": kname + (" (FP32 panels, %d right-hand sides)" % bsz
                                   if target.startswith("mixed") and bsz > 1 else ""),
                "bytes_per_launch": per_launch, "avg_launch_s": avg_s, "launches": launches,
                "peak_source": peak_kind}
    if bsz > 1:
        roofline["queued_solves"] = int(ei["block_solve_calls"])

    # ---- the reference's CPU solver on the same operator (rank 0, N=1)
    cpu, check = None, {}
    base = keep["fp64"]["lam"]
    tl = keep[target]["lam"]
    check["eig_rel_err_vs_fp64"] = [float(x) for x in np.abs(tl - base) / np.abs(base)]
    check["max_resid_over_anorm"] = forms[target]["max_resid_over_anorm"]
    check["flag"] = forms[target]["flag"]
    if ctx["rank"] == 0 and ctx["world"] == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
        times, rlam, rinfo = cpu_reference_times(pkg, A, wl, steps=2, warmup=1, budget_s=30.0)
        cpu = {"value": statistics.median(times), "unit": "s", "cores": os.cpu_count(),
               "kind": "reference",
               "sample": f"{len(times)} full solve(s) of the same operator by the reference's "
                         "src/speigs_core.c (CHOLMOD stand-in + OpenBLAS, all host threads), "
                         "median"}
        rlam = np.sort(np.asarray(rlam))
        check["eig_rel_err_vs_reference"] = [float(x) for x in np.abs(np.sort(tl) - rlam) /
                                             np.abs(rlam)]
        check["reference_nops"] = int(rinfo["nops"])
    tv = forms[target]["value_s"]
    t = torch.tensor([tv], dtype=torch.float64, device=dev)
    ctx["max"](t)
    tv = float(t.item())
    if ctx["rank"] == 0:
        line = {
            "metric": METRIC, "value": tv, "unit": "s", "n_gpus": ctx["world"],
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tv * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 factor panels, f64 refinement / recurrence / Ritz" if target.startswith(
                "mixed") else "f64",
            "data": "synthetic",
            "config": {"workload": wl["desc"], "n": int(n), "nnz": int(nnz), "k": k, "tol": TOL,
                       "form": target + (" (block thick-restart Lanczos, first block = the "
                                         "network's %d-column proposal)" % P if net else ""),
                       "form_params": form_params,
                       "tuning": tuning or None,
                       "tuning_operator": f"48^3 GRF seed {TUNE_SEED} (a training operator)"
                                          if tuning else None,
                       "checkpoint": os.path.relpath(L.CHECKPOINT, ROOT) if have_net else None,
                       "parallelism": f"replicas x{ctx['world']}",
                       "l2": "256 MiB buffer written between timed steps",
                       "value_scope": "numeric factor + proposal on the device + Lanczos, "
                                      "matrix and analysis resident"},
            "ratio_target_over_fp64": tv / forms["fp64"]["value_s"],
            "forms": forms, "proposal_ms": proposal_ms, "check": check, "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e[target], "e2e_fp64": e2e["fp64"],
            "gpu_launches": int(keep[target]["launches"]), "clocks": keep[target]["clocks"],
        }
        print(json.dumps(line))
    return 0


def run_one_form(args, pkg, wl, ctx):
    """One form of the 48^3 GRF metric alone, for profiling launch lists and
    single kernels: --form NAME (fp64, mixed, fp64+learned, mixed+learned,
    fp64+block, mixed+block) with --block / --ncv, W warm-up and K timed
    solves on a resident plan.  Prints one JSON line with the per-solve
    device times and phases; no CPU baseline, no end-to-end leg."""
    import torch
    s, w, L = pkg.speigs, pkg.workloads, pkg.learned
    lib, dev = ctx["lib"], ctx["dev"]
    N, seed = 48, 3200
    A = wl["build"]()
    n, k = A.shape[0], wl["k"]
    name = args.form
    prec = s.MIXED if name.startswith("mixed") else s.FP64
    learned = "learned" in name
    block = -1 if "+" not in name else args.block
    ext = s.ext_opts(lib, precision=prec, block=block)
    Yw = None
    if learned:
        net = L.WarmStartNet.load(L.CHECKPOINT, lib=lib)
        kap = w.grf_conductivity(N, seed)
        rowptr, col, wts = L.grid_graph(N, kap)
        tt = [torch.from_numpy(a).to(dev) for a in (rowptr, col, wts, L.features(N, kap))]
        Y32 = torch.empty((n, net.nout), dtype=torch.float32, device=dev)
        rc = net.forward_device(n, tt[0].data_ptr(), tt[1].data_ptr(), tt[2].data_ptr(),
                                tt[3].data_ptr(), Y32.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise RuntimeError(f"mpnn forward rc={rc}")
        Yw = Y32.t().contiguous().to(torch.float64)
        ext.warm = Yw.data_ptr()
        ext.warm_cols = net.nout
    opts = s.default_opts(lib, tol=TOL, ncv=args.ncv if "+" in name else 0)
    plan = s.Plan(A, s.SM, opts, lib=lib, ext=ext)
    st = torch.cuda.ExternalStream(plan.stream(), device=dev)
    lam = torch.zeros(k, dtype=torch.float64, device=dev)
    V = torch.zeros((k, n), dtype=torch.float64, device=dev)
    res = torch.zeros(k, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ms, info = [], None
    for it in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc, info = plan.solve_device(k, lam.data_ptr(), V.data_ptr(), res.data_ptr())
        e1.record(st)
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(f"{name}: rc={rc} {s.last_error(lib)}")
        if it >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    ei = plan.ext_info()
    costs = plan.costs()
    plan.close()
    print(json.dumps({"form": name, "block": block, "ncv": opts.ncv, "step_ms": ms,
                      "costs": costs,
                      "nops": int(info["nops"]), "restarts": int(info["restarts"]),
                      "flag": int(info["flag"]), "block_solves": int(ei["block_solves"]),
                      "refine_steps": int(ei["refine_steps"]),
                      "phases_ms": {kk: round(info[kk] * 1e3, 3) for kk in
                                    ("t_factor", "t_op", "t_ortho", "t_resid", "t_ritz")}}))
    return 0


def run_batched(args, pkg, wl, rank=0, world=1, local=0):
    """k eigenpairs of every component through speigs_batched -- the
    components on the Krylov route solved together by the segmented lockstep
    Lanczos (one forest-wide factorization, one solve launch per step for all
    of them) -- end to end from host CSC arrays.  With N ranks the components
    are split by estimated cost (shard.assign), each rank solves its share on
    its own GPU with no collective on the data path, the step time is the
    maximum over the ranks, and the per-component results are gathered once
    after the timed region.  The reference's CPU solver is timed on a sample
    stratified by component size: the components sorted by size, every
    `stride`-th one solved once by the reference's own speigs(), each sampled
    time standing for the `stride` components of its stratum."""
    s = pkg.speigs
    shard = pkg.shard
    lib = s.load()
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    t0 = time.perf_counter()
    A = wl["build"]()
    t_build = time.perf_counter() - t0
    n, k = A.shape[0], wl["k"]
    opts = s.default_opts(lib, tol=TOL)
    ncomp, comp = s.components(A, lib)
    sizes = np.bincount(comp, minlength=ncomp)
    mine = shard.assign(sizes, world)[rank]
    if world > 1:
        Aloc, _, comp_loc = shard.submatrix(A, comp, mine)
    else:
        Aloc, comp_loc = A, comp

    def solve():
        if len(mine) == 0:
            return 0, None
        rc, lam, V, res, nv, info = s.speigs_batched(Aloc, k, s.SM, opts, comp=comp_loc, lib=lib)
        if rc != 0:
            raise RuntimeError(f"batched rc={rc} {s.last_error(lib)}")
        return rc, (lam, res, nv, info)

    def tmax(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        solve()
    ts = []
    c0 = s.counters(lib)
    phases = []
    for _ in range(args.steps):
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        _, out = solve()
        ts.append(tmax(time.perf_counter() - t0))
        if out is not None:
            phases.append(s.batched_stats(lib))
    c1 = s.counters(lib)
    launches = tmax((c1[0] - c0[0]) // args.steps)
    h2d = tmax((c1[1] - c0[1]) // args.steps)
    d2h = tmax((c1[2] - c0[2]) // args.steps)
    local_res = {"lam": np.zeros((0, k)), "res": np.zeros((0, k)),
                 "nv": np.zeros(0, dtype=np.int64), "flag": np.zeros(0, dtype=np.int64),
                 "nops": np.zeros(0, dtype=np.int64)}
    if out is not None:
        lam_l, res_l, nv_l, info = out
        local_res = {"lam": lam_l, "res": res_l, "nv": nv_l,
                     "flag": np.full(len(mine), int(info["flag"]), dtype=np.int64),
                     "nops": np.full(len(mine), int(info["nops"]), dtype=np.int64)}
    allr = shard.gather(local_res, mine, ncomp, dist)
    lam = allr["lam"]
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    cpu, check = None, {"flag": int(allr["flag"].max()), "ncomp": int(ncomp),
                        "min_nvals": int(allr["nv"].min()),
                        "max_resid": float(allr["res"].max())}
    if world == 1:
        check["nops"] = int(allr["nops"].max())
    if os.path.exists(REF_LIB) and not args.no_cpu_baseline:
        ref = s.load(REF_LIB)
        o = s.default_opts(ref, tol=TOL)
        Ad = A.tocsr()
        order = np.argsort(sizes, kind="stable")
        stride = max(1, len(order) // 128)
        t_est, sampled, worst, nodes = 0.0, 0, 0.0, 0
        for q in range(0, len(order), stride):
            c = order[q]
            rows = np.flatnonzero(comp == c)
            weight = min(stride, len(order) - q)
            kc = min(k, len(rows))
            Ac = Ad[rows][:, rows].tocsc()
            t1 = time.perf_counter()
            rr, rlam, *_ = s.speigs(Ac, kc, s.SM, o, vectors=True, lib=ref)
            t_est += (time.perf_counter() - t1) * weight
            sampled += 1
            nodes += len(rows)
            if rr == 0:
                worst = max(worst, float(np.max(np.abs(lam[c, :kc] - rlam) / np.abs(rlam))))
        cpu = {"value": t_est, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
               "sample": f"{sampled} components ({nodes} nodes), every {stride}-th by size, each "
                         f"solved once by the reference's src/speigs_core.c (CHOLMOD stand-in + "
                         f"OpenBLAS, all host threads); each sampled time weighted by its "
                         f"stratum's {stride} components"}
        check["max_eig_rel_err_vs_reference_on_sample"] = worst
    v = statistics.mean(ts)
    line = {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
        "higher_is_better": False, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "n": int(n), "nnz": int(A.nnz), "ncomp": int(ncomp),
                   "k": k, "tol": TOL, "form": "batched (speigs_batched, segmented lockstep "
                   "Lanczos over the Krylov-route components)",
                   "value_scope": "end to end: host CSC in, per-component results out; with N "
                                  "ranks each rank's share of the components (split by "
                                  "estimated cost before the timed region), max over ranks",
                   "parallelism": f"components sharded over {world} GPU(s), no collective on "
                                  "the data path",
                   "l2": "inputs copied from the host every step",
                   "matrix_build_s": t_build},
        "check": check, "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "step_s": [round(x, 4) for x in ts],
        "phases_rank0": phases[-1] if phases else None,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="grf48")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default=None,
                    help="time this form of the 48^3 GRF metric alone (profiling): fp64, mixed, "
                         "fp64+learned, mixed+learned, fp64+block, mixed+block")
    ap.add_argument("--block", type=int, default=8, help="block size of --form's block forms")
    ap.add_argument("--ncv", type=int, default=96, help="basis size of --form's block forms")
    ap.add_argument("--no-tune", action="store_true",
                    help="learned forms with the automatic block method instead of the block "
                         "and basis sizes the tuner picks on a training operator")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="operator of the timed line: plain FP64 factor, or FP32 factor on the "
                         "tensor cores with FP64 refinement")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the side-by-side measurement of the other precision")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pkg = import_pkg()
    s, w = pkg.speigs, pkg.workloads
    wl = workloads(w, s)[args.workload]

    if args.impl == "reference":
        return run_reference(args, pkg, wl, rank)
    if args.workload in ("rgg", "rgg256"):
        return run_batched(args, pkg, wl, rank, world, local)

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = s.load()
    if args.workload == "grf48":
        def barrier():
            if world > 1:
                dist.barrier()

        def tmax(t):
            if world > 1:
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ctx = {"lib": lib, "dev": dev, "rank": rank, "world": world, "barrier": barrier,
               "max": tmax}
        rc = run_one_form(args, pkg, wl, ctx) if args.form else run_metric(args, pkg, wl, ctx)
        if world > 1:
            dist.destroy_process_group()
        return rc

    A = wl["build"]()
    n, k = A.shape[0], wl["k"]
    opts = s.default_opts(lib, tol=TOL)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peak, peak_kind = measured_peaks()

    def measure(precision, steps, with_clocks):
        """Time `steps` full solves of one form on the device, then its operator,
        then the drop-in call end to end."""
        prec = s.MIXED if precision == "mixed" else s.FP64
        ext = s.ext_opts(lib, precision=prec)
        plan = s.Plan(A, wl["which"], opts, lib=lib, ext=ext)
        pstream = torch.cuda.ExternalStream(plan.stream(), device=dev)
        lam = torch.zeros(k, dtype=torch.float64, device=dev)
        V = torch.zeros((k, n), dtype=torch.float64, device=dev)    # column-major n x k
        res = torch.zeros(k, dtype=torch.float64, device=dev)

        def solve():
            rc, info = plan.solve_device(k, lam.data_ptr(), V.data_ptr(), res.data_ptr())
            if rc != 0:
                raise RuntimeError(f"solve rc={rc}: {s.last_error(lib)}")
            return info

        torch.cuda.synchronize()
        for _ in range(args.warmup):
            info = solve()
        # ---- timed region: device time per solve, L2 flushed between steps
        sampler = ClockSampler()
        if with_clocks:
            sampler.start()
            sampler.ready()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = s.counters(lib)[0]
        step_ms, step_phase = [], []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(pstream)
            info = solve()
            e1.record(pstream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            step_phase.append([round(info["t_factor"], 4), round(info["t_iter"], 4)])
        torch.cuda.synchronize()
        launches = (s.counters(lib)[0] - l0) // max(steps, 1)
        if world > 1:
            dist.barrier()
        clocks = sampler.stop(gpu_index=None) if with_clocks else None
        einfo = plan.ext_info()
        ms = statistics.mean(step_ms)
        lam_h = lam.cpu().numpy()
        Vh = V.cpu().numpy().T

        # ---- the operator (the dominant kernel: the solve pair, or the SpMV)
        costs = plan.costs()
        x = torch.randn(n, dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        for _ in range(3):
            plan.apply_device(x.data_ptr(), y.data_ptr())
        op_ms = []
        for _ in range(20):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(pstream)
            plan.apply_device(x.data_ptr(), y.data_ptr())
            e1.record(pstream)
            e1.synchronize()
            op_ms.append(e0.elapsed_time(e1))
        plan.close()

        # ---- end to end through the drop-in API: host CSC in, host results out
        # (untimed warm-up calls first, as for the device timing)
        for _ in range(args.warmup):
            rc, *_ = s.speigs_ex(A, k, wl["which"], opts, ext, vectors=True, lib=lib)
        e2e_t, e2e_lib = [], []
        c0 = s.counters(lib)
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc, l2, V2, r2, inf2, ei2 = s.speigs_ex(A, k, wl["which"], opts, ext, vectors=True,
                                                    lib=lib)
            e2e_t.append(time.perf_counter() - t0)
            e2e_lib.append([round(v, 4) for v in (inf2["t_analyze"], ei2["t_checks"],
                                                  ei2["t_setup"], inf2["t_factor"],
                                                  inf2["t_iter"], ei2["t_release"])])
            if rc != 0:
                raise RuntimeError(f"speigs rc={rc}")
        c1 = s.counters(lib)
        e2e = {"value": statistics.mean(e2e_t), "unit": "s",
               "h2d_bytes_per_step": (c1[1] - c0[1]) // steps,
               "d2h_bytes_per_step": (c1[2] - c0[2]) // steps,
               "steps_s": [round(x, 4) for x in e2e_t],
               "steps_inside_library_s": {
                   "fields": ["analyze", "checks", "setup", "factor", "iterate", "release"],
                   "steps": e2e_lib},
               "phase_s": dict({kk: inf2[kk] for kk in ("t_analyze", "t_factor", "t_iter")},
                            **{kk: ei2[kk] for kk in ("t_checks", "t_setup", "t_release")})}
        return dict(ms=ms, step_ms=step_ms, step_phase=step_phase, info=info, einfo=einfo,
                    lam=lam_h, V=Vh,
                    launches=launches, clocks=clocks, costs=costs,
                    op_s=statistics.mean(op_ms) * 1e-3, e2e=e2e)

    main_m = measure(args.precision, args.steps, True)
    t = torch.tensor([main_m["ms"]], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    info = main_m["info"]

    # ---- correctness of the timed result
    lam_h, Vh = main_m["lam"], main_m["V"]
    resid = np.linalg.norm(A @ Vh - Vh * lam_h, axis=0)
    check = {"max_resid_over_anorm": float(resid.max() / info["anorm"]),
             "nops": int(info["nops"]), "restarts": int(info["restarts"]),
             "shift": info["shift"], "flag": int(info["flag"]),
             "refine_steps": int(main_m["einfo"]["refine_steps"])}
    if wl["exact"] is not None:
        ex = wl["exact"]()
        check["max_rel_err_vs_closed_form"] = float(np.max(np.abs(lam_h - ex) / np.abs(ex)))

    # ---- roofline of the dominant kernel: the operator application.  For
    # the mixed form the algorithmic bytes are those of every FP32 solve pair
    # and FP64 residual the refined application performs.
    costs = main_m["costs"]
    op_bytes = costs["op_bytes"]
    if args.precision == "mixed" and info["nops"] > 0:
        per_app = 1.0 + main_m["einfo"]["refine_steps"] / info["nops"]
        nnz = float(A.nnz)
        op_bytes = costs["op_bytes"] * per_app + per_app * (12.0 * nnz + 40.0 * n)
    achieved = op_bytes / main_m["op_s"] / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"{args.workload}:{args.precision}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": ("shift-invert solve pair (task-queue multifrontal solve)"
                           + (", FP32 panels + FP64 refinement" if args.precision == "mixed" else ""))
                if wl["which"] == s.SM else "CSR SpMV",
                "op_ms": main_m["op_s"] * 1e3, "op_bytes": op_bytes, "peak_source": peak_kind}

    # ---- the other precision on the same workload, same B200 (the metric's
    # comparison), with the per-eigenpair error between the two forms
    compare = None
    if wl["which"] == s.SM and not args.no_compare and world == 1:
        other = "mixed" if args.precision == "fp64" else "fp64"
        om = measure(other, max(2, min(args.steps, 3)), False)
        fp64_lam = om["lam"] if other == "fp64" else lam_h
        mixed_lam = lam_h if other == "fp64" else om["lam"]
        compare = {"precision": other, "value": om["ms"] * 1e-3, "unit": "s",
                   "step_ms": [round(x, 3) for x in om["step_ms"]],
                   "step_factor_iterate_s": om["step_phase"],
                   "e2e": om["e2e"]["value"], "nops": int(om["info"]["nops"]),
                   "refine_steps": int(om["einfo"]["refine_steps"]),
                   "mixed_over_fp64_value": (om["ms"] / ms) if other == "mixed" else (ms / om["ms"]),
                   "eig_rel_err_mixed_vs_fp64": [float(abs(a - b) / abs(b))
                                                 for a, b in zip(mixed_lam, fp64_lam)]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
        times, _, _ = cpu_reference_times(pkg, A, wl, steps=3, warmup=1, budget_s=30.0)
        cpu = {"value": statistics.median(times), "unit": "s", "cores": os.cpu_count(),
               "kind": "reference",
               "sample": f"{len(times)} full solve(s) of the same workload by the reference's "
                         "src/speigs_core.c (CHOLMOD stand-in + OpenBLAS, all host threads), "
                         "median"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms * 1e-3, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else
                     "f32 factor panels, f64 refinement / recurrence / Ritz",
            "data": "synthetic",
            "config": {"workload": wl["desc"], "n": int(n), "nnz": int(A.nnz), "k": k, "tol": TOL,
                       "precision": "plain FP64" if args.precision == "fp64" else
                       "mixed: FP32 factor (TF32 tensor-core updates) + FP64 refinement",
                       "parallelism": f"replicas x{world}",
                       "l2": "256 MiB buffer written between timed steps",
                       "value_scope": "numeric factor + Lanczos, matrix and analysis resident"},
            "check": check, "roofline": roofline, "cpu_baseline": cpu, "e2e": main_m["e2e"],
            "gpu_launches": int(main_m["launches"]), "clocks": main_m["clocks"],
            "step_ms": [round(x, 3) for x in main_m["step_ms"]],
            "step_factor_iterate_s": main_m["step_phase"],
            "phase_s": {kk: info[kk] for kk in ("t_factor", "t_iter", "t_op", "t_ortho",
                                                "t_resid", "t_ritz")},
            "compare": compare,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
