#!/usr/bin/env python
"""Train the learned warm start on eigenvectors this solver computes.

Family: 3-D finite-volume diffusion operators on an N^3 grid whose cell
conductivity is exp of a Gaussian random field (squared-exponential
covariance, correlation length 0.1, variance 1), seeds 1000, 1001, ...
For every instance the plain FP64 solver (one plan, one symbolic analysis,
new values per instance) computes the k smallest eigenpairs; the network
(learned.WarmStartNet, BF16 kernels of csrc/kernels/mpnn.cu) is trained to
make the span of its P outputs hold those eigenvectors.  Held-out instances
then measure what the proposal buys: operator applications and device time
of the Lanczos with the learned start, with the closed-form Laplace modes as
start, and with the reference's random start.

  python train_warmstart.py --N 48 --ntrain 2000 --nheld 200 --k 16 \
      --out data/warmstart_grf48.npz --report report.json
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def import_pkg():
    if "speigs_b200" in sys.modules:
        return sys.modules["speigs_b200"]
    spec = importlib.util.spec_from_file_location(
        "speigs_b200", os.path.join(HERE, "__init__.py"), submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["speigs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def grf_field(N, seed, torch, dev, corr_len=0.1, variance=1.0):
    """workloads.grf_conductivity with the FFTs on the GPU (same noise stream)."""
    rng = np.random.default_rng(seed)
    M = 2 * N
    k = 2.0 * np.pi * np.fft.fftfreq(M, d=1.0 / N)
    noise = torch.from_numpy(rng.standard_normal((M, M, M))).to(dev)
    kk = torch.from_numpy(k).to(dev)
    kx, ky, kz = torch.meshgrid(kk, kk, kk, indexing="ij")
    spec = torch.exp(-0.5 * corr_len ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    g = torch.fft.ifftn(torch.fft.fftn(noise) * torch.sqrt(spec)).real[:N, :N, :N]
    g = (g - g.mean()) / g.std() * np.sqrt(variance)
    return torch.exp(g).cpu().numpy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=48)
    ap.add_argument("--ntrain", type=int, default=2000)
    ap.add_argument("--nheld", type=int, default=200)
    ap.add_argument("--neval", type=int, default=20, help="held-out instances solved 3 ways")
    ap.add_argument("--k", type=int, default=16)
    ap.add_argument("--nout", type=int, default=24)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--out", default=os.path.join(HERE, "data", "warmstart_grf48.npz"))
    ap.add_argument("--report", default=None)
    args = ap.parse_args()

    import torch
    pkg = import_pkg()
    s, w, L = pkg.speigs, pkg.workloads, pkg.learned
    dev = torch.device("cuda")
    lib = s.load()
    N, k, n = args.N, args.k, args.N ** 3
    pat = w.FVPattern(N)
    opts = s.default_opts(lib, tol=args.tol)
    plan = s.Plan(pat.A, s.SM, opts, lib=lib)
    lam = torch.zeros(k, dtype=torch.float64, device=dev)
    V = torch.zeros((k, n), dtype=torch.float64, device=dev)
    res = torch.zeros(k, dtype=torch.float64, device=dev)
    rowptr, col, _ = L.grid_graph(N, np.ones((N, N, N)))
    t_rp = torch.from_numpy(rowptr).to(dev)
    t_ci = torch.from_numpy(col).to(dev)

    total = args.ntrain + args.nheld
    Ws = torch.empty((total, len(col)), dtype=torch.float32, device=dev)
    Xs = torch.empty((total, n, 1 + L.NMODES), dtype=torch.float32, device=dev)
    Us = torch.empty((total, n, k), dtype=torch.float32, device=dev)
    kaps = []
    t0 = time.time()
    nops_plain = []
    for i in range(total):
        kap = grf_field(N, 1000 + i, torch, dev)
        if i >= args.ntrain:
            kaps.append(kap)
        plan.set_values(pat.values(kap))
        rc, info = plan.solve_device(k, lam.data_ptr(), V.data_ptr(), res.data_ptr())
        if rc != 0:
            raise RuntimeError(f"solve {i}: rc={rc} {s.last_error(lib)}")
        nops_plain.append(info["nops"])
        torch.cuda.synchronize()
        Us[i] = V.t().float()
        _, _, wv = L.grid_graph(N, kap)
        Ws[i] = torch.from_numpy(wv).to(dev)
        Xs[i] = torch.from_numpy(L.features(N, kap)).to(dev)
    t_data = time.time() - t0

    net = L.WarmStartNet(nout=args.nout, layers=args.layers, seed=7, lib=lib)
    steps = args.epochs * args.ntrain
    hist = []
    t0 = time.time()
    rng = np.random.default_rng(0)
    step = 0
    for ep in range(args.epochs):
        order = rng.permutation(args.ntrain)
        el = []
        for i in order:
            lr = args.lr * 0.5 * (1.0 + np.cos(np.pi * step / steps))
            loss = net.train_step_device(n, t_rp.data_ptr(), t_ci.data_ptr(), Ws[i].data_ptr(),
                                         Xs[i].data_ptr(), Us[i].data_ptr(), k, float(lr), 0)
            el.append(loss)
            step += 1
        hist.append(float(np.mean(el)))
        print(f"epoch {ep}: mean training loss {hist[-1]:.4f}", flush=True)
    t_train = time.time() - t0
    held = []
    for i in range(args.ntrain, total):
        held.append(net.train_step_device(n, t_rp.data_ptr(), t_ci.data_ptr(), Ws[i].data_ptr(),
                                          Xs[i].data_ptr(), Us[i].data_ptr(), k, 0.0, 0))
    net.save(args.out, N=N, k=k, ntrain=args.ntrain, train_loss=np.array(hist),
             held_loss=float(np.mean(held)))

    # ---- what the proposal buys on held-out operators
    modes = w.laplace_modes(N, args.nout)
    cmp = {"random": [], "laplace": [], "learned": []}
    tms = {"random": [], "laplace": [], "learned": []}
    t_prop = []
    for j, kap in enumerate(kaps[:args.neval]):
        A = pat.matrix(kap)
        tp = time.perf_counter()
        Y = L.propose(net, N, kap)
        t_prop.append(time.perf_counter() - tp)
        ref = None
        for name, warm in (("random", None), ("laplace", modes), ("learned", Y)):
            t1 = time.perf_counter()
            rc, lam_h, V_h, r_h, info, ei = s.speigs_ex(A, k, s.SM, opts, lib=lib, warm=warm,
                                                        vectors=False)
            tms[name].append(time.perf_counter() - t1)
            if rc != 0:
                raise RuntimeError(f"held-out solve {j} ({name}) rc={rc}")
            cmp[name].append(int(info["nops"]))
            if ref is None:
                ref = lam_h
            else:
                assert np.max(np.abs(lam_h - ref) / np.abs(ref)) <= 1e-9
    report = {
        "N": N, "n": n, "k": k, "nout": args.nout, "layers": args.layers,
        "ntrain": args.ntrain, "nheld": args.nheld, "epochs": args.epochs,
        "train_loss_per_epoch": hist, "held_out_loss": float(np.mean(held)),
        "laplace_modes_loss_note": "loss of the closed-form modes is not trained",
        "data_generation_s": t_data, "training_s": t_train,
        "mean_nops_training_solves": float(np.mean(nops_plain)),
        "held_out_eval": {kk: {"mean_nops": float(np.mean(v)), "nops": v,
                               "mean_e2e_s": float(np.mean(tms[kk]))} for kk, v in cmp.items()},
        "mean_proposal_s": float(np.mean(t_prop)) if t_prop else None,
    }
    print(json.dumps(report))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f)
    plan.close()


if __name__ == "__main__":
    main()
