"""One rank of the two-process check of the batched form's sharding (gloo on
CPU).  Each rank takes its share of the components of a block-diagonal
matrix (shard.assign), cuts its submatrix (shard.submatrix), computes the k
smallest eigenvalues of each of its components with a dense solver (the
check's stand-in for the device solve), and the ranks gather the results
(shard.gather).  Every rank compares the gathered table with the same
eigenvalues computed on the whole matrix, component by component, and writes
its verdict to argv[1]."""
import importlib.util
import json
import os
import sys

import numpy as np
import torch.distributed as dist

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
PKG_DIR = os.path.join(ROOT, "sparse-eigs-mex_b200")


def load_pkg():
    spec = importlib.util.spec_from_file_location(
        "speigs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["speigs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def smallest(A, rows, k):
    return np.linalg.eigvalsh(A[rows][:, rows].toarray())[:k]


def main():
    out = sys.argv[1]
    pkg = load_pkg()
    shard, w = pkg.shard, pkg.workloads
    dist.init_process_group("gloo")
    rank, world = dist.get_rank(), dist.get_world_size()
    k = 3
    A = w.rgg_blocks(24, seed=7, nmin=5, nmax=60)
    ncomp, comp = w.components_of(A)
    sizes = np.bincount(comp, minlength=ncomp)
    parts = shard.assign(sizes, world)
    mine = parts[rank]
    sub, rows, lab = shard.submatrix(A, comp, mine)
    Asub = sub.tocsr()
    lam = np.full((len(mine), k), np.nan)
    for j in range(len(mine)):
        r = np.flatnonzero(lab == j)
        v = smallest(Asub, r, k)
        lam[j, :len(v)] = v
    got = shard.gather({"lam": lam, "size": sizes[mine]}, mine, ncomp, dist)
    Ar = A.tocsr()
    want = np.full((ncomp, k), np.nan)
    for c in range(ncomp):
        v = smallest(Ar, np.flatnonzero(comp == c), k)
        want[c, :len(v)] = v
    # the split every rank computed must be the same one
    allparts = [None] * world
    dist.all_gather_object(allparts, [p.tolist() for p in parts])
    ok = bool(np.array_equal(got["lam"], want, equal_nan=True)
              and np.array_equal(got["size"], sizes)
              and all(a == allparts[0] for a in allparts)
              and len(rows) == int(sizes[mine].sum()))
    dist.destroy_process_group()
    with open(out, "w") as f:
        json.dump({"rank": rank, "ok": ok, "ncomp": int(ncomp), "mine": len(mine)}, f)


if __name__ == "__main__":
    main()
