"""Sharding of the batched form over ranks: the cost-balanced split, the
per-rank submatrix, and the gather of per-component results across two gloo
ranks on the CPU (the path bench.py --workload rgg takes with N GPUs)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_assign_is_a_balanced_partition(pkg):
    shard = pkg.shard
    rng = np.random.default_rng(3)
    sizes = rng.integers(1, 5000, size=4096)
    cost = shard.component_cost(sizes)
    for world in (1, 2, 3, 8):
        parts = shard.assign(sizes, world)
        assert len(parts) == world
        allc = np.sort(np.concatenate(parts))
        assert np.array_equal(allc, np.arange(len(sizes)))
        loads = np.array([cost[p].sum() for p in parts])
        # longest-processing-time bound: no rank exceeds the mean by more
        # than one component's cost
        assert loads.max() <= cost.sum() / world + cost.max()
        again = shard.assign(sizes, world)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def test_assign_more_ranks_than_components(pkg):
    parts = pkg.shard.assign(np.array([10, 20]), 4)
    assert [len(p) for p in parts] == [1, 1, 0, 0]
    assert parts[0][0] == 1          # the costlier component goes first, to rank 0


def test_submatrix_keeps_components_whole(pkg):
    shard, w = pkg.shard, pkg.workloads
    A = w.rgg_blocks(12, seed=5, nmin=5, nmax=40)
    ncomp, comp = w.components_of(A)
    mine = shard.assign(np.bincount(comp), 3)[1]
    sub, rows, lab = shard.submatrix(A, comp, mine)
    assert np.array_equal(rows, np.flatnonzero(np.isin(comp, mine)))
    assert sub.shape == (len(rows), len(rows))
    assert abs(sub).sum() == abs(A.tocsr()[rows][:, rows]).sum()
    nsub, csub = w.components_of(sub)
    assert nsub == len(mine)
    # same partition of the rows, labels renumbered in the order of `mine`
    for j, c in enumerate(mine):
        assert np.array_equal(lab == j, comp[rows] == c)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gather_two_gloo_ranks(tmp_path):
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "host", "shard_rank.py"),
                                       str(tmp_path / f"r{r}.json")], env=env))
    for p in procs:
        assert p.wait(timeout=300) == 0
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert all(x["ok"] for x in res)
    assert sum(x["mine"] for x in res) == res[0]["ncomp"]
