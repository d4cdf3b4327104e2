"""Sharding the batched form across GPUs (one process per GPU).

The components of a block-diagonal matrix are independent, so N ranks split
them with no collective on the data path: each rank solves its share with
speigs_batched on its own GPU, and only the per-component results (k values,
residuals and counts per component) are gathered at the end.  The split is
the longest-processing-time rule on an estimated cost per component
(n_c^1.5, the growth of a 3-D nested-dissection factor's work): components in
decreasing cost, each to the rank with the least cost so far, ties to the
lower rank -- deterministic, so every rank computes the same split without
communicating.
"""
from __future__ import annotations

import numpy as np


def component_cost(sizes: np.ndarray) -> np.ndarray:
    """Estimated solve cost of components of the given sizes."""
    return np.asarray(sizes, dtype=np.float64) ** 1.5


def assign(sizes, world: int) -> list[np.ndarray]:
    """Component indices per rank (each list ascending)."""
    sizes = np.asarray(sizes)
    cost = component_cost(sizes)
    order = np.lexsort((np.arange(len(sizes)), -cost))     # decreasing cost, then index
    load = np.zeros(world)
    parts: list[list[int]] = [[] for _ in range(world)]
    for c in order:
        r = int(np.argmin(load))                           # first minimum: lowest rank
        parts[r].append(int(c))
        load[r] += cost[c]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def submatrix(A, comp: np.ndarray, mine: np.ndarray):
    """The rows and columns of the components in `mine` (ascending row order),
    with their labels renumbered 0..len(mine)-1 in the order of `mine`."""
    keep = np.isin(comp, mine)
    rows = np.flatnonzero(keep)
    sub = A.tocsr()[rows][:, rows].tocsc()
    sub.sort_indices()
    relabel = np.full(int(comp.max()) + 1, -1, dtype=np.int64)
    relabel[mine] = np.arange(len(mine))
    return sub, rows, relabel[comp[rows]]


def gather(local: dict, mine: np.ndarray, ncomp: int, dist=None):
    """Merge per-component results into component order on every rank.

    local: arrays with the rank's components along axis 0 (in the order of
    `mine`); returns the same keys with all ncomp components.  With dist
    (torch.distributed, any backend) the ranks' pieces are exchanged with
    all_gather_object; without it the single rank's result is placed."""
    pieces = [(mine, local)]
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        allp = [None] * dist.get_world_size()
        dist.all_gather_object(allp, (mine, local))
        pieces = allp
    out = {}
    for idx, loc in pieces:
        for key, val in loc.items():
            val = np.asarray(val)
            if key not in out:
                out[key] = np.zeros((ncomp,) + val.shape[1:], dtype=val.dtype)
            out[key][idx] = val
    return out
