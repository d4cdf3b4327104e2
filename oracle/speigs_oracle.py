"""ORACLE TEST INFRASTRUCTURE -- a CPU restatement of the reference solver.

Not part of the shipped library: only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module, and only as a checker.

numpy/scipy restatement of moatas19m/sparse-eigs-mex src/speigs_core.c for
the 'sm' / 'lm' Krylov path, function by function:

  rng_next / rand_vec      :49-54   xorshift64*, uniform in [-0.5, 0.5)
  orth_block               :122-132 CGS2 (DGKS), projection coefficients
                                    accumulated into the H column
  lanczos                  :146-315 thick restart, breakdown re-injection,
                                    Rayleigh-Ritz, true residuals vs A
  check_symmetry           :363-401
  find_components          :445-466
  speigs (Krylov route)    :783-1024 minus the diag/dense/banded/LU routes

The shift-invert operator uses scipy's sparse LU of A + delta*I (the
reference uses CHOLMOD; the factorization method only changes rounding), with
the reference's capped shift escalation decided by a sparse Cholesky-style
test: the LU pivots of an SPD matrix factored without pivoting must be
positive.  Meant for small sizes: it is plain Python loops over the basis.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

MASK = (1 << 64) - 1
DEFAULT_SEED = 88172645463325252


def rng_next(s: int) -> tuple[int, int]:
    """One xorshift64* step (speigs_core.c:49-51): returns (new state, output)."""
    x = s
    x ^= x >> 12
    x ^= (x << 25) & MASK
    x ^= x >> 27
    return x, (x * 0x2545F4914F6CDD1D) & MASK


def rand_vec(s: int, n: int) -> tuple[int, np.ndarray]:
    """n draws, (out >> 11) / 2^53 - 0.5 (speigs_core.c:52-54)."""
    v = np.empty(n)
    for i in range(n):
        s, out = rng_next(s)
        v[i] = float(out >> 11) / 9007199254740992.0 - 0.5
    return s, v


def orth_block(B: np.ndarray, w: np.ndarray, hout: np.ndarray | None = None) -> np.ndarray:
    """w <- (I - B B^T) w twice (speigs_core.c:122-132)."""
    if B.shape[1] == 0:
        return w
    for _ in range(2):
        tmp = B.T @ w
        w = w - B @ tmp
        if hout is not None:
            hout += tmp
    return w


def check_symmetry(A: sp.csc_matrix) -> int:
    """1 full symmetric, 2 upper only, 3 lower only, 0 not symmetric (:363-401)."""
    A = A.tocoo()
    up = bool(np.any(A.row < A.col))
    lo = bool(np.any(A.row > A.col))
    if up and not lo:
        return 2
    if lo and not up:
        return 3
    if not up and not lo:
        return 1
    C = A.tocsc()
    T = C.T.tocsc()
    C.sort_indices()
    T.sort_indices()
    if not (np.array_equal(C.indptr, T.indptr) and np.array_equal(C.indices, T.indices)):
        return 0
    m = np.maximum(np.abs(C.data), np.abs(T.data))
    return 1 if np.all(np.abs(C.data - T.data) <= 1e-12 * np.where(m > 0, m, 1.0)) else 0


def find_components(A: sp.csc_matrix) -> tuple[int, np.ndarray]:
    """Connected components over numerically nonzero entries (:445-466)."""
    C = A.tocoo()
    keep = C.data != 0.0
    G = sp.coo_matrix((np.ones(keep.sum()), (C.row[keep], C.col[keep])), shape=A.shape)
    nc, lab = sp.csgraph.connected_components(G, directed=False)
    # relabel in order of first appearance, as the reference does
    order = {}
    out = np.empty_like(lab)
    for i, l in enumerate(lab):
        if l not in order:
            order[l] = len(order)
        out[i] = order[l]
    return nc, out


def symmetric_from_upper(A: sp.csc_matrix) -> sp.csc_matrix:
    """The matrix the reference actually uses: stype=1 reads the upper triangle."""
    U = sp.triu(A, format="csc")
    return (U + sp.triu(U, 1).T).tocsc()


def norm1(A: sp.csc_matrix) -> float:
    return float(np.abs(A).sum(axis=0).max()) if A.nnz else 0.0


def _is_pd(A: sp.csc_matrix) -> bool:
    """Positive-definiteness test standing in for CHOLMOD's NOT_POSDEF status."""
    n = A.shape[0]
    if n <= 3000:
        try:
            sla.cholesky(A.toarray(), lower=True)
            return True
        except np.linalg.LinAlgError:
            return False
    lu = spla.splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                   options={"SymmetricMode": True})
    return bool(np.all(lu.U.diagonal() > 0))


def lanczos(apply, multA, n: int, k: int, anorm: float, tol=0.0, maxit=0, ncv=0,
            seed=0) -> dict:
    """Thick-restart Lanczos with full reorthogonalisation (:146-315)."""
    ncv = ncv if ncv else max(2 * k + 1, 20)
    if ncv > n:
        ncv = n
    if ncv <= k:
        ncv = min(n, k + 1)
    if ncv < 2:
        ncv = min(n, 2)
    maxit = maxit if maxit else 300
    tol = tol if tol > 0 else 1e-14
    rtol = tol * max(anorm, 1.0)
    bthr = 1e-13 * max(anorm, 1.0)
    s = seed if seed else DEFAULT_SEED
    V = np.zeros((n, ncv + 1))
    H = np.zeros((ncv, ncv))
    s, w = rand_vec(s, n)
    nr = np.linalg.norm(w)
    V[:, 0] = w * (1.0 / nr)
    j = restarts = nconv = nops = 0
    lam = np.zeros(k)
    res = np.zeros(k)
    X = np.zeros((n, k))
    while True:
        while j < ncv:
            w = apply(V[:, j])
            nops += 1
            H[: j + 1, j] = 0.0
            hcol = np.zeros(j + 1)
            w = orth_block(V[:, : j + 1], w, hcol)
            H[: j + 1, j] = hcol
            beta = np.linalg.norm(w)
            beta_rec = beta
            if beta <= bthr:
                beta_rec = 0.0
                att = 0
                while att < 3 and beta <= bthr:
                    s, w = rand_vec(s, n)
                    w = orth_block(V[:, : j + 1], w)
                    beta = np.linalg.norm(w)
                    att += 1
                if beta <= bthr:
                    ncv = j + 1
                    break
            V[:, j + 1] = w * (1.0 / beta)
            if j + 1 < ncv:
                H[j + 1, j] = H[j, j + 1] = beta_rec
            j += 1
        m = ncv
        Hs = np.triu(H[:m, :m]) + np.triu(H[:m, :m], 1).T
        theta, S = np.linalg.eigh(Hs)
        ordr = sorted(range(m), key=lambda i: -abs(theta[i]))
        nconv = 0
        nwant = min(k, m)
        for t in range(nwant):
            x = V[:, :m] @ S[:, ordr[t]]
            xn = np.linalg.norm(x)
            if xn > 0:
                x = x * (1.0 / xn)
            Ax = multA(x)
            la = float(x @ Ax)
            r = float(np.linalg.norm(Ax - la * x))
            X[:, t] = x
            lam[t] = la
            res[t] = r
            if r <= rtol:
                nconv += 1
        if nconv >= min(k, m) or restarts >= maxit or m < ncv:
            break
        restarts += 1
        l = max(1, min(k + 5, ncv - 1))
        Vn = np.zeros((n, ncv + 1))
        ths = []
        nret = 0
        for t in range(m):
            if nret >= l:
                break
            i = ordr[t]
            v = V[:, :m] @ S[:, i]
            v = orth_block(Vn[:, :nret], v)
            nr = np.linalg.norm(v)
            if nr < 1e-10:
                continue
            Vn[:, nret] = v * (1.0 / nr)
            ths.append(theta[i])
            nret += 1
        w = orth_block(Vn[:, :nret], V[:, m].copy())
        nr = np.linalg.norm(w)
        if nr < 1e-10:
            s, w = rand_vec(s, n)
            w = orth_block(Vn[:, :nret], w)
            nr = np.linalg.norm(w)
        if nr < 1e-10:
            break
        Vn[:, nret] = w * (1.0 / nr)
        V = Vn
        H = np.zeros((ncv, ncv))
        H[np.arange(nret), np.arange(nret)] = ths
        j = nret
    return {"lam": lam[:nwant].copy(), "resid": res[:nwant].copy(), "V": X[:, :nwant].copy(),
            "nconv": nconv, "restarts": restarts, "nops": nops,
            "flag": 0 if nconv >= min(k, ncv) else 1}


def speigs(A: sp.spmatrix, k: int, which: str = "sm", tol=0.0, maxit=0, ncv=0, seed=0,
           shift0=0.0) -> dict:
    """The Krylov route of speigs() for a connected matrix (:829-1012)."""
    A = symmetric_from_upper(sp.csc_matrix(A))
    n = A.shape[0]
    anorm = norm1(A)
    if anorm <= 0:
        anorm = 1.0
    multA = lambda x: A @ x  # noqa: E731
    shift = 0.0
    if which == "lm":
        apply, path = multA, 3
    else:
        I = sp.identity(n, format="csc")
        if not _is_pd(A):
            d0 = anorm * (shift0 if shift0 > 0 else 1e-6)
            dcap = max(anorm * 1e-3, d0)
            shift = d0
            ok = False
            while shift <= dcap * 1.0000001:
                if _is_pd((A + shift * I).tocsc()):
                    ok = True
                    break
                shift *= 10.0
            if not ok:
                raise ValueError("indefinite: the LU route is outside this restatement")
        lu = spla.splu((A + shift * I).tocsc())
        apply, path = lu.solve, 2
    out = lanczos(apply, multA, n, k, anorm, tol, maxit, ncv, seed)
    key = np.abs(out["lam"])
    order = np.argsort(key, kind="stable") if which == "sm" else np.argsort(-key, kind="stable")
    out["lam"] = out["lam"][order]
    out["resid"] = out["resid"][order]
    out["V"] = out["V"][:, order]
    out.update(path=path, shift=shift, anorm=anorm)
    return out
