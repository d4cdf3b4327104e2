"""Seeded synthetic operators for the solver's workloads and tests.

The Laplacians follow the reference's own builders (test/test_speigs.c:31-47
lap3d: 7-point stencil, x fastest, Dirichlet diagonal 6 or Neumann diagonal
= degree) and closed-form spectra (:53-62).  The variable-coefficient
finite-volume operator is the one named for the mixed-precision workload:
cell conductivities log-normal, face transmissibility the harmonic mean
2 k_i k_j / (k_i + k_j), Dirichlet boundary faces 2 k_i.
All matrices are returned as scipy CSC with both triangles and sorted rows.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _lap1d(N: int, dirichlet: bool) -> sp.csr_matrix:
    main = np.full(N, 2.0)
    if not dirichlet:
        main[0] = main[-1] = 1.0
        if N == 1:
            main[0] = 0.0
    off = -np.ones(N - 1)
    return sp.diags([off, main, off], [-1, 0, 1], format="csr")


def lap3d(N: int, dirichlet: bool = True) -> sp.csc_matrix:
    """3-D 7-point Laplacian on an N^3 grid (Dirichlet: diag 6; Neumann: degree)."""
    L = _lap1d(N, dirichlet)
    I = sp.identity(N, format="csr")
    A = sp.kron(I, sp.kron(I, L)) + sp.kron(I, sp.kron(L, I)) + sp.kron(L, sp.kron(I, I))
    A = A.tocsc()
    A.sort_indices()
    A.eliminate_zeros()
    return A


def lap2d(N: int) -> sp.csc_matrix:
    """2-D 5-point Dirichlet Laplacian (diag 4) on an N^2 grid."""
    L = _lap1d(N, True)
    I = sp.identity(N, format="csr")
    A = (sp.kron(I, L) + sp.kron(L, I)).tocsc()
    A.sort_indices()
    return A


def lap1d(n: int) -> sp.csc_matrix:
    A = _lap1d(n, True).tocsc()
    A.sort_indices()
    return A


def spectrum3d(N: int, dirichlet: bool = True) -> np.ndarray:
    """All eigenvalues of lap3d(N), ascending (reference exact_spectrum)."""
    p = np.arange(N)
    e1 = 2.0 - 2.0 * np.cos((p + 1) * np.pi / (N + 1)) if dirichlet else \
        2.0 - 2.0 * np.cos(p * np.pi / N)
    return np.sort((e1[:, None, None] + e1[None, :, None] + e1[None, None, :]).ravel())


def spectrum2d_extreme(N: int, k: int, largest: bool) -> np.ndarray:
    """k smallest (or largest) eigenvalues of lap2d(N) from the closed form."""
    p = np.arange(1, N + 1)
    e1 = 2.0 - 2.0 * np.cos(p * np.pi / (N + 1))
    e1 = np.sort(e1)
    m = min(N, k + 2)
    cand = (e1[-m:][:, None] + e1[-m:][None, :]).ravel() if largest else \
        (e1[:m][:, None] + e1[:m][None, :]).ravel()
    cand = np.sort(cand)
    return cand[::-1][:k] if largest else cand[:k]


def varcoef3d(N: int, seed: int = 3, sigma: float = 1.0) -> sp.csc_matrix:
    """3-D finite-volume diffusion operator with log-normal cell conductivity."""
    rng = np.random.default_rng(seed)
    kap = np.exp(sigma * rng.standard_normal((N, N, N)))   # index [z, y, x]
    return _fv_operator(kap)


def grf_conductivity(N: int, seed: int, corr_len: float = 0.1, variance: float = 1.0) -> np.ndarray:
    """kappa = exp(g) on an N^3 cell grid, g a stationary Gaussian random field with
    squared-exponential covariance variance * exp(-|x-y|^2 / (2 corr_len^2)) on the
    unit cube, by spectral synthesis: white noise filtered by the square root of
    the field's power spectrum on a periodic 2N grid (cropped), then scaled to
    the requested variance.  Index order [z, y, x] like varcoef3d."""
    rng = np.random.default_rng(seed)
    M = 2 * N
    h = 1.0 / N
    k = 2.0 * np.pi * np.fft.fftfreq(M, d=h)
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    spec = np.exp(-0.5 * corr_len ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    noise = rng.standard_normal((M, M, M))
    g = np.fft.ifftn(np.fft.fftn(noise) * np.sqrt(spec)).real[:N, :N, :N]
    g = (g - g.mean()) / g.std() * np.sqrt(variance)
    return np.exp(g)


def grf3d(N: int, seed: int) -> sp.csc_matrix:
    """Finite-volume diffusion operator with kappa = exp(GRF) (grf_conductivity)."""
    return _fv_operator(grf_conductivity(N, seed))


class FVPattern:
    """The fixed sparsity pattern of the N^3 finite-volume operator and the map
    from face transmissibilities to its CSC values, so a family of operators
    (same grid, new conductivities) is assembled without rebuilding the pattern."""

    def __init__(self, N: int):
        self.N = N
        base = _fv_operator(np.ones((N, N, N)))
        self.A = base
        n = N ** 3
        idx = np.arange(n).reshape(N, N, N)
        # locate every matrix entry in CSC order: (row, col) -> position
        A = base.tocsc()
        cols = np.repeat(np.arange(n), np.diff(A.indptr))
        rows = A.indices
        key = rows.astype(np.int64) * n + cols
        order = np.argsort(key)
        sk = key[order]

        def pos(r, c):
            return order[np.searchsorted(sk, r.astype(np.int64) * n + c)]
        self.faces = []
        for ax in range(3):
            a = [slice(None)] * 3
            b = [slice(None)] * 3
            a[ax] = slice(0, N - 1)
            b[ax] = slice(1, N)
            ia, ib = idx[tuple(a)].ravel(), idx[tuple(b)].ravel()
            self.faces.append((tuple(a), tuple(b), ia, ib, pos(ia, ib), pos(ib, ia)))
        self.diag_pos = pos(idx.ravel(), idx.ravel())

    def values(self, kap: np.ndarray) -> np.ndarray:
        """CSC values of the operator for cell conductivities kap[z, y, x]."""
        N = self.N
        x = np.zeros(self.A.nnz)
        diag = np.zeros((N, N, N))
        for ax, (a, b, ia, ib, pab, pba) in enumerate(self.faces):
            ka, kb = kap[a], kap[b]
            t = 2.0 * ka * kb / (ka + kb)
            diag[a] += t
            diag[b] += t
            x[pab] = -t.ravel()
            x[pba] = -t.ravel()
            lo = [slice(None)] * 3
            hi = [slice(None)] * 3
            lo[ax] = 0
            hi[ax] = N - 1
            diag[tuple(lo)] += 2.0 * kap[tuple(lo)]
            diag[tuple(hi)] += 2.0 * kap[tuple(hi)]
        x[self.diag_pos] = diag.ravel()
        return x

    def matrix(self, kap: np.ndarray) -> sp.csc_matrix:
        A = self.A.copy()
        A.data = self.values(kap)
        return A


def _fv_operator(kap: np.ndarray) -> sp.csc_matrix:
    N = kap.shape[0]
    n = N ** 3
    idx = np.arange(n).reshape(N, N, N)
    diag = np.zeros((N, N, N))
    rows, cols, vals = [], [], []
    for ax in range(3):
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[ax] = slice(0, N - 1)
        b[ax] = slice(1, N)
        ka, kb = kap[tuple(a)], kap[tuple(b)]
        t = 2.0 * ka * kb / (ka + kb)
        diag[tuple(a)] += t
        diag[tuple(b)] += t
        ia, ib = idx[tuple(a)].ravel(), idx[tuple(b)].ravel()
        rows += [ia, ib]
        cols += [ib, ia]
        vals += [-t.ravel(), -t.ravel()]
        # Dirichlet boundary faces on both ends of this axis
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = 0
        hi[ax] = N - 1
        diag[tuple(lo)] += 2.0 * kap[tuple(lo)]
        diag[tuple(hi)] += 2.0 * kap[tuple(hi)]
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def laplace_modes(N: int, p: int) -> np.ndarray:
    """The p lowest eigenvectors of the Dirichlet 7-point Laplacian on the N^3
    grid (products of sines, closed form), n x p, unit 2-norm columns, ordered
    by eigenvalue (ties in a fixed order).  Index order x fastest."""
    m = int(np.ceil(p ** (1.0 / 3.0))) + 2
    e1 = 2.0 - 2.0 * np.cos(np.arange(1, m + 1) * np.pi / (N + 1))
    trip = [(e1[a] + e1[b] + e1[c], a, b, c) for a in range(m) for b in range(m) for c in range(m)]
    trip.sort()
    g = np.arange(1, N + 1) * np.pi / (N + 1)
    Y = np.empty((N ** 3, p))
    for t, (_, a, b, c) in enumerate(trip[:p]):
        sx, sy, sz = np.sin((a + 1) * g), np.sin((b + 1) * g), np.sin((c + 1) * g)
        f = (sz[:, None, None] * sy[None, :, None] * sx[None, None, :]).ravel()
        Y[:, t] = f / np.linalg.norm(f)
    return Y


def rgg_component(nc: int, rng: np.random.Generator, degree: float = 8.0) -> sp.csr_matrix:
    """Graph Laplacian of a 3-D random geometric graph on nc points uniform in the
    unit cube, unit weights, + 1e-3 I; the connection radius is calibrated so the
    measured mean degree is within 0.5 of `degree` (starting from the bulk value
    (6 degree / (8 pi nc))^(1/3))."""
    from scipy.spatial import cKDTree
    pts = rng.random((nc, 3))
    tree = cKDTree(pts)
    r = (3.0 * degree / (4.0 * np.pi * nc)) ** (1.0 / 3.0)
    for _ in range(8):
        pairs = tree.query_pairs(r, output_type="ndarray")
        md = 2.0 * len(pairs) / nc
        if abs(md - degree) <= 0.5:
            break
        r *= (degree / max(md, 1e-3)) ** (1.0 / 3.0)
    i, j = pairs[:, 0], pairs[:, 1]
    W = sp.csr_matrix((np.ones(len(i)), (i, j)), shape=(nc, nc))
    W = W + W.T
    deg = np.asarray(W.sum(axis=1)).ravel()
    return (sp.diags(deg + 1e-3) - W).tocsr()


def rgg_blocks(ncomp: int, seed: int = 4, nmin: int = 50, nmax: int = 5000,
               first: int | None = None) -> sp.csc_matrix:
    """Block-diagonal SPD matrix of ncomp random-geometric-graph Laplacians
    (+1e-3 I), sizes uniform in [nmin, nmax] from `seed`.  A component whose
    graph is itself disconnected splits further (isolated vertices become 1x1
    blocks with value 1e-3).  first: keep only the first `first` blocks of
    the ncomp-block family -- the same blocks, bit for bit, as in the full
    matrix, since each block draws from the generator after the ones before it."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=ncomp)
    if first is not None:
        sizes = sizes[:first]
    A = sp.block_diag([rgg_component(int(nc), rng) for nc in sizes], format="csc")
    A.sort_indices()
    return A


def rgg_sample(nblocks: int = 120) -> sp.csc_matrix:
    """The first `nblocks` blocks of the 4,096-block random-geometric-graph
    workload (sizes U[50, 5000], seed 4): a sample of it small enough for a
    per-component comparison with a CPU solver."""
    return rgg_blocks(4096, seed=4, first=nblocks)


def components_of(A: sp.spmatrix) -> tuple[int, np.ndarray]:
    """Connected components over the nonzero entries, labelled in order of
    first appearance by row (the labelling speigs_components returns)."""
    from scipy.sparse.csgraph import connected_components
    A = A.tocsr().copy()
    A.eliminate_zeros()
    nc, lab = connected_components(A, directed=False)
    first = np.full(nc, -1, dtype=np.int64)
    seen = 0
    remap = np.empty(nc, dtype=np.int64)
    for i, l in enumerate(lab):
        if first[l] < 0:
            first[l] = i
            remap[l] = seen
            seen += 1
    return int(nc), remap[lab].astype(np.int64)


def upper(A: sp.spmatrix) -> sp.csc_matrix:
    """Upper triangle (with diagonal) in CSC, the other storage speigs accepts."""
    U = sp.triu(A, format="csc")
    U.sort_indices()
    return U


def block_diag(*blocks) -> sp.csc_matrix:
    A = sp.block_diag(blocks, format="csc")
    A.sort_indices()
    return A
