"""Learned warm start for the 'sm' Lanczos on finite-volume diffusion operators.

A small message-passing network (csrc/kernels/mpnn.cu, reached through the C
ABI of include/speigs_b200.h) reads the operator's graph -- the normalised
face transmissibilities of the N^3 grid -- and per-node features (the log
conductivity and the lowest closed-form Laplace modes) and proposes P vectors
whose span should hold the k wanted eigenvectors.  speigs_ex() turns the
proposal into the Lanczos start vector (speigs_ext_opts.warm); the random
start stays the fallback, and the true-residual test of the Lanczos decides
convergence either way, so the proposal changes the cost, never the answer.

The network is trained on eigenvectors this solver computes for a family of
operators (GRF conductivities, workloads.grf_conductivity): see
train_warmstart.py beside this file.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int64, c_uint64, c_void_p

import numpy as np

from . import speigs as _s
from . import workloads as _w

HERE = os.path.dirname(os.path.abspath(__file__))
CHECKPOINT = os.path.join(HERE, "data", "warmstart_grf48.npz")
NMODES = 7          # Laplace modes among the node features
HIDDEN = 64


def _bind(lib):
    sig = {
        "speigs_b200_mpnn_create": (c_int, [c_int, c_int, c_int, c_int, c_uint64,
                                            POINTER(c_void_p)]),
        "speigs_b200_mpnn_destroy": (None, [c_void_p]),
        "speigs_b200_mpnn_tensor_cores": (c_int, [c_void_p, c_int]),
        "speigs_b200_mpnn_grid_graph": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                                c_void_p, c_void_p]),
        "speigs_b200_mpnn_params": (c_int, [c_void_p, c_void_p, POINTER(c_int64), c_int]),
        "speigs_b200_mpnn_grads": (c_int, [c_void_p, c_void_p]),
        "speigs_b200_mpnn_forward": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p]),
        "speigs_b200_mpnn_train_step": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                                c_void_p, c_void_p, c_int, c_float,
                                                POINTER(c_double), c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def grid_graph(N: int, kap: np.ndarray):
    """Normalised adjacency of the N^3 finite-volume operator: w_ij = t_ij /
    sqrt(s_i s_j), t the face transmissibilities, s_i = sum_j t_ij.  Returns
    (rowptr int32, col int32, w float32), rows in the operator's order.

    Built straight in CSR order: node i = (z, y, x) has the neighbours
    i - N^2, i - N, i - 1, i + 1, i + N, i + N^2 (ascending), each present when
    it lies in the grid."""
    n = N ** 3
    kap = np.asarray(kap, dtype=np.float64).reshape(N, N, N)
    T = np.zeros((N, N, N, 6))                  # face transmissibility per neighbour slot
    for ax in range(3):
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[ax] = slice(0, N - 1)
        b[ax] = slice(1, N)
        ka, kb = kap[tuple(a)], kap[tuple(b)]
        t = 2.0 * ka * kb / (ka + kb)
        # axis 0 has stride N^2, axis 2 stride 1: slot ax is the lower
        # neighbour along ax (seen from the upper cell), slot 5 - ax the upper
        # one (seen from the lower cell)
        T[tuple(b) + (ax,)] = t
        T[tuple(a) + (5 - ax,)] = t
    T = T.reshape(n, 6)
    present = T > 0.0
    step = np.array([-N * N, -N, -1, 1, N, N * N], dtype=np.int64)
    cols = np.arange(n, dtype=np.int64)[:, None] + step[None, :]
    s = T.sum(axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):    # absent slots are dropped below
        W = T / np.sqrt(s[:, None] * s[np.where(present, cols, 0)])
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(present.sum(axis=1), out=rowptr[1:])
    return rowptr, cols[present].astype(np.int32), W[present].astype(np.float32)


_MODES: dict = {}


def features(N: int, kap: np.ndarray) -> np.ndarray:
    """n x (1 + NMODES) float32: standardised log conductivity and the lowest
    Laplace modes scaled to unit RMS."""
    if N not in _MODES:
        _MODES[N] = (_w.laplace_modes(N, NMODES) * np.sqrt(N ** 3)).astype(np.float32)
    g = np.log(kap).ravel()
    g = (g - g.mean()) / (g.std() + 1e-12)
    return np.concatenate([g[:, None].astype(np.float32), _MODES[N]], axis=1)


class WarmStartNet:
    """The device network (C ABI) with numpy-side save/load."""

    def __init__(self, nout: int = 24, layers: int = 4, nfeat: int = 1 + NMODES, seed: int = 7,
                 lib=None):
        self.lib = _bind(lib or _s.load())
        self.nout, self.layers, self.nfeat = nout, layers, nfeat
        h = c_void_p()
        rc = self.lib.speigs_b200_mpnn_create(nfeat, HIDDEN, layers, nout, seed, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"mpnn_create: {_s.errmsg(rc, self.lib)} ({_s.last_error(self.lib)})")
        self.h = h
        cnt = c_int64()
        self.lib.speigs_b200_mpnn_params(self.h, None, ctypes.byref(cnt), 0)
        self.nparam = cnt.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.nparam, dtype=np.float32)
        cnt = c_int64(self.nparam)
        self.lib.speigs_b200_mpnn_params(self.h, p.ctypes.data, ctypes.byref(cnt), 0)
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparam
        cnt = c_int64(self.nparam)
        rc = self.lib.speigs_b200_mpnn_params(self.h, p.ctypes.data, ctypes.byref(cnt), 1)
        if rc != 0:
            raise RuntimeError("mpnn_params")

    def grads(self) -> np.ndarray:
        g = np.zeros(self.nparam, dtype=np.float32)
        self.lib.speigs_b200_mpnn_grads(self.h, g.ctypes.data)
        return g

    def tensor_cores(self, on: int = -1) -> int:
        """Select the dense-layer kernels of the forward pass (1: tcgen05
        where the shapes fit, 0: FP32 FMA; -1: query); returns the previous
        setting."""
        return int(self.lib.speigs_b200_mpnn_tensor_cores(self.h, on))

    def grid_graph_device(self, N, kap, rowptr, col, w, stream=0):
        """grid_graph on the device: kap (N^3 float64), rowptr (N^3 + 1 int32),
        col (int32) and w (float32) with room for 6 N^2 (N - 1) entries, all
        device pointers.  The CSR is grid_graph's to the bit."""
        return self.lib.speigs_b200_mpnn_grid_graph(self.h, N, kap, rowptr, col, w, stream)

    def forward_device(self, n, rowptr, col, w, X, Y, stream=0):
        """All arguments are device pointers (ints)."""
        return self.lib.speigs_b200_mpnn_forward(self.h, n, rowptr, col, w, X, Y, stream)

    def train_step_device(self, n, rowptr, col, w, X, U, k, lr, stream=0):
        loss = c_double()
        rc = self.lib.speigs_b200_mpnn_train_step(self.h, n, rowptr, col, w, X, U, k, lr,
                                                  ctypes.byref(loss), stream)
        if rc != 0:
            raise RuntimeError(f"mpnn_train_step rc={rc}: {_s.last_error(self.lib)}")
        return loss.value

    def save(self, path: str, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.get_params(), nout=self.nout, layers=self.layers,
                 nfeat=self.nfeat, **meta)

    @classmethod
    def load(cls, path: str = CHECKPOINT, lib=None):
        z = np.load(path)
        net = cls(int(z["nout"]), int(z["layers"]), int(z["nfeat"]), lib=lib)
        net.set_params(z["params"])
        return net

    def close(self):
        if getattr(self, "h", None):
            self.lib.speigs_b200_mpnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def propose(net: WarmStartNet, N: int, kap: np.ndarray, on_device: bool = False):
    """The network's proposal for one operator: n x nout float64 (host), or
    with on_device a CUDA tensor of shape (nout, n) -- column-major n x nout,
    usable directly as speigs_ext_opts.warm."""
    import torch
    X = features(N, kap)
    dev = torch.device("cuda")
    n = N ** 3
    # the graph is built on the device from the conductivities
    t_kap = torch.from_numpy(np.ascontiguousarray(kap, dtype=np.float64).ravel()).to(dev)
    t_rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    nnz = 6 * N * N * max(N - 1, 0)
    t_ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    t_w = torch.empty(max(nnz, 1), dtype=torch.float32, device=dev)
    t_X = torch.from_numpy(X).to(dev)
    t_Y = torch.empty((n, net.nout), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = net.grid_graph_device(N, t_kap.data_ptr(), t_rp.data_ptr(), t_ci.data_ptr(),
                               t_w.data_ptr(), 0)
    if rc != 0:
        raise RuntimeError(f"mpnn_grid_graph rc={rc}")
    rc = net.forward_device(n, t_rp.data_ptr(), t_ci.data_ptr(), t_w.data_ptr(), t_X.data_ptr(),
                            t_Y.data_ptr(), 0)
    if rc != 0:
        raise RuntimeError(f"mpnn_forward rc={rc}")
    if on_device:
        Y = t_Y.t().double().contiguous()
        # the solver reads it on its own stream
        torch.cuda.synchronize()
        return Y
    torch.cuda.synchronize()
    return t_Y.double().cpu().numpy()
