"""ctypes binding of the speigs C ABI (include/speigs.h, include/speigs_b200.h).

The same binding drives any library that exports the reference interface,
so a test can call the B200 library and a CPU build of the reference through
identical code.  Loading the B200 library fails loudly when it has not been
built: there is no Python or CPU stand-in behind these calls.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libspeigs.so")

SM, LM = 0, 1
PATH_DIAG, PATH_DENSE, PATH_SHIFTINV, PATH_DIRECT, PATH_BLOCKS, PATH_LU, PATH_BANDED = range(7)
OK, ERR_ARG, ERR_MEM, ERR_FACTOR, ERR_LAPACK, ERR_INTERNAL, ERR_NOTSYM = 0, -1, -2, -3, -4, -5, -6


class Opts(ctypes.Structure):
    """speigs_opts (reference include/speigs.h:40-55)."""
    _fields_ = [("tol", c_double), ("maxit", c_int64), ("ncv", c_int64), ("dense_max", c_int),
                ("detect", c_int), ("seed", c_uint64), ("check_sym", c_int), ("band_max", c_int),
                ("ordering", c_int), ("shift0", c_double)]


class Info(ctypes.Structure):
    """speigs_info (reference include/speigs.h:57-68)."""
    _fields_ = [("flag", c_int), ("nconv", c_int64), ("restarts", c_int64), ("nops", c_int64),
                ("shift", c_double), ("anorm", c_double), ("path", c_int), ("ncomp", c_int64),
                ("t_analyze", c_double), ("t_factor", c_double), ("t_iter", c_double),
                ("t_op", c_double), ("t_ortho", c_double), ("t_resid", c_double),
                ("t_ritz", c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ExtOpts(ctypes.Structure):
    """speigs_ext_opts (include/speigs_b200.h): operator precision, start subspace."""
    _fields_ = [("precision", c_int), ("refine_max", c_int), ("refine_tol", c_double),
                ("warm", c_void_p), ("warm_cols", c_int64), ("block", c_int),
                ("handoff", c_int)]


class ExtInfo(ctypes.Structure):
    """speigs_ext_info (include/speigs_b200.h)."""
    _fields_ = [("precision", c_int), ("refine_steps", c_int64), ("factor_solves", c_int64),
                ("warm_cols", c_int64), ("block", c_int), ("block_solves", c_int64),
                ("t_checks", c_double), ("t_setup", c_double), ("t_release", c_double),
                ("t_block_solve", c_double), ("block_solve_calls", c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


FP64, MIXED = 0, 1

_I64P = POINTER(c_int64)
_DP = POINTER(c_double)

_SIGNATURES = {
    "speigs_default_opts": (None, [POINTER(Opts)]),
    "speigs": (c_int, [c_int64, _I64P, _I64P, _DP, c_int64, c_int, POINTER(Opts), _DP, _DP, _DP,
                       POINTER(Info)]),
    "speigs_z": (c_int, [c_int64, _I64P, _I64P, _DP, _DP, c_int64, c_int, POINTER(Opts), _DP, _DP,
                         _DP, _DP, POINTER(Info)]),
    "speigs_errmsg": (c_char_p, [c_int]),
}
_EXT_SIGNATURES = {
    "speigs_plan_create": (c_int, [c_int64, _I64P, _I64P, _DP, c_int, POINTER(Opts),
                                   POINTER(c_void_p)]),
    "speigs_plan_set_values": (c_int, [c_void_p, _DP]),
    "speigs_plan_solve_device": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                         POINTER(Info)]),
    "speigs_plan_apply_device": (c_int, [c_void_p, c_void_p, c_void_p]),
    "speigs_plan_apply_block_device": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int64,
                                               c_int]),
    "speigs_plan_factor": (c_int, [c_void_p, _DP]),
    "speigs_plan_stream": (c_void_p, [c_void_p]),
    "speigs_plan_costs": (c_int, [c_void_p, _DP, _DP, _DP]),
    "speigs_plan_destroy": (None, [c_void_p]),
    "speigs_b200_rand_vec": (c_int, [c_int64, c_uint64, _DP]),
    "speigs_default_ext_opts": (None, [POINTER(ExtOpts)]),
    "speigs_ex": (c_int, [c_int64, _I64P, _I64P, _DP, c_int64, c_int, POINTER(Opts),
                          POINTER(ExtOpts), _DP, _DP, _DP, POINTER(Info), POINTER(ExtInfo)]),
    "speigs_plan_create_ex": (c_int, [c_int64, _I64P, _I64P, _DP, c_int, POINTER(Opts),
                                      POINTER(ExtOpts), POINTER(c_void_p)]),
    "speigs_plan_ext_info": (c_int, [c_void_p, POINTER(ExtInfo)]),
    "speigs_components": (c_int, [c_int64, _I64P, _I64P, _DP, _I64P, _I64P]),
    "speigs_batched": (c_int, [c_int64, _I64P, _I64P, _DP, c_int64, c_int, POINTER(Opts),
                               POINTER(ExtOpts), _I64P, c_int64, _DP, _DP, _DP, _I64P,
                               POINTER(Info)]),
    "speigs_b200_syev_small": (c_int, [c_int, _DP, _DP, _DP, POINTER(c_int)]),
    "speigs_b200_syev_small_noalloc": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                               c_void_p, c_void_p]),
    "speigs_b200_factor_cache": (c_int, [c_int]),
    "speigs_b200_factor_cache_size": (c_int, []),
    "speigs_b200_last_error": (c_char_p, []),
    "speigs_b200_counters": (None, [POINTER(ctypes.c_longlong)] * 3),
}

_cache: dict[str, ctypes.CDLL] = {}


def load(path: str | None = None) -> ctypes.CDLL:
    """Load a library exporting the speigs ABI (default: the B200 build)."""
    path = os.path.abspath(path or LIB_PATH)
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise RuntimeError(f"speigs library not built: {path} (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    for name, (res, args) in _EXT_SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is not None:
            fn.restype, fn.argtypes = res, args
    _cache[path] = lib
    return lib


def default_opts(lib=None, **kw) -> Opts:
    lib = lib or load()
    o = Opts()
    lib.speigs_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def ext_opts(lib=None, warm=None, **kw) -> ExtOpts:
    """Extension options; warm: optional (n, p) start subspace kept alive by the caller."""
    lib = lib or load()
    e = ExtOpts()
    lib.speigs_default_ext_opts(ctypes.byref(e))
    for k, v in kw.items():
        setattr(e, k, v)
    if warm is not None:
        e.warm = warm.ctypes.data
        e.warm_cols = warm.shape[1]
    return e


def _csc_arrays(A):
    """(n, Ap, Ai, Ax) int64/float64 contiguous from a scipy sparse matrix or a tuple."""
    if isinstance(A, tuple):
        n, Ap, Ai, Ax = A
    else:
        A = A.tocsc()
        A.sort_indices()
        n, Ap, Ai, Ax = A.shape[0], A.indptr, A.indices, A.data
    return (int(n), np.ascontiguousarray(Ap, dtype=np.int64),
            np.ascontiguousarray(Ai, dtype=np.int64), np.ascontiguousarray(Ax, dtype=np.float64))


def _p(a, t=c_double):
    return a.ctypes.data_as(POINTER(t))


def speigs(A, k, which=SM, opts: Opts | None = None, vectors=True, lib=None):
    """Call speigs() through the C ABI.

    Returns (rc, lam[k], V[n, k] or None, resid[k], info dict).
    """
    lib = lib or load()
    n, Ap, Ai, Ax = _csc_arrays(A)
    lam = np.zeros(k)
    res = np.zeros(k)
    V = np.zeros((k, n)) if vectors else None   # column-major n x k == row-major k x n
    info = Info()
    o = opts if opts is not None else default_opts(lib)
    rc = lib.speigs(n, _p(Ap, c_int64), _p(Ai, c_int64), _p(Ax), k, which, ctypes.byref(o),
                    _p(lam), _p(V) if vectors else None, _p(res), ctypes.byref(info))
    return rc, lam, (V.T.copy() if vectors else None), res, info.as_dict()


def speigs_ex(A, k, which=SM, opts: Opts | None = None, ext: ExtOpts | None = None,
              vectors=True, lib=None, warm=None):
    """speigs_ex() through the C ABI: (rc, lam, V, resid, info, ext_info).

    warm: optional (n, p) float64 start subspace (overrides ext.warm)."""
    lib = lib or load()
    n, Ap, Ai, Ax = _csc_arrays(A)
    lam = np.zeros(k)
    res = np.zeros(k)
    V = np.zeros((k, n)) if vectors else None
    info, einfo = Info(), ExtInfo()
    o = opts if opts is not None else default_opts(lib)
    e = ext if ext is not None else ext_opts(lib)
    W = None
    if warm is not None:
        W = np.asfortranarray(warm, dtype=np.float64)
        e.warm = W.ctypes.data
        e.warm_cols = W.shape[1]
    rc = lib.speigs_ex(n, _p(Ap, c_int64), _p(Ai, c_int64), _p(Ax), k, which, ctypes.byref(o),
                       ctypes.byref(e), _p(lam), _p(V) if vectors else None, _p(res),
                       ctypes.byref(info), ctypes.byref(einfo))
    return rc, lam, (V.T.copy() if vectors else None), res, info.as_dict(), einfo.as_dict()


def components(A, lib=None):
    """speigs_components(): (ncomp, labels[n])."""
    lib = lib or load()
    n, Ap, Ai, Ax = _csc_arrays(A)
    comp = np.zeros(n, dtype=np.int64)
    nc = c_int64()
    rc = lib.speigs_components(n, _p(Ap, c_int64), _p(Ai, c_int64), _p(Ax), _p(comp, c_int64),
                               ctypes.byref(nc))
    if rc:
        raise RuntimeError(f"speigs_components: {errmsg(rc, lib)}")
    return nc.value, comp


def speigs_batched(A, k, which=SM, opts: Opts | None = None, ext: ExtOpts | None = None,
                   comp=None, vectors=False, lib=None):
    """speigs_batched(): k eigenpairs per connected component.

    Returns (rc, lam[ncomp, k], V[n, k] or None, resid[ncomp, k], nvals[ncomp], info)."""
    lib = lib or load()
    n, Ap, Ai, Ax = _csc_arrays(A)
    if comp is None:
        ncomp, comp = components((n, Ap, Ai, Ax), lib)
    else:
        comp = np.ascontiguousarray(comp, dtype=np.int64)
        ncomp = int(comp.max()) + 1
    lam = np.zeros((ncomp, k))
    res = np.zeros((ncomp, k))
    nv = np.zeros(ncomp, dtype=np.int64)
    V = np.zeros((k, n)) if vectors else None
    info = Info()
    o = opts if opts is not None else default_opts(lib)
    rc = lib.speigs_batched(n, _p(Ap, c_int64), _p(Ai, c_int64), _p(Ax), k, which,
                            ctypes.byref(o), ctypes.byref(ext) if ext is not None else None,
                            _p(comp, c_int64), ncomp, _p(lam), _p(V) if vectors else None,
                            _p(res), _p(nv, c_int64), ctypes.byref(info))
    return rc, lam, (V.T.copy() if vectors else None), res, nv, info.as_dict()


BATCHED_TIMES = ("t_checks", "t_group", "t_analyze", "t_factor", "t_iter", "t_lockstep",
                 "t_one_by_one", "t_total", "t_engine")
BATCHED_COUNTS = ("lockstep_components", "one_by_one_components", "handed_off", "steps",
                  "cycles", "lockstep_rows", "graph")


def batched_stats(lib=None) -> dict:
    """speigs_b200_batched_stats(): phases of this thread's last speigs_batched."""
    lib = lib or load()
    t = np.zeros(len(BATCHED_TIMES))
    c = np.zeros(len(BATCHED_COUNTS), dtype=np.int64)
    rc = lib.speigs_b200_batched_stats(_p(t), _p(c, c_int64))
    if rc:
        raise RuntimeError(f"batched_stats: {errmsg(rc, lib)}")
    out = {name: float(v) for name, v in zip(BATCHED_TIMES, t)}
    out.update({name: int(v) for name, v in zip(BATCHED_COUNTS, c)})
    return out


def speigs_z(A_re, A_im, k, which=SM, opts: Opts | None = None, lib=None):
    """Complex Hermitian through the C ABI: A_re/A_im share one CSC pattern."""
    lib = lib or load()
    n, Ap, Ai, Axr = _csc_arrays(A_re)
    Axi = np.ascontiguousarray(A_im, dtype=np.float64)
    lam = np.zeros(k)
    res = np.zeros(k)
    Vr = np.zeros((k, n))
    Vi = np.zeros((k, n))
    info = Info()
    o = opts if opts is not None else default_opts(lib)
    rc = lib.speigs_z(n, _p(Ap, c_int64), _p(Ai, c_int64), _p(Axr), _p(Axi), k, which,
                      ctypes.byref(o), _p(lam), _p(Vr), _p(Vi), _p(res), ctypes.byref(info))
    return rc, lam, (Vr.T + 1j * Vi.T), res, info.as_dict()


def errmsg(rc, lib=None) -> str:
    return (lib or load()).speigs_errmsg(rc).decode()


def last_error(lib=None) -> str:
    return (lib or load()).speigs_b200_last_error().decode()


class Plan:
    """speigs_plan: a matrix kept on the GPU across solves (speigs_b200.h)."""

    def __init__(self, A, which=SM, opts: Opts | None = None, lib=None,
                 ext: ExtOpts | None = None):
        self.lib = lib or load()
        self.n, self._Ap, self._Ai, Ax = _csc_arrays(A)
        self.which = which
        h = c_void_p()
        o = opts if opts is not None else default_opts(self.lib)
        self._ext = ext
        rc = self.lib.speigs_plan_create_ex(self.n, _p(self._Ap, c_int64), _p(self._Ai, c_int64),
                                            _p(Ax), which, ctypes.byref(o),
                                            ctypes.byref(ext) if ext is not None else None,
                                            ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"speigs_plan_create: {errmsg(rc, self.lib)} ({last_error(self.lib)})")
        self.h = h

    def set_values(self, Ax):
        Ax = np.ascontiguousarray(Ax, dtype=np.float64)
        return self.lib.speigs_plan_set_values(self.h, _p(Ax))

    def solve_device(self, k, lam_ptr, V_ptr, resid_ptr):
        info = Info()
        rc = self.lib.speigs_plan_solve_device(self.h, k, lam_ptr, V_ptr, resid_ptr,
                                               ctypes.byref(info))
        return rc, info.as_dict()

    def ext_info(self):
        e = ExtInfo()
        self.lib.speigs_plan_ext_info(self.h, ctypes.byref(e))
        return e.as_dict()

    def apply_device(self, x_ptr, y_ptr):
        return self.lib.speigs_plan_apply_device(self.h, x_ptr, y_ptr)

    def apply_block_device(self, x_ptr, ldx, y_ptr, ldy, nr):
        """Y = Op X for nr <= 32 device columns (column-major, leading dims ldx, ldy)."""
        return self.lib.speigs_plan_apply_block_device(self.h, x_ptr, ldx, y_ptr, ldy, nr)

    def factor(self):
        s = c_double()
        rc = self.lib.speigs_plan_factor(self.h, ctypes.byref(s))
        return rc, s.value

    def stream(self) -> int:
        return self.lib.speigs_plan_stream(self.h) or 0

    def costs(self):
        b, f, z = c_double(), c_double(), c_double()
        self.lib.speigs_plan_costs(self.h, ctypes.byref(b), ctypes.byref(f), ctypes.byref(z))
        return {"op_bytes": b.value, "factor_flops": f.value, "nnz_factor": z.value}

    def close(self):
        if getattr(self, "h", None):
            self.lib.speigs_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def counters(lib=None):
    """(kernel launches, H2D bytes, D2H bytes) issued by the library so far."""
    lib = lib or load()
    a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    lib.speigs_b200_counters(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def rand_vec(n, seed, lib=None):
    lib = lib or load()
    v = np.zeros(n)
    rc = lib.speigs_b200_rand_vec(n, seed, _p(v))
    if rc:
        raise RuntimeError(f"rand_vec: {errmsg(rc, lib)} ({last_error(lib)})")
    return v


def syev_small(H, lib=None):
    lib = lib or load()
    H = np.asfortranarray(H, dtype=np.float64)
    m = H.shape[0]
    th = np.zeros(m)
    S = np.zeros((m, m), order="F")
    ordv = np.zeros(m, dtype=np.int32)
    rc = lib.speigs_b200_syev_small(m, H.ctypes.data_as(_DP), _p(th),
                                    S.ctypes.data_as(_DP), ordv.ctypes.data_as(POINTER(c_int)))
    if rc:
        raise RuntimeError(f"syev_small: {errmsg(rc, lib)} ({last_error(lib)})")
    return th, S, ordv
