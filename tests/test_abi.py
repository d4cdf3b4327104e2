"""The C-ABI library loads on a CPU-only machine and exports exactly the
entry points include/*.h declares; defaults and messages match the reference
(include/speigs.h, src/speigs_core.c:635-639, :770-781).  No compute calls."""
import ctypes
import os
import re

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("speigs.h", "speigs_b200.h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(speigs\w*)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "speigs" in names and "speigs_z" in names and "speigs_plan_create" in names
    for name in names:
        assert hasattr(lib, name), f"libspeigs.so does not export {name}"


def test_no_private_symbols_leak(pkg):
    out = os.popen(f"nm -D --defined-only {pkg.LIB_PATH}").read()
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = set(declared_functions())
    extra = {s for s in exported if not s.startswith("_")} - declared
    assert not extra, f"undeclared exports: {sorted(extra)}"


def test_struct_layouts(pkg):
    s = pkg.speigs
    assert ctypes.sizeof(s.Opts) == 64
    assert ctypes.sizeof(s.Info) == 120
    assert s.Info.path.offset == 48 and s.Info.ncomp.offset == 56


def test_default_opts(lib, pkg):
    o = pkg.speigs.default_opts(lib)
    assert (o.tol, o.maxit, o.ncv, o.dense_max, o.detect, o.seed, o.check_sym, o.band_max,
            o.ordering, o.shift0) == (0.0, 0, 0, -1, 1, 0, 1, 0, 0, 0.0)


def test_errmsg(lib, pkg):
    e = pkg.speigs.errmsg
    assert e(0, lib) == "ok"
    assert e(-1, lib) == "invalid argument"
    assert e(-3, lib) == "factorization failed"
    assert e(-6, lib).startswith("matrix is not symmetric")
    assert e(-99, lib) == "internal error"


def test_argument_errors_need_no_gpu(lib, pkg):
    """Argument checks run before any device work (reference :791-792)."""
    A = pkg.workloads.lap3d(4)
    rc, *_ = pkg.speigs.speigs(A, 0, lib=lib)
    assert rc == pkg.speigs.ERR_ARG
    rc, *_ = pkg.speigs.speigs(A, A.shape[0] + 1, lib=lib)
    assert rc == pkg.speigs.ERR_ARG


def test_nonsymmetric_rejected_before_gpu(lib, pkg):
    import scipy.sparse as sp
    import numpy as np
    n = 50
    A = sp.diags([-4 * np.ones(n - 1), 5 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csc")
    rc, *_ = pkg.speigs.speigs(A, 3, lib=lib)
    assert rc == pkg.speigs.ERR_NOTSYM


def test_extension_argument_errors_need_no_gpu(lib, pkg):
    """The extension entry points reject bad arguments before any device
    work: component labels outside [0, ncomp) or a label with no rows, k <= 0,
    and a non-symmetric matrix for the batched call."""
    import numpy as np
    import scipy.sparse as sp
    s = pkg.speigs
    A = sp.block_diag([pkg.workloads.lap3d(3), pkg.workloads.lap3d(3)], format="csc")
    n = A.shape[0]
    comp = np.repeat([0, 1], n // 2)
    rc, *_ = s.speigs_batched(A, 0, comp=comp, lib=lib)
    assert rc == s.ERR_ARG
    # labels 1 and 2 only: ncomp is 3 and label 0 has no rows
    rc, *_ = s.speigs_batched(A, 2, comp=np.where(comp == 0, 2, comp), lib=lib)
    assert rc == s.ERR_ARG
    B = A.tolil()
    B[0, 1] = 7.0
    rc, *_ = s.speigs_batched(B.tocsc(), 2, comp=comp, lib=lib)
    assert rc == s.ERR_NOTSYM
    rc, *_ = s.speigs_ex(A, 0, lib=lib)
    assert rc == s.ERR_ARG
