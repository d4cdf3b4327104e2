"""The reference's MATLAB gateway links against the B200 library.

oracle/_ref/speigs_mex_b200.so and speigs_mex_b200_sep.so are the
reference's src/speigs_mex.c, unmodified, compiled against declaration-only
stubs of MATLAB's C API (oracle/mexstub/; interleaved- and separate-complex
variants) and linked against sparse-eigs-mex_b200/lib/libspeigs.so
(oracle/Makefile).  MATLAB is not available, so this is a link check: the
gateway defines mexFunction, needs libspeigs.so, and every speigs symbol it
leaves undefined is exported by libspeigs.so; the only other undefined
symbols are MATLAB's own (mx*, mex*) and the C library's.
"""
import os
import subprocess

import pytest

from conftest import ORACLE_DIR


def _syms(path, flag):
    out = subprocess.run(["nm", "-D", flag, path], capture_output=True, text=True, check=True)
    return {ln.split()[-1].split("@")[0] for ln in out.stdout.splitlines() if ln.strip()}


@pytest.mark.parametrize("name", ["speigs_mex_b200.so", "speigs_mex_b200_sep.so"])
def test_gateway_links_against_b200_library(pkg, name):
    path = os.path.join(ORACLE_DIR, "_ref", name)
    if not os.path.exists(path):
        pytest.skip("gateway link check not built (needs the reference tree at build)")
    needed = subprocess.run(["readelf", "-d", path], capture_output=True, text=True).stdout
    assert "[libspeigs.so]" in needed
    assert "mexFunction" in _syms(path, "--defined-only")
    undef = _syms(path, "--undefined-only")
    exported = _syms(pkg.LIB_PATH, "--defined-only")
    ours = {s for s in undef if s.startswith("speigs")}
    assert ours >= {"speigs", "speigs_z", "speigs_default_opts", "speigs_errmsg"}
    assert ours <= exported, ours - exported
    other = {s for s in undef - ours
             if not (s.startswith("mx") or s.startswith("mex") or s.startswith("_"))}
    libc = {"memcpy", "memset", "strcmp", "free", "malloc", "calloc", "strlen", "snprintf",
            "__stack_chk_fail", "sprintf", "memmove", "strncpy", "__memcpy_chk", "__sprintf_chk",
            "__snprintf_chk", "__strcpy_chk", "strcpy"}
    assert other <= libc, other - libc
