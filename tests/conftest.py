"""Shared fixtures: the package (imported by path; its directory name is not a
Python identifier), the B200 library, and the compiled reference oracle."""
import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "sparse-eigs-mex_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libspeigs_ref.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def import_package():
    if "speigs_b200" in sys.modules:
        return sys.modules["speigs_b200"]
    spec = importlib.util.spec_from_file_location(
        "speigs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["speigs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def import_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import speigs_oracle  # noqa: E402
    return speigs_oracle


@pytest.fixture(scope="session")
def pkg():
    return import_package()


@pytest.fixture(scope="session")
def oracle():
    return import_oracle()


@pytest.fixture(scope="session")
def lib(pkg):
    if not os.path.exists(pkg.LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", PKG_DIR])
    return pkg.speigs.load()


@pytest.fixture(scope="session")
def ref_lib(pkg):
    """The reference's own solver compiled on the CPU (oracle/_ref)."""
    if not os.path.exists(REF_LIB):
        if not os.path.isdir("/root/reference"):
            pytest.skip("oracle/_ref not built and the reference tree is absent")
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    return pkg.speigs.load(REF_LIB)
