"""CPU tests of the C ABI library: it loads without a GPU and exports every
function that include/shtcuda.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "shtcuda.h")).read()
    return re.findall(r"SHTC_API\s+(?:const\s+)?\w+\*?\s+\**(\w+)\s*\(", txt)


@pytest.fixture(scope="module")
def lib():
    from shtools_b200 import build, _lib
    build.build()
    return _lib.load()


def test_header_declares_the_reference_dropins():
    names = declared_functions()
    for ref in ("MakeGridDH", "SHExpandDH", "MakeGridGLQ", "SHExpandGLQ",
                "SHGLQ", "PreGLQ", "DHaj", "MakeGridDHC", "SHExpandDHC",
                "MakeGridGLQC", "SHExpandGLQC"):
        assert ref in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_python_binding_covers_exports(lib):
    from shtools_b200 import _lib
    assert set(_lib.EXPORTS) <= set(declared_functions())


def test_status_strings_without_gpu(lib):
    from shtools_b200 import _lib
    assert "dimensions" in _lib.status_string(1)
    assert "bounds" in _lib.status_string(2)
    assert "allocating" in _lib.status_string(3)
    assert lib.shtc_version() >= 100


def test_null_plan_rejected(lib):
    # handle checks happen before any CUDA call
    assert lib.shtc_plan_destroy(None) == 7
    assert lib.shtc_workspace_bytes(None, 1) == 0


def test_probe_library_builds():
    path = os.path.join(ROOT, "shtools_b200", "lib", "libshtc_probe.so")
    assert os.path.exists(path)
    probe = ctypes.CDLL(path)
    assert hasattr(probe, "shtc_probe_dfma")
