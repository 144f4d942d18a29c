"""CPU checks of the C ABI: the shared library builds, loads and exports every symbol of include/dga_b200.h."""

import ctypes
import os
import re

import pytest

from conftest import REPO
from dgamore_b200 import _lib, build


def header_functions() -> list[str]:
    text = open(os.path.join(REPO, "include", "dga_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(dga_\w+)\s*\(", text, flags=re.M)))


def test_library_builds_for_sm100a():
    path = build.build()
    assert os.path.exists(path)
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH_FLAGS)


def test_library_exports_every_header_symbol():
    build.build()
    handle = ctypes.CDLL(build.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(handle, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header():
    assert set(header_functions()) == set(_lib.SIGNATURES)


def test_version_and_error_string_without_gpu():
    lib = _lib.lib()
    assert lib.dga_version() == 100
    assert isinstance(lib.dga_last_error_string(), bytes)


def test_argument_errors_are_reported_without_launching():
    lib = _lib.lib()
    # null pointers are rejected before any CUDA call
    rc = lib.dga_strided_copy_c128(None, None, 0, None, None, None, 1.0, None)
    assert rc == 1
    assert b"invalid" in lib.dga_last_error_string()
    with pytest.raises(_lib.DgaError):
        _lib.call("dga_strided_copy_c128", None, None, 0, None, None, None, 1.0, None)
