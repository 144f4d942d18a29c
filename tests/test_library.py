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


def test_batch_descriptor_matches_the_c_struct():
    # dga_bse_problem: four pointers, four ints, two doubles, no padding on LP64
    assert ctypes.sizeof(_lib.BseProblem) == 64
    assert _lib.BseProblem.beta.offset == 48 and _lib.BseProblem.n_q.offset == 44


def test_batch_rejects_unsupported_mixes_without_launching():
    lib = _lib.lib()
    # orbital counts may differ where the kernels choose the right-hand-side count per item (the 128-thread
    # kernels, and the mixed form's block kernel for 1 to 3 orbitals); the 4-orbital block kernel is compiled
    # alone, so a mixed-precision batch of 4- and 2-orbital problems is refused
    arr = (_lib.BseProblem * 2)(
        _lib.BseProblem(n_orb=4, niv=10, niw_half=3, n_q=2, beta=1.0),
        _lib.BseProblem(n_orb=2, niv=40, niw_half=3, n_q=2, beta=1.0),
    )
    assert lib.dga_bse_batch_scratch_bytes(arr, 2, 10, 1) == 0
    rc = lib.dga_bse_solve_sum_batch_c128(arr, None, 2, None, 10, 1, 0, 0.0, None, None, None, 0, None)
    assert rc == 1 and b"n_orb" in lib.dga_last_error_string()
    five = (_lib.BseProblem * 1)(_lib.BseProblem(n_orb=5, niv=4, niw_half=3, n_q=2, beta=1.0))
    assert lib.dga_bse_batch_scratch_bytes(five, 1, 10, 0) == 0
    one = (_lib.BseProblem * 1)(_lib.BseProblem(n_orb=1, niv=4, niw_half=3, n_q=2, beta=1.0))
    # null input pointers are caught before any CUDA call; an unknown mode too
    rc = lib.dga_bse_solve_sum_batch_c128(one, 1, 1, 1, 10, 0, 0, 0.0, 1, None, 1, 1 << 30, None)
    assert rc == 1 and b"null pointer" in lib.dga_last_error_string()
    assert lib.dga_bse_solve_sum_batch_c128(one, 1, 1, 1, 10, 3, 0, 0.0, 1, None, 1, 1 << 30, None) == 1


def test_tuning_struct_and_rejected_choices_without_gpu():
    assert ctypes.sizeof(_lib.BseTuning) == 16  # int kernel, int ctas_per_sm, long long wait_limit
    lib = _lib.lib()
    bad = _lib.BseTuning(kernel=5, ctas_per_sm=0)
    assert lib.dga_bse_tuned_scratch_bytes(720, 9, 100, 1, ctypes.byref(bad)) == 0
    panel_fp64 = _lib.BseTuning(kernel=1, ctas_per_sm=0)  # the panel kernel is mixed-precision only
    assert lib.dga_bse_tuned_scratch_bytes(720, 9, 100, 0, ctypes.byref(panel_fp64)) == 0
    rc = lib.dga_bse_solve_sum_tuned_c128(3, 40, 41, 153, 2, 20.0, 1 / 400, None, None, None, None, 10, 1, 4, 1e-10,
                                          None, None, None, ctypes.byref(bad), None, 0, None)
    assert rc == 1
