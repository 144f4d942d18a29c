"""ctypes binding of libdga_b200.so (the C ABI declared in include/dga_b200.h).

The product path has no CPU fallback: ``lib()`` raises if the shared library is missing or does not load,
and every wrapper raises ``DgaError`` on a non-zero return code with the library's last error message.
"""

from __future__ import annotations

import ctypes
import os

from . import build as _build

_c = ctypes
VP, I, D, LL, SZ = _c.c_void_p, _c.c_int, _c.c_double, _c.c_longlong, _c.c_size_t
PLL = _c.POINTER(_c.c_longlong)
PI = _c.c_void_p  # device int pointers are passed as raw addresses
PD = _c.c_void_p

# name -> (restype, argtypes); must match include/dga_b200.h
SIGNATURES = {
    "dga_version": (I, []),
    "dga_device_sm_count": (I, []),
    "dga_bse_block_ctas_per_sm": (I, [I]),
    "dga_bse_default_kernel": (I, [I, I, I]),
    "dga_bse_preload": (I, []),
    "dga_last_error_string": (_c.c_char_p, []),
    "dga_strided_copy_c128": (I, [VP, VP, I, PLL, PLL, PLL, D, VP]),
    "dga_dft_planes_c128": (I, [VP, LL, LL, LL, VP, LL, LL, LL, I, I, I, I, I, VP, D, VP]),
    "dga_bubble_c128": (I, [VP, I, I, I, I, I, I, PI, I, VP, D, VP, PLL, VP]),
    "dga_chi0_prep_c128": (I, [VP, I, I, I, I, I, D, VP, VP, VP, PI, VP]),
    "dga_bse_scratch_bytes": (SZ, [I, I, I]),
    "dga_bse_solve_sum_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, VP, PI, VP, SZ, VP]),
    "dga_invert_sum_dense_c128": (I, [I, I, I, I, D, VP, PI, I, VP, PI, VP, SZ, VP]),
    "dga_bse_solve_sum_noalloc_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, VP, PI, VP]),
    "dga_bse_mixed_scratch_bytes": (SZ, [I, I, I]),
    "dga_bse_solve_sum_mixed_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, I, D, VP, PI, PI, VP, SZ, VP]),
    "dga_bse_resolve_fp64_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, VP, PI, I, VP, SZ, VP]),
    "dga_chi_phys_c128": (I, [VP, VP, VP, VP, I, I, I, I, I, D, VP, PI, VP]),
    "dga_lambda_c128": (I, [VP, I, I, I, PI, VP, D, D, D, D, I, PD, PI, PI, VP, VP]),
    "dga_kernel_assembly_c128": (I, [VP, VP, VP, VP, VP, I, I, I, I, D, VP, VP, VP]),
    "dga_dc_scratch_bytes": (SZ, [I, I, I, I]),
    "dga_dc_kernel_c128": (I, [VP, VP, VP, I, I, I, I, I, VP, VP, SZ, VP]),
    "dga_sigma_scratch_bytes": (SZ, [I, I, I, I]),
    "dga_sigma_c128": (I, [VP, VP, I, I, I, I, I, I, I, PI, VP, D, I, VP, VP, SZ, VP]),
    "dga_sigma_rspace_c128": (I, [VP, VP, I, I, I, I, I, I, I, PI, VP, D, I, VP, VP, SZ, VP]),
    "dga_dft_planes_gather_c128": (I, [VP, LL, LL, LL, VP, LL, LL, LL, I, I, I, I, I, VP, D, PI, VP]),
    "dga_eli_vertex_scratch_bytes": (SZ, [I, I, I, I]),
    "dga_eli_full_vertex_c128": (I, [I, I, I, I, I, I, D, D, VP, VP, VP, VP, VP, PI, I, VP, PI, VP, SZ, VP]),
    "dga_eli_pairing_vertex_c128": (I, [VP, I, I, I, I, VP, VP]),
    "dga_eli_chi0pp_c128": (I, [VP, I, I, I, I, VP, VP]),
    "dga_eli_matvec_scratch_bytes": (SZ, [I, I, I]),
    "dga_eli_matvec_c128": (I, [VP, VP, VP, I, I, I, I, I, VP, VP, D, D, VP, VP, SZ, VP]),
    "dga_eli_matvec_c64mat_c128": (I, [VP, VP, VP, I, I, I, I, I, VP, VP, D, D, VP, VP, SZ, VP]),
    "dga_narrow_c128_to_c64": (I, [VP, VP, LL, VP]),
    "dga_bse_batch_scratch_bytes": (SZ, [VP, I, I, I]),
    "dga_bse_solve_sum_batch_c128": (I, [VP, VP, I, PI, I, I, I, D, PI, PI, VP, SZ, VP]),
    "dga_bse_tuned_scratch_bytes": (SZ, [I, I, I, I, VP]),
    "dga_hartree_fock_c128": (I, [VP, VP, VP, VP, I, I, I, I, VP, VP, VP, I, VP]),
    "dga_g_full_c128": (I, [VP, VP, I, I, I, D, D, VP, VP]),
    "dga_fill_sums_c128": (I, [VP, VP, PD, I, I, I, D, D, PD, PD, VP]),
    "dga_sigma_kmean_c128": (I, [VP, I, I, I, I, I, VP, VP]),
    "dga_bse_solve_sum_tuned_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, I, I, D, VP, PI, PI, VP, VP, SZ, VP]),
    "dga_bse_eli_scratch_bytes": (SZ, [I, I, I]),
    "dga_bse_solve_sum_eli_c128": (I, [I, I, I, I, I, D, D, VP, VP, VP, PI, I, I, I, VP, VP, PI, VP, SZ, VP]),
    "dga_eli_ladder_term_c128": (I, [VP, VP, VP, I, I, I, I, I, I, VP, VP]),
    "dga_sigma_wedge_scratch_bytes": (SZ, [I, I, I, I, I, I]),
    "dga_sigma_wedge_c128": (I, [VP, VP, I, I, I, I, I, I, I, PI, VP, VP, D, I, I, VP, VP, SZ, VP]),
    "dga_fbz_rotate_c128": (I, [VP, PI, I, VP, PD, VP, I, PLL, LL, I, LL, I, LL, VP, VP]),
    "dga_lu_batched_c128": (I, [VP, I, I, LL, PI, PI, VP]),
    "dga_lu_solve_batched_c128": (I, [VP, PI, I, I, LL, VP, LL, LL, LL, I, VP, LL, PI, VP]),
    "dga_local_bubble_c128": (I, [VP, I, I, I, I, D, VP, VP]),
    "dga_local_chi_c128": (I, [VP, I, I, I, I, I, VP, I, D, I, VP, VP]),
    "dga_local_ucorr_c128": (I, [VP, VP, VP, I, I, VP, PI, VP]),
    "dga_local_gamma_c128": (I, [VP, LL, VP, VP, I, I, I, D, VP, VP]),
    "dga_local_fvertex_operands_c128": (I, [VP, VP, VP, I, I, I, I, D, VP, VP, VP]),
    "dga_local_sigma_c128": (I, [VP, VP, VP, VP, VP, VP, I, I, I, I, D, VP, VP, VP]),
}


class BseTuning(_c.Structure):
    """``dga_bse_tuning`` of include/dga_b200.h (kernel choice and CTAs per SM of the BSE solvers)."""

    _fields_ = [("kernel", I), ("ctas_per_sm", I), ("wait_limit", LL)]


class BseProblem(_c.Structure):
    """``dga_bse_problem`` of include/dga_b200.h (one request of a heterogeneous BSE batch)."""

    _fields_ = [
        ("gamma_cm", VP),
        ("chi0_inv", VP),
        ("uv", VP),
        ("out", VP),
        ("n_orb", I),
        ("niv", I),
        ("niw_half", I),
        ("n_q", I),
        ("beta", D),
        ("inv_beta2", D),
    ]


class DgaError(RuntimeError):
    """A libdga_b200 entry point returned an error code."""


_LIB = None


def lib_path() -> str:
    return _build.LIB_PATH


def lib() -> ctypes.CDLL:
    """Loads libdga_b200.so (built in-tree by ``python -m dgamore_b200.build``)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise DgaError(f"{path} is missing: build it with `python -m dgamore_b200.build` (no CPU fallback)")
        handle = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def check(rc: int, name: str) -> None:
    if rc != 0:
        msg = lib().dga_last_error_string()
        raise DgaError(f"{name} returned {rc}: {msg.decode() if msg else ''}")


def call(name: str, *args) -> None:
    """Calls an int-returning entry point and raises on failure."""
    check(getattr(lib(), name)(*args), name)


def ll_array(values) -> ctypes.Array:
    arr = (ctypes.c_longlong * len(values))(*[int(v) for v in values])
    return arr
