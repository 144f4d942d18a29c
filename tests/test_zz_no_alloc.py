"""GPU test of the allocation-free BSE entry point (collected last on purpose).

``dga_bse_solve_sum_noalloc_c128`` exists for callers that cannot call cudaMalloc -- a host that binds only the
C ABI and has no device allocator of its own, or a steady-state loop that must not pay cudaMalloc's device-wide
synchronisation.  It keeps its working matrices in a fixed 64 MiB array inside the library instead of a caller
buffer.  This test calls it through the C ABI twice in a row and compares each result with the regular entry
point ``dga_bse_solve_sum_c128`` (caller scratch) at the FP64 tolerance of the other GPU tests (1e-10 relative),
and checks that a compound size too large for the fixed array is refused with a clear error.
"""

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.fixture(scope="module")
def prepared():
    from dgamore_b200.pipeline import LadderPass

    inp, _ = load_golden("t3")
    lp = LadderPass(inp, keep_intermediates=False)
    lp.bubble()
    lp.chi0_prep()
    lp.bse()  # the regular entry point with a caller-provided scratch buffer
    torch.cuda.synchronize()
    return lp


def _noalloc_call(lp, out, status):
    from dgamore_b200 import _lib

    sh = lp.sh
    return _lib.lib().dga_bse_solve_sum_noalloc_c128(
        sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, lp.inv_beta2, _p(lp.gamma_cm), _p(lp.chi0_inv), _p(lp.uv),
        _p(lp.work), lp.n_items, _p(out), _p(status), _stream(),
    )


def test_noalloc_matches_regular_entry_point_twice(prepared):
    lp = prepared
    expect = lp.X.cpu().numpy()
    for _ in range(2):
        out = torch.full_like(lp.X, float("nan"))
        status = torch.full((lp.n_items,), -1, dtype=torch.int32, device="cuda")
        rc = _noalloc_call(lp, out, status)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(status.abs().sum().item()) == 0
        assert rel_err(out.cpu().numpy(), expect) < TOL


def test_noalloc_rejects_oversize_problem():
    from dgamore_b200 import _lib

    lib = _lib.lib()
    dummy = torch.zeros(4, dtype=torch.complex128, device="cuda")
    work = torch.zeros((1, 3), dtype=torch.int32, device="cuda")
    # N = n_orb^2 * 2 niv = 4 * 2 * 256 = 2048: one 2048x2048 complex matrix needs 64 MiB + the solution
    rc = lib.dga_bse_solve_sum_noalloc_c128(2, 256, 1, 1, 1, 1.0, 1.0, _p(dummy), _p(dummy), _p(dummy), _p(work), 1,
                                            _p(dummy), None, _stream())
    assert rc == 2
    assert b"fixed" in lib.dga_last_error_string()
