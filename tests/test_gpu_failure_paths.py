"""Failure paths of the BSE solvers on the GPU, made on the host (no GPU fault is provoked):

* a NaN planted in one entry of Gamma_r: exactly the work items that read it (one channel, one bosonic
  frequency, every q) come back flagged DGA_ITEM_NONFINITE, in the FP64 and the mixed form, and every other
  item is bitwise the clean run's result;
* an exactly singular matrix through the array-level mirror of FourPoint.invert_and_sum_over_last_vn
  raises numpy.linalg.LinAlgError, as the upstream's np.linalg.inv does (dgamore/four_point.py:620-642);
* a bounded wait that runs out: launched with a negative wait limit (the test hook of dga_bse_tuning), each CTA
  of the mixed tensor-core kernel first waits, for that many polls, on a barrier phase that nothing completes;
  the wait runs out, the CTA issues no more bulk copies or tiles, every item comes back DGA_ITEM_WAIT_TIMEOUT,
  and the FP64 re-solve then brings every item to the FP64 result; the context stays usable.

The 3-orbital cases use the full compound size of the benchmark configuration (N = 720) on a 4x4 grid, so the
mixed launch runs the tensor-core panel kernel.
"""

import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu

NONFINITE, WAIT_TIMEOUT = 2, 8


@pytest.fixture(scope="module")
def c3_small():
    from dgamore_b200 import synthetic
    from dgamore_b200.profile_case import reduced_config

    return synthetic.make_inputs(reduced_config("c3", 4, 2))


def _bse(inp, precision):
    from dgamore_b200.pipeline import LadderPass

    lp = LadderPass(inp, keep_intermediates=False, precision=precision)
    lp.pre_bse()
    lp.bse()
    torch.cuda.synchronize()
    return lp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_in_gamma_flags_exactly_its_items(c3_small, precision):
    clean = _bse(c3_small, precision)
    x_clean = clean.X.cpu().numpy()
    assert int(clean.bse_status.abs().sum()) == 0
    work = clean.work.cpu().numpy()
    del clean
    bad = dict(c3_small)
    bad["gamma_magn"] = np.array(c3_small["gamma_magn"], copy=True)
    w_bad = 1
    bad["gamma_magn"][0, 0, 0, 0, w_bad, 3, 5] = np.nan
    lp = _bse(bad, precision)
    status = lp.bse_status.cpu().numpy()
    hit = (work[:, 0] == 1) & (work[:, 2] == w_bad)
    assert np.all(status[hit] & NONFINITE), status[hit]
    assert np.all(status[~hit] == 0), status[~hit]
    x = lp.X.cpu().numpy()
    for ch, q, w in work[~hit]:
        assert np.array_equal(x[ch, q, w], x_clean[ch, q, w]), (ch, q, w)


def test_singular_matrix_raises_linalgerror():
    from dgamore_b200.four_point import invert_and_sum_over_last_vn

    rng = np.random.default_rng(3)
    nq, nb, nw, nv = 2, 2, 2, 4
    shape = (nq, nb, nb, nb, nb, nw, nv, nv)
    mat = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ok = invert_and_sum_over_last_vn(mat, 5.0)
    assert np.all(np.isfinite(ok))
    mat[1, :, :, 0, 1, 0, :, 2] = 0.0  # one compound column of the (q=1, w=0) matrix is zero: rank-deficient
    with pytest.raises(np.linalg.LinAlgError):
        invert_and_sum_over_last_vn(mat, 5.0)


@pytest.mark.parametrize("kernel", [3, 4])
def test_wait_that_runs_out_is_flagged_and_resolved(c3_small, kernel):
    from dgamore_b200 import autotune
    from dgamore_b200._lib import BseTuning, call
    from dgamore_b200.pipeline import LadderPass

    ref = _bse(c3_small, "fp64")
    x64 = ref.X.cpu().numpy()
    del ref
    lp = LadderPass(c3_small, keep_intermediates=False, precision="mixed")
    lp.pre_bse()
    sh = lp.sh
    t = BseTuning(kernel=kernel, ctas_per_sm=0, wait_limit=-1000)
    nbytes = int(autotune.lib().dga_bse_tuned_scratch_bytes(sh.N, sh.n2, lp.n_items, 1, ctypes.byref(t)))
    assert nbytes > 0
    scratch = torch.empty(nbytes // 16 + 1, dtype=torch.complex128, device="cuda")
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lp.X.zero_()
    call("dga_bse_solve_sum_tuned_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, lp.inv_beta2, p(lp.gamma_cm),
         p(lp.chi0_inv), p(lp.uv), p(lp.work), lp.n_items, 1, lp.refine_max_iter, lp.refine_tol, p(lp.X),
         p(lp.bse_status), p(lp.bse_iters), ctypes.byref(t), p(scratch), scratch.numel() * 16, s)
    torch.cuda.synchronize()
    status = lp.bse_status.cpu().numpy()
    assert np.all(status & WAIT_TIMEOUT), status
    assert np.all((status & ~(WAIT_TIMEOUT | NONFINITE | 4)) == 0), status
    call("dga_bse_resolve_fp64_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, lp.inv_beta2, p(lp.gamma_cm),
         p(lp.chi0_inv), p(lp.uv), p(lp.work), lp.n_items, p(lp.X), p(lp.bse_status), lp.resolve_grid,
         p(lp.bse_scratch), lp.bse_scratch.numel() * 16, s)
    torch.cuda.synchronize()
    assert int(lp.bse_status.abs().sum()) == 0
    assert rel_err(lp.X.cpu().numpy(), x64) < 1e-12
    # the same pass afterwards, with the default limit, is clean (the context and the kernel are still usable)
    lp.set_tuning((kernel, 0))
    lp.bse()
    torch.cuda.synchronize()
    assert int(lp.bse_status.abs().sum()) == 0
    assert rel_err(lp.X.cpu().numpy(), x64) < 1e-10
