"""GPU parity of the FP64 device pass against the upstream FP64 outputs (golden fixtures) and the oracle.

Tolerance: the FP64 drop-in bar is 1e-10 relative (max abs error / max abs value) on every intermediate;
the lambda values agree to 1e-10 absolute.
"""

import numpy as np
import pytest
import torch

from conftest import GOLDEN_CONFIGS, load_golden, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module", params=GOLDEN_CONFIGS)
def device_pass(request):
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(request.param)
    lp = LadderPass(inp)
    lp.run()
    torch.cuda.synchronize()
    return request.param, inp, ref, lp


def test_bubble(device_pass):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.chi0_ref_layout(), ref["chi0"]) < TOL


def test_chi0_inverse(device_pass):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.orbmat_ref_layout(lp.chi0_inv), ref["chi0_inv"]) < TOL


def test_double_counting_kernel(device_pass):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.orbmat_ref_layout(lp.k_dc), ref["kernel_dc"]) < TOL


@pytest.mark.parametrize("ch,chname", [(0, "dens"), (1, "magn")])
def test_bse_solve_sum(device_pass, ch, chname):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.x_ref_layout(ch), ref[f"chi_aux_sum_{chname}"]) < TOL
    assert int(lp.bse_status.abs().sum().item()) == 0


@pytest.mark.parametrize("ch,chname", [(0, "dens"), (1, "magn")])
def test_chi_phys_and_lambda(device_pass, ch, chname):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.chi_phys_ref_layout(lp.chi_phys, ch), ref[f"chi_phys_{chname}_before_lambda"]) < TOL
    if lp.do_lambda:
        lam = lp.lambdas.cpu().numpy()[ch]
        assert abs(lam - float(ref[f"lambda_{chname}"])) < 1e-10 * max(1.0, abs(lam))
        # the application 1/(1/chi + lambda) amplifies the last-Newton-step rounding of lambda near the
        # divergence, so it is checked against the oracle applied with the device's own lambda
        from oracle import ladder as oracle

        expect = oracle.apply_lambda(ref[f"chi_phys_{chname}_before_lambda"], lam)
        assert rel_err(lp.chi_phys_ref_layout(lp.chi_lam, ch), expect) < TOL
        assert rel_err(lp.chi_phys_ref_layout(lp.chi_lam, ch), ref[f"chi_phys_{chname}"]) < 1e-7
        assert int(lp.lambda_iters.cpu().numpy()[ch]) < 1000


def test_vertex_gamma(device_pass):
    name, inp, ref, lp = device_pass
    for ch, chname in ((0, "dens"), (1, "magn")):
        g = lp.orbmat_ref_layout(lp.gamma3[ch])
        assert rel_err(g, ref[f"vrg_{chname}"]) < TOL


def test_kernel(device_pass):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.orbmat_ref_layout(lp.K), ref["kernel"]) < TOL


def test_sigma(device_pass):
    name, inp, ref, lp = device_pass
    assert rel_err(lp.sigma.cpu().numpy(), ref["sigma"]) < TOL
    assert int(lp.status.abs().sum().item()) == 0


def test_e2e_host_roundtrip(device_pass):
    name, inp, ref, lp = device_pass
    sig = lp.run_e2e()
    assert rel_err(sig, ref["sigma"]) < TOL


def test_dense_invert_sum_known_answer():
    """FourPoint.invert_and_sum_over_last_vn on the upstream KAT input (tests/test_four_point.py:46-63)."""
    import os

    from conftest import REPO
    from dgamore_b200.four_point import invert_and_sum_over_last_vn

    kat = np.load(os.path.join(REPO, "tests/golden/bse_kat.npz"))
    rng = np.random.default_rng(1234)
    shape = (16, 2, 2, 2, 2, 7, 6, 6)
    mat = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    out = invert_and_sum_over_last_vn(mat[..., 3:, :, :], float(kat["beta"]))
    assert rel_err(out, kat["v1"]) < TOL


def test_lambda_without_root_reports_nonconvergence():
    """A negative target has no root above lambda_start: the device stops and flags DGA_ITEM_NOCONVERGE."""
    import ctypes

    from dgamore_b200 import _lib

    Q, W = 6, 5
    rng = np.random.default_rng(7)
    chi = torch.tensor(0.1 + 0.05 * rng.random((1, Q, W)) + 0j, dtype=torch.complex128, device="cuda")
    weights = torch.tensor([1, 2, 2, 4, 4, 3], dtype=torch.int64, device="cuda")
    target = torch.tensor([-0.5 + 0j], dtype=torch.complex128, device="cuda")
    lam = torch.zeros(1, dtype=torch.float64, device="cuda")
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.empty_like(chi)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.call("dga_lambda_c128", p(chi), Q, W, 1, p(weights), p(target), 10.0, 16.0, 0.1, 1e-7, 1000, p(lam), p(iters),
              p(status), p(out), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(status.item()) & 4
    assert np.isfinite(lam.item())


@pytest.fixture(scope="module", params=GOLDEN_CONFIGS)
def mixed_pass(request):
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(request.param)
    lp = LadderPass(inp, precision="mixed", refine_tol=1e-12)
    lp.run()
    torch.cuda.synchronize()
    return request.param, inp, ref, lp


def test_mixed_bse_matches_fp64_reference(mixed_pass):
    """Mixed form (FP32 LU + FP64 refinement to 1e-12): every solve converges and matches the upstream FP64 BSE."""
    name, inp, ref, lp = mixed_pass
    for ch, chname in ((0, "dens"), (1, "magn")):
        assert rel_err(lp.x_ref_layout(ch), ref[f"chi_aux_sum_{chname}"]) < 1e-11
    assert int(lp.bse_status.abs().sum().item()) == 0
    iters = lp.bse_iters.cpu().numpy()
    assert iters.max() <= lp.refine_max_iter and iters.min() >= 1


def test_mixed_sigma_error_bound(mixed_pass):
    """Sigma from the mixed pass is within 1e-8 of the FP64 upstream Sigma (the mixed-form bound)."""
    name, inp, ref, lp = mixed_pass
    assert rel_err(lp.sigma.cpu().numpy(), ref["sigma"]) < 1e-8


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_mixed_sigma_bound_at_default_tolerance(name):
    """With the default refinement tolerance (1e-10) Sigma is still within the 1e-8 mixed-form bound."""
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(name)
    lp = LadderPass(inp, precision="mixed", keep_intermediates=False)
    lp.run()
    torch.cuda.synchronize()
    assert int(lp.bse_status.abs().sum().item()) == 0
    assert rel_err(lp.sigma.cpu().numpy(), ref["sigma"]) < 1e-8
