"""GPU parity of the BSE at the full compound size of the 3-orbital configuration (N = 9 x 80 = 720).

The golden configurations have compound sizes up to a few hundred, so the tensor-core panel kernel (the mixed
default from N = 320) runs there with one or two row tiles per strip.  This case keeps the 3-orbital
configuration's orbitals and fermionic box (niv = 40, so N = 720: 23 panels, up to six 128-row tiles per strip)
on a 4x4 momentum grid (6 irreducible q) with niw = 2, 36 solves in all:

* the FP64 drop-in BSE against the oracle's linear solve (numpy, the upstream's invert_and_sum_over_last_vn_v2,
  four_point.py:644-684) on the corner (q, w) items of both channels, at the FP64 bar of 1e-10 relative;
* every mixed kernel choice, refined to 1e-12, against the FP64 device result at 1e-10 relative;
* Sigma of the mixed pass at its default refinement tolerance against Sigma of the FP64 pass, within the
  mixed-form bound of 1e-8 relative.
"""

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    from dgamore_b200 import synthetic
    from dgamore_b200.pipeline import LadderPass
    from dgamore_b200.profile_case import reduced_config

    inp = synthetic.make_inputs(reduced_config("c3", 4, 2))
    lp = LadderPass(inp, keep_intermediates=False)
    assert lp.sh.N == 720
    lp.run()
    torch.cuda.synchronize()
    x64 = [lp.x_ref_layout(ch) for ch in (0, 1)]
    sigma64 = lp.sigma.cpu().numpy()
    assert int(lp.bse_status.abs().sum()) == 0
    del lp
    torch.cuda.empty_cache()
    return inp, x64, sigma64


def test_fp64_bse_matches_oracle_at_n720(case):
    from oracle import ladder as oracle

    inp, x64, _ = case
    beta, niw, niv_core = inp["beta"], inp["niw"], inp["niv_core"]
    chi0 = oracle.chi0_q_fft(inp["g_k"], niw, niv_core + inp["niv_shell"], inp["irrk_ind"], beta)
    chi0_core_inv = oracle.chi0_inv(oracle.cut_niv(chi0, niv_core, 1))
    qs = [0, chi0_core_inv.shape[0] - 1]
    ws = [0, chi0_core_inv.shape[5] - 1]
    for ch, chname in ((0, "dens"), (1, "magn")):
        uv = oracle.u_as_channel(inp["u"], chname)[None] + oracle.v_as_channel(inp["v_q_irr"], chname)
        ref = oracle.bse_sum_solve(chi0_core_inv[qs][..., ws, :], inp[f"gamma_{chname}"][..., ws, :, :], uv[qs], beta)
        got = x64[ch][qs][..., ws, :]
        assert rel_err(got, ref) < 1e-10, chname


def test_mixed_choices_match_fp64_at_n720(case):
    from dgamore_b200.autotune import CANDIDATES, scratch_bytes
    from dgamore_b200.pipeline import LadderPass

    inp, x64, _ = case
    lp = LadderPass(inp, keep_intermediates=False, precision="mixed", refine_tol=1e-12)
    lp.pre_bse()
    ran = 0
    for choice in CANDIDATES["mixed"]:
        if scratch_bytes(lp, lp.n_items, 1, choice) == 0:
            continue
        lp.set_tuning(choice)
        lp.X.zero_()
        lp.bse()
        torch.cuda.synchronize()
        assert int(lp.bse_status.abs().sum()) == 0, choice
        for ch in (0, 1):
            assert rel_err(lp.x_ref_layout(ch), x64[ch]) < 1e-10, (choice, ch)
        ran += 1
    assert ran >= 3  # the tensor-core panel kernel, the FP32-tile panel kernel and the 128-thread kernel


def test_mixed_sigma_bound_at_n720(case):
    from dgamore_b200.pipeline import LadderPass

    inp, _, sigma64 = case
    lp = LadderPass(inp, keep_intermediates=False, precision="mixed")
    lp.run()
    torch.cuda.synchronize()
    assert int(lp.bse_status.abs().sum()) == 0
    assert rel_err(lp.sigma.cpu().numpy(), sigma64) < 1e-8
