"""The files a device pass writes in the upstream's conventions (dgamore_b200/outputs.py).

After one pass of the t3 golden configuration: Σ, χ_phys and the Eliashberg hand-off read back equal to the
pass's device arrays in the upstream layouts, χ_phys matches the upstream's own χ_phys output, and a restart
picks up the written Σ.
"""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


def test_pass_outputs_and_restart(tmp_path):
    from dgamore_b200 import outputs
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden("t3")
    lp = LadderPass(inp)
    lp.run()
    torch.cuda.synchronize()
    out = tmp_path / outputs.output_dir_name(lp.sh.nk_tot, lp.sh.nk_tot, lp.sh.niw, lp.sh.niv, lp.sh.niv_shell)
    eli = out / "Eliashberg"
    written = outputs.save_pass(lp, str(out), 1, eliashberg_dir=str(eli), mu_history=[0.25, 0.26])
    names = {p.split("/")[-1] for p in written}
    assert {"sigma_dga_iteration_1.npy", "chi_phys_q_dens.npy", "chi_phys_q_magn.npy", "mu_history.npy",
            "gchi0_q_rank_0.npy", "gchi0_q_inv_rank_0.npy", "gchi_aux_q_magn_sum_rank_0.npy"} <= names
    sigma = np.load(out / "sigma_dga_iteration_1.npy")
    np.testing.assert_array_equal(sigma, lp.sigma.cpu().numpy())
    chi_r = lp.chi_lam if lp.do_lambda else lp.chi_phys
    for ch, name in enumerate(("dens", "magn")):
        saved = np.load(out / f"chi_phys_q_{name}.npy")
        np.testing.assert_array_equal(saved, lp.chi_phys_ref_layout(chi_r, ch))
    assert rel_err(np.load(out / "chi_phys_q_magn.npy"), ref["chi_phys_magn"]) < 1e-10
    got, it = outputs.get_starting_sigma(str(out), None)
    assert it == 1
    np.testing.assert_array_equal(got, sigma)
