"""Mixing of successive self-energies (dgamore_b200/selfconsistency.apply_mixing; CPU) against the upstream's
apply_mixing_strategy run in FP64 (tests/golden/glue.npz): linear, Pulay and Anderson with a history of three
earlier self-energies read back from sigma_dga_iteration_{N}.npy files, to 1e-12 relative."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err


@pytest.mark.parametrize("name", ["g1", "g3"])
@pytest.mark.parametrize("strategy", ["linear", "pulay", "anderson"])
def test_mixing_matches_the_upstream(tmp_path, name, strategy):
    from dgamore_b200 import outputs, selfconsistency as sc

    d = np.load(os.path.join(GOLDEN, "glue.npz"))
    c = {k[3:]: d[k] for k in d.files if k.startswith(name + "_")}
    for i, h in enumerate(c["hist"]):
        outputs.save_sigma_iteration(h, str(tmp_path), i + 1)
    niv_core = c["sigma"].shape[-1] // 4
    got = sc.apply_mixing(strategy, c["sigma_new"].copy(), c["sigma_old"], c["sigma_dmft"], 4, 3, 0.3, niv_core,
                          str(tmp_path))
    assert rel_err(got, c[f"mix_{strategy}"]) < 1e-12
