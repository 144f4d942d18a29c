"""The local Schwinger-Dyson oracle against the upstream run (tests/golden/local_sde.npz), without a GPU.

* oracle/local_sde.py reproduces all 11 results of upstream ``local_sde.perform_local_schwinger_dyson`` in FP64
  on four seeded cases (1, 2 and 3 orbitals, with and without a shell) to 1e-12 relative;
* the fixtures' two-particle functions were made from the model vertex, so the upstream's Gamma_r equals it
  (a round trip through both channels' inversions);
* the closed form of the shell correction that the device uses (csrc/local_sde.cu: Gamma = beta^2 chi^-1 -
  delta beta^2 chi0^-1 + U_r - U_eff, U_eff = U_r [1 + (S_full - S_core) U_r]^-1) equals the upstream's dense
  inversions of the full-box chi~;
* the C entries reject bad sizes before launching anything.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
from oracle import local_sde as osde

CASES = ("l1", "l2", "l3", "l3s")
RESULTS = ("gamma_d", "gamma_m", "chi_d", "chi_m", "vrg_d", "vrg_m", "f_d", "f_m", "gchi_d", "gchi_m", "sigma_loc")


def load(case: str) -> dict:
    z = np.load(os.path.join(GOLDEN, "local_sde.npz"), allow_pickle=False)
    return {k[len(case) + 1:]: z[k] for k in z.files if k.startswith(case + "_")}


def inputs(d: dict) -> tuple:
    niw, niv, sh = (int(x) for x in d["box"])
    g2d, g2m = osde.full_niw(d["g2_dens_half"], 3), osde.full_niw(d["g2_magn_half"], 3)
    return d["g"], g2d, g2m, d["u"], float(d["beta"]), niw, niv, sh, d["occ"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_upstream(case):
    d = load(case)
    res = osde.perform_local_schwinger_dyson(*inputs(d))
    for name, r in zip(RESULTS, res):
        assert r.shape == d[name].shape, name
        assert rel_err(r, d[name]) < 1e-12, name


@pytest.mark.parametrize("case", CASES)
def test_upstream_gamma_is_the_model_vertex(case):
    d = load(case)
    assert rel_err(d["gamma_d"], d["gamma_model_dens"]) < 1e-12
    assert rel_err(d["gamma_m"], d["gamma_model_magn"]) < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_closed_form_shell_correction(case):
    d = load(case)
    g, g2d, g2m, u, beta, niw, niv, sh, _ = inputs(d)
    n = u.shape[0]
    n2 = n * n
    chi0h = osde.half_niw(osde.local_bubble(g, niw, niv + sh, beta), 2)
    core = chi0h[..., sh : sh + 2 * niv]
    ds = (chi0h.sum(-1) - core.sum(-1)) / beta**2
    for ch, g2, key in (("dens", g2d, "gamma_d"), ("magn", g2m, "gamma_m")):
        u_r = osde.u_as_channel(u, ch)
        uc = u_r.transpose(0, 1, 3, 2).reshape(n2, n2)
        gchi = osde.generalized_chi(g2, g, beta, niv, ch == "dens")
        gam = beta**2 * osde.inv_dense(gchi) - beta**2 * osde.extend_diag(osde.inv_diag(core))
        for w in range(niw + 1):
            s = ds[..., w].transpose(0, 1, 3, 2).reshape(n2, n2)
            u_eff = uc @ np.linalg.inv(np.eye(n2) + s @ uc)
            gam[..., w, :, :] += (uc - u_eff).reshape(n, n, n, n).transpose(0, 1, 3, 2)[..., None, None]
        assert rel_err(gam, d[key]) < 1e-12, ch


def test_local_entries_reject_bad_sizes_without_launching():
    from dgamore_b200._lib import SIGNATURES, lib

    L = lib()
    fake = ctypes.c_void_p(16)
    null = ctypes.c_void_p(0)
    # G holds too few frequencies for the bubble box
    assert L.dga_local_bubble_c128(fake, 1, 4, 5, 4, 10.0, fake, null) != 0
    # the frequency offset of G2 leaves its bosonic axis
    assert L.dga_local_chi_c128(fake, 1, 4, 5, 3, 6, fake, 20, 10.0, 1, fake, null) != 0
    # more than 4 orbitals
    assert L.dga_local_ucorr_c128(fake, fake, fake, 5, 3, fake, fake, null) != 0
    # dense LU beyond its size limit, and a solve whose output cannot hold its column blocks
    assert L.dga_lu_batched_c128(fake, 9000, 1, 9000 * 9000, fake, fake, null) != 0
    assert L.dga_lu_solve_batched_c128(fake, fake, 20, 1, 400, null, 0, 0, 0, 20, fake, 20 * 20, fake, null) != 0
    assert b"invalid" in L.dga_last_error_string()
    assert all(name in SIGNATURES for name in ("dga_local_gamma_c128", "dga_local_fvertex_operands_c128",
                                                "dga_local_sigma_c128"))
