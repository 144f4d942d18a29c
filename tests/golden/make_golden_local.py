"""Generates tests/golden/local_sde.npz by running the upstream local Schwinger-Dyson equation on seeded inputs.

Run in a container that holds the upstream sources (DGAMORE_REFERENCE_ROOT, see _ref_harness.py):

    python tests/golden/make_golden_local.py

For each case: the local G(nu) is the k-mean of the synthetic configuration's lattice G (Hubbard-I self-energy);
the two-particle Green's functions are made so that the local SDE returns the synthetic model vertex Gamma_r
(dgamore_b200/synthetic.py gamma_model) in the core box:

    chi_r = [chi~_core^-1 + (Gamma_r - U_r)/beta^2]^-1,  G2_r = chi_r / beta
            (+ 2 G_ab(nu) G_cd(nu') at w = 0 in the density channel),

with chi~_core^-1 the shell-corrected bubble term of create_gamma_r_with_shell_correction (oracle/local_sde.py
chi_tilde_core_inv),

extended to the full w range by the time-reversal rule.  upstream ``local_sde.perform_local_schwinger_dyson``
(``IHaveMat.mat`` patched to keep complex128) then gives the 11 results stored as ``{case}_{name}``; G2 is
stored in its w >= 0 half (the full range follows exactly from it).  The upstream needs an even niw_core.
"""

from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import _ref_harness as harness  # noqa: E402

harness.install()
harness.patch_fp64()

from dgamore import config, local_sde  # noqa: E402
from dgamore.greens_function import GreensFunction  # noqa: E402
from dgamore.interaction import LocalInteraction  # noqa: E402
from dgamore.local_four_point import LocalFourPoint  # noqa: E402
from dgamore.n_point_base import SpinChannel  # noqa: E402

from dgamore_b200 import synthetic  # noqa: E402
from dgamore_b200.kgrid import KGrid  # noqa: E402
from oracle import local_sde as osde  # noqa: E402

# name: (synthetic configuration, niw_core, niv_core, niv_shell)
CASES = {
    "l1": ("t1b", 4, 6, 4),
    "l2": ("t4e", 2, 4, 2),
    "l3": ("t3", 2, 3, 0),
    "l3s": ("t3", 2, 2, 2),
}

RESULTS = ("gamma_d", "gamma_m", "chi_d", "chi_m", "vrg_d", "vrg_m", "f_d", "f_m", "gchi_d", "gchi_m", "sigma_loc")


class _Logger:
    def info(self, *a, **k):
        pass

    debug = warning = info


def make_inputs(name: str) -> dict:
    base, niw, niv, niv_shell = CASES[name]
    cfg = dataclasses.replace(synthetic.CONFIGS[base], niw=niw, niv=niv, niv_shell=niv_shell)
    rng = np.random.default_rng(cfg.seed + 101)
    grid = KGrid(cfg.nk, cfg.symmetries)
    ek = synthetic.dispersion(cfg, grid)
    mu = synthetic.find_mu(cfg, ek)
    niv_g = niv + niv_shell + niw + 4
    g_loc = synthetic.g_lattice(ek, synthetic.hubbard_i_sigma(cfg, mu, niv_g), mu, cfg.beta).mean(axis=(0, 1, 2))
    u = synthetic.kanamori_u(cfg)
    beta = cfg.beta
    chi0_half = osde.half_niw(osde.local_bubble(g_loc, niw, niv + niv_shell, beta), 2)
    out = {"g": g_loc, "u": u, "beta": beta, "box": np.array([niw, niv, niv_shell])}
    for ch in ("dens", "magn"):
        u_r = osde.u_as_channel(u, ch)
        gamma = synthetic.gamma_model(cfg, u, ch, rng, niv)
        a = osde.chi_tilde_core_inv(chi0_half, u_r, beta, niv) + (gamma - u_r[..., None, None, None]) / beta**2
        g2 = osde.inv_dense(a) / beta
        if ch == "dens":
            gs = g_loc[..., g_loc.shape[-1] // 2 - niv : g_loc.shape[-1] // 2 + niv]
            g2[:, :, :, :, 0] += 2.0 * gs[:, :, None, None, :, None] * gs[None, None, :, :, None, :]
        out[f"g2_{ch}_half"] = g2
        out[f"gamma_model_{ch}"] = gamma
    out["occ"] = synthetic.make_occupations(cfg)[0]
    return out


def run_upstream(inp: dict) -> dict:
    niw, niv, niv_shell = (int(x) for x in inp["box"])
    config.logger = _Logger()
    config.sys.beta = float(inp["beta"])
    config.sys.occ_dmft = inp["occ"]
    config.box.niw_core = niw
    config.box.niv_core = niv
    config.box.niv_shell = niv_shell
    config.box.niv_full = niv + niv_shell
    config.dmft.symmetrize_orbitals = []
    config.eliashberg.perform_eliashberg = False
    g_dmft = GreensFunction(inp["g"].copy())
    g2_d = LocalFourPoint(osde.full_niw(inp["g2_dens_half"], 3), SpinChannel.DENS, 1, 2)
    g2_m = LocalFourPoint(osde.full_niw(inp["g2_magn_half"], 3), SpinChannel.MAGN, 1, 2)
    res = local_sde.perform_local_schwinger_dyson(g_dmft, g2_d, g2_m, LocalInteraction(inp["u"].copy()))
    return {k: np.asarray(v.mat) for k, v in zip(RESULTS, res)}


def main():
    fix = {}
    for name in CASES:
        inp = make_inputs(name)
        res = run_upstream(inp)
        for k, v in list(inp.items()) + list(res.items()):
            fix[f"{name}_{k}"] = np.asarray(v)
        print(name, {k: v.shape for k, v in res.items()})
    path = os.path.join(HERE, "local_sde.npz")
    np.savez_compressed(path, **fix)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
