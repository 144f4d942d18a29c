"""Generates tests/golden/glue.npz by running the upstream's self-consistency glue on seeded inputs.

Run in a container that holds the upstream sources (DGAMORE_REFERENCE_ROOT, see _ref_harness.py):

    python tests/golden/make_golden_glue.py

Two cases: 1 orbital on 8x8 (niv = 40, β = 10) and 3 orbitals on 4x4 (niv = 20, β = 20).  e_k is the synthetic
configurations' dispersion (dgamore_b200/synthetic.py); Σ(k, ν) = Σ_HubbardI(ν) + δ_k/(iν + 1) with δ_k a seeded
Hermitian n×n matrix per k of norm ~0.1.  For each case the upstream functions give, in FP64 (``IHaveMat.mat``
patched to keep complex128): SelfEnergy.fit_smom; get_total_fill at μ0; update_mu to the filling at μ0 + 0.1;
GreensFunction.get_g_full; GreensFunction.get_fill_nonlocal; and apply_mixing_strategy (linear, Pulay and
Anderson, history of 3 earlier self-energies written as sigma_dga_iteration_{1..3}.npy, current iteration 4,
α = 0.3, core window niv/2).
"""

from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import _ref_harness as harness  # noqa: E402

harness.install()
harness.patch_fp64()

from dgamore import config, nonlocal_sde  # noqa: E402
import dgamore.brillouin_zone as bz  # noqa: E402
from dgamore import greens_function  # noqa: E402
from dgamore.greens_function import GreensFunction  # noqa: E402
from dgamore.self_energy import SelfEnergy  # noqa: E402

from dgamore_b200 import synthetic  # noqa: E402
from dgamore_b200.kgrid import KGrid  # noqa: E402

CASES = {"g1": ("t1b", (8, 8, 1), 40, 10.0), "g3": ("t3", (4, 4, 1), 20, 20.0)}


class _Logger:
    def info(self, *a, **k):
        pass

    debug = warning = info


def make_case(name: str) -> dict:
    base, nk, niv, beta = CASES[name]
    cfg = synthetic.CONFIGS[base]
    import dataclasses

    cfg = dataclasses.replace(cfg, nk=nk, beta=beta)
    grid = KGrid(cfg.nk, cfg.symmetries)
    ek = synthetic.dispersion(cfg, grid)  # [kx, ky, kz, n, n]
    n = cfg.n_bands
    nk_tot = int(np.prod(nk))
    mu0 = synthetic.find_mu(cfg, ek)
    sig_loc = synthetic.hubbard_i_sigma(cfg, mu0, niv)  # [n, n, 2 niv]
    rng = np.random.default_rng(2024 + n)
    d = rng.standard_normal((nk_tot, n, n)) + 1j * rng.standard_normal((nk_tot, n, n))
    d = 0.05 * (d + np.conj(np.swapaxes(d, -1, -2)))
    iv = 1j * (2 * np.arange(-niv, niv) + 1) * np.pi / beta
    sigma = sig_loc[None] + d[..., None] / (iv[None, None, None, :] + 1.0)  # [Nk, n, n, 2 niv]

    config.logger = _Logger()
    config.sys.beta = beta
    config.sys.n_bands = n
    config.sys.mu = mu0
    config.lattice.nk = nk
    config.lattice.nq = nk
    config.lattice.k_grid = bz.KGrid(nk, symmetries=bz.two_dimensional_square_symmetries())
    config.lattice.q_grid = config.lattice.k_grid
    config.box.niv_core = niv // 2

    out = {"ek": ek.reshape(nk_tot, n, n), "sigma": sigma, "beta": beta, "mu0": mu0, "nk": np.array(nk)}
    siw = SelfEnergy(sigma.copy(), nk, True, True, False)
    smom0, smom1 = siw.fit_smom()
    out["smom0"], out["smom1"] = smom0, smom1
    out["fill_mu0"] = greens_function.get_total_fill(mu0, ek, sigma.copy(), beta, smom0)
    target = greens_function.get_total_fill(mu0 + 0.1, ek, sigma.copy(), beta, smom0)
    out["target"] = target
    out["mu_new"] = greens_function.update_mu(mu0, target, ek, sigma.copy(), beta, smom0)
    g = GreensFunction.get_g_full(SelfEnergy(sigma.copy(), nk, True, True, False), mu0, ek)
    out["g_full"] = g.mat.reshape(nk_tot, n, n, 2 * niv)
    n_el, occ, occ_k = g.get_fill_nonlocal()  # at config.sys.mu = mu0, with the Σ get_g_full decompressed
    out["n_el"], out["occ"], out["occ_k"] = n_el, occ, occ_k.reshape(nk_tot, n, n)

    # mixing: a history of three earlier self-energies, this iteration's result and the DMFT one
    hist = [sigma * (1.0 + 0.02 * (i + 1)) + 0.01j * (i + 1) for i in range(3)]
    sigma_old = hist[-1]
    sigma_new = sigma * 0.97 + 0.015
    sigma_dmft = sig_loc[None]
    out["hist"] = np.stack(hist)
    out["sigma_new"], out["sigma_old"], out["sigma_dmft"] = sigma_new, sigma_old, sigma_dmft
    with tempfile.TemporaryDirectory() as tmp:
        for i, h in enumerate(hist):
            np.save(os.path.join(tmp, f"sigma_dga_iteration_{i + 1}.npy"), h)
        config.output.output_path = tmp
        config.self_consistency.previous_sc_path = ""
        config.self_consistency.mixing_history_length = 3
        config.self_consistency.mixing = 0.3
        config.lattice.k_grid = bz.KGrid(nk, symmetries=bz.two_dimensional_square_symmetries())
        for strategy in ("linear", "pulay", "anderson"):
            config.self_consistency.mixing_strategy = strategy
            res = nonlocal_sde.apply_mixing_strategy(
                SelfEnergy(sigma_new.copy(), nk, True, True, False),
                SelfEnergy(sigma_old.copy(), nk, True, True, False),
                SelfEnergy(sigma_dmft.copy(), (1, 1, 1), True, True, False), 4)
            out[f"mix_{strategy}"] = np.asarray(res.mat)
    return out


def main():
    fix = {}
    for name in CASES:
        for k, v in make_case(name).items():
            fix[f"{name}_{k}"] = np.asarray(v)
    path = os.path.join(HERE, "glue.npz")
    np.savez_compressed(path, **fix)
    print("wrote", path, sorted(fix)[:6], "...")


if __name__ == "__main__":
    main()
