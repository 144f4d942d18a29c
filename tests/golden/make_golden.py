"""Generates the golden fixtures under tests/golden/ by running the upstream DGAmore code itself.

Run in a container that holds the upstream sources, at the path given by the DGAMORE_REFERENCE_ROOT environment
variable (see _ref_harness.py); the sources are not needed where the tests run, the committed .npz files are:

    python tests/golden/make_golden.py

For each small synthetic configuration (``dgamore_b200.synthetic.CONFIGS``: t1, t1b, t2, t3, and t3a, whose
anisotropic t2g hoppings are reduced by the upstream's symmetry discovery with per-k orbital rotations) it builds the
inputs of one nonlocal pass, then replays the upstream call sequence of ``calculate_self_energy_q``
(dgamore/nonlocal_sde.py:786-879) with the upstream functions, in FP64 (``IHaveMat.mat`` patched to keep
complex128), and stores inputs and every intermediate into ``<name>.npz``.

It also copies the upstream's own end-to-end fixtures that pin the bubble (``g_dga.npy``,
``gchi0_q_rank_0.npy``, ``gchi0_q_inv_rank_0.npy`` from tests/test_data/end_2_end) and the lambda-correction
fixtures (tests/test_data/lambda_correction/{sp,spch}) into ``upstream_fixtures.npz``, and the upstream BSE
known-answer case (tests/test_four_point.py:466-532, rng 1234) into ``bse_kat.npz``.
"""

from __future__ import annotations

import os
import sys
from copy import deepcopy

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import _ref_harness as harness  # noqa: E402

harness.install()
harness.patch_fp64()

from dgamore import config  # noqa: E402
import dgamore.brillouin_zone as bz  # noqa: E402
import dgamore.lambda_correction as lc  # noqa: E402
from dgamore import nonlocal_sde, mpi_utils  # noqa: E402
from dgamore.bubble_gen import BubbleGenerator  # noqa: E402
from dgamore.four_point import FourPoint  # noqa: E402
from dgamore.greens_function import GreensFunction  # noqa: E402
from dgamore.interaction import LocalInteraction, Interaction  # noqa: E402
from dgamore.local_four_point import LocalFourPoint  # noqa: E402
from dgamore.n_point_base import SpinChannel  # noqa: E402
from dgamore.self_energy import SelfEnergy  # noqa: E402
from dgamore import eliashberg_solver  # noqa: E402
from dgamore.n_point_base import FrequencyNotation  # noqa: E402

from dgamore_b200 import synthetic  # noqa: E402

UPSTREAM_DATA = os.path.join(harness.REFERENCE_ROOT, "tests", "test_data")


class _Logger:
    def info(self, *a, **k):
        pass

    debug = warning = info

    def log_memory_usage(self, *a, **k):
        pass


def _setup_config(cfg: synthetic.DgaConfig, inp: dict):
    config.logger = _Logger()
    config.sys.beta = cfg.beta
    config.sys.n_bands = cfg.n_bands
    config.sys.mu = inp["mu"]
    config.box.niw_core = cfg.niw
    config.box.niv_core = cfg.niv
    config.box.niv_shell = cfg.niv_shell
    config.box.niv_full = cfg.niv_full
    config.lattice.nk = tuple(cfg.nk)
    config.lattice.nq = tuple(cfg.nk)
    config.lattice.k_grid = bz.KGrid(tuple(cfg.nk), symmetries=bz.two_dimensional_square_symmetries())
    config.lattice.q_grid = config.lattice.k_grid
    config.eliashberg.perform_eliashberg = False
    config.self_consistency.restrict_chi_phys = False
    config.lambda_correction.perform_lambda_correction = False


class _OnlyKeys(dict):
    """A result dict that keeps only the named keys (the at-size fixtures store a few outputs; the upstream's
    intermediates at the 3-orbital size are gigabytes each)."""

    def __init__(self, keys):
        super().__init__()
        self._keys = set(keys)

    def __setitem__(self, key, value):
        if key in self._keys:
            super().__setitem__(key, value)


def run_reference_pass(name: str, variants: bool = True, bse_variant: str = "v1", keep_keys=None) -> dict:
    """The upstream pass in FP64; with ``variants`` also its alternative forms (direct-q bubble, v3 BSE, direct
    Sigma), which the at-size fixtures skip because they cost far more than the pass at 64x64.  ``bse_variant``
    "v3" takes the auxiliary sums from the upstream's q-by-q form (nonlocal_sde.py:129-156) instead of the
    materialised v1 (nonlocal_sde.py:85-126); ``keep_keys`` names the outputs to keep."""
    cfg = synthetic.CONFIGS[name]
    inp = synthetic.make_inputs(cfg)
    _setup_config(cfg, inp)
    if name in AUTO_CONFIGS:
        # the upstream's symmetry discovery on H(k) (brillouin_zone.py:365-449, DGAmore.py:98-109): its irreducible
        # wedge and per-k orbital rotations replace the synthetic grid's and travel with the inputs
        auto = bz.KGrid(tuple(cfg.nk), symmetries=bz.get_lattice_symmetries_from_string("auto"))
        auto.specify_auto_symmetries(inp["ek"])
        config.lattice.k_grid = auto
        config.lattice.q_grid = auto
        nk_tot, nb = int(np.prod(cfg.nk)), cfg.n_bands
        inp["irrk_ind"] = np.asarray(auto.irrk_ind)
        inp["irrk_inv"] = np.asarray(auto.irrk_inv).ravel()
        inp["irrk_count"] = np.asarray(auto.irrk_count)
        inp["v_q_irr"] = np.asarray(inp["v_q_full"])[inp["irrk_ind"]]
        inp["orbital_us"] = np.asarray(auto._auto_us).reshape(nk_tot, nb, nb).astype(np.complex128)
        inp["orbital_sigmas"] = np.asarray(auto._auto_sigmas).reshape(nk_tot).astype(np.float64)
        inp["orbital_conjs"] = np.asarray(auto._auto_conjs).reshape(nk_tot).astype(bool)
    grid = config.lattice.q_grid
    assert np.array_equal(grid.irrk_ind, inp["irrk_ind"]), "irreducible wedge differs from upstream"
    assert np.array_equal(grid.irrk_inv.ravel(), inp["irrk_inv"]), "irreducible inverse map differs"
    assert np.array_equal(grid.irrk_count, inp["irrk_count"]), "irreducible counts differ"

    beta = cfg.beta
    dist = harness.FakeDistributor(grid.nk_irr)
    giwk = GreensFunction(inp["g_k"], None, None, True, False, False)
    u_loc = LocalInteraction(inp["u"])
    v_full = Interaction(inp["v_q_full"].reshape(*cfg.nk, *inp["v_q_full"].shape[1:]), SpinChannel.NONE, tuple(cfg.nk))
    irr_q_list = grid.get_irrq_list()
    v_nonloc = v_full.reduce_q(irr_q_list)

    out = {} if keep_keys is None else _OnlyKeys(keep_keys)
    # bubble (nonlocal_sde.py:801-809)
    gchi0_q = BubbleGenerator.create_generalized_chi0_q_fft_cpu(dist, giwk, cfg.niw, cfg.niv_full, grid, beta)
    out["chi0"] = gchi0_q.mat.copy()
    # direct-q bubble variant (bubble_gen.py:147-183)
    if variants:
        gchi0_direct = BubbleGenerator.create_generalized_chi0_q_cpu(giwk, cfg.niw, cfg.niv_full, irr_q_list, grid,
                                                                     beta)
        out["chi0_direct"] = gchi0_direct.mat.copy()

    # double-counting kernel (nonlocal_sde.py:817-820)
    f_dc_loc = 2 * LocalFourPoint(inp["f_magn_loc"], SpinChannel.NONE, 1, 2, False, True).permute_orbitals("abcd->cbad")
    kernel = -nonlocal_sde.calculate_sigma_dc_kernel(f_dc_loc, gchi0_q, u_loc)
    out["kernel_dc"] = -kernel.mat.copy()

    # chi0 sums and inverse (nonlocal_sde.py:824-835)
    gchi0_q_full_sum = 1.0 / beta * gchi0_q.sum_over_all_vn(beta)
    gchi0_q_core = gchi0_q.cut_niv(cfg.niv)
    gchi0_q_core_inv = deepcopy(gchi0_q_core).invert(False)
    out["chi0_inv"] = gchi0_q_core_inv.mat.copy()
    gchi0_q_core_sum = 1.0 / beta * gchi0_q_core.sum_over_all_vn(beta)

    keep = {}
    for ch, chan in (("dens", SpinChannel.DENS), ("magn", SpinChannel.MAGN)):
        gamma_r = LocalFourPoint(inp[f"gamma_{ch}"], chan, 1, 2, False, True)
        keep[ch] = {"gamma": gamma_r}
        # calculate_sigma_kernel_r_q (nonlocal_sde.py:257-336), both BSE variants
        if bse_variant == "v3":
            aux = nonlocal_sde.create_auxiliary_chi_r_q_sum_v3(gamma_r, gchi0_q_core_inv, u_loc, v_nonloc, dist)
        else:
            aux = nonlocal_sde.create_auxiliary_chi_r_q_sum_v1(gamma_r, gchi0_q_core_inv, u_loc, v_nonloc)
        out[f"chi_aux_sum_{ch}"] = aux.mat.copy()
        if variants:
            aux3 = nonlocal_sde.create_auxiliary_chi_r_q_sum_v3(gamma_r, gchi0_q_core_inv, u_loc, v_nonloc, dist)
            out[f"chi_aux_sum_v3_{ch}"] = aux3.mat.copy()
        vrg_q = nonlocal_sde.create_vrg_r_q(aux, gchi0_q_core_inv)
        out[f"vrg_{ch}"] = vrg_q.mat.copy()
        chi_phys = aux.sum_over_all_vn(beta)
        chi_phys = nonlocal_sde.create_generalized_chi_q_with_shell_correction(
            chi_phys, gchi0_q_full_sum, gchi0_q_core_sum, u_loc, v_nonloc
        )
        out[f"chi_phys_{ch}_before_lambda"] = chi_phys.mat.copy()
        if cfg.n_bands == 1:
            chi_phys, lam = lc.perform_single_lambda_correction(chi_phys, inp[f"chi_loc_sum_{ch}"])
            out[f"lambda_{ch}"] = np.float64(lam)
        out[f"chi_phys_{ch}"] = chi_phys.mat.copy()
        keep[ch]["vrg"] = deepcopy(vrg_q)
        keep[ch]["chi_phys"] = deepcopy(chi_phys)
        k_r = nonlocal_sde.calculate_kernel_r_q(vrg_q, chi_phys, v_nonloc, u_loc)
        out[f"kernel_{ch}"] = k_r.mat.copy()
        kernel += k_r if ch == "dens" else 3 * k_r

    out["kernel"] = kernel.mat.copy()
    # IBZ -> FBZ and the Sigma contraction through real space (nonlocal_sde.py:861, 874-878)
    kernel_full = deepcopy(kernel).map_to_full_bz(grid)
    kernel_full._nq = tuple(cfg.nk)
    sigma_r = nonlocal_sde.calculate_sigma_from_kernel_fft_cpu(dist, deepcopy(kernel_full), giwk)
    sigma = sigma_r.ifft().to_full_niv_range()
    out["sigma"] = sigma.compress_q_dimension().mat.copy()
    # direct Sigma variant (nonlocal_sde.py:430-469) on the full q list
    if variants:
        sig_direct = nonlocal_sde.calculate_sigma_from_kernel_cpu(deepcopy(kernel_full), giwk, grid.get_q_list())
        out["sigma_direct"] = sig_direct.compress_q_dimension().mat.copy()

    if name in ELIASHBERG_CONFIGS:
        out.update(run_reference_eliashberg(cfg, inp, giwk, u_loc, v_nonloc, gchi0_q_core_inv, keep, grid))

    save = {k: v for k, v in inp.items() if k not in ("config",)}
    save.update({f"ref_{k}": v for k, v in out.items()})
    save["config_name"] = np.array(name)
    return save


ELIASHBERG_CONFIGS = ("t4e", "t5e", "t3a")
AUTO_CONFIGS = ("t3a",)


def run_reference_eliashberg(cfg, inp, giwk, u_loc, v_nonloc, gchi0_q_core_inv, keep, grid) -> dict:
    """Full vertex, pp transform, pairing vertices and the Lanczos eigen-solve with the upstream functions
    (eliashberg_solver.py:175-204, 44-75, 620-628, 376-471), d-wave start, n_eig = 4, tol 1e-12."""
    config.eliashberg.save_fq = False
    config.eliashberg.construct_fq_cheap = False
    config.eliashberg.n_eig = 4
    config.eliashberg.epsilon = 1e-12
    config.eliashberg.symmetry = "d-wave"
    niv_pp = min(cfg.niw // 2, cfg.niv // 2)
    out = {"niv_pp": np.int64(niv_pp)}
    f_pp = {}
    for ch in ("dens", "magn"):
        mats = []
        for idx in range(grid.nk_irr):
            f = eliashberg_solver.create_full_vertex_q_r_v2(
                u_loc, v_nonloc, keep[ch]["gamma"], gchi0_q_core_inv, keep[ch]["vrg"], keep[ch]["chi_phys"], niv_pp, idx
            )
            mats.append(f.mat[0])
        f_pp[ch] = np.stack(mats)
        out[f"f_pp_{ch}"] = f_pp[ch]
    gam = {
        "sing": 0.5 * f_pp["dens"] - 1.5 * f_pp["magn"],
        "trip": 0.5 * f_pp["dens"] + 0.5 * f_pp["magn"],
    }
    chi0pp = BubbleGenerator.create_generalized_chi0_q_pp_w0(giwk, niv_pp, grid)
    out["chi0pp"] = chi0pp.mat.copy()
    for ch, chan in (("sing", SpinChannel.SING), ("trip", SpinChannel.TRIP)):
        out[f"gamma_pp_{ch}"] = gam[ch]
        gp = FourPoint(gam[ch], chan, tuple(cfg.nk), 0, 2, False, True, True, FrequencyNotation.PP)
        c0 = deepcopy(chi0pp)
        lambdas, gaps = eliashberg_solver.solve_eliashberg_lanczos(gp, c0, (0, 0))
        out[f"lambdas_{ch}"] = np.asarray(lambdas)
        out[f"gap_{ch}_0"] = gaps[0].mat.copy()
    return out


def upstream_fixtures() -> dict:
    e2e = os.path.join(UPSTREAM_DATA, "end_2_end")
    out = {}
    for f in ("g_dga", "gchi0_q_rank_0", "gchi0_q_inv_rank_0", "mu_history"):
        out[f] = np.load(os.path.join(e2e, f + ".npy"))
    for kind in ("sp", "spch"):
        d = os.path.join(UPSTREAM_DATA, "lambda_correction", kind)
        for f in sorted(os.listdir(d)):
            if f.endswith(".npy"):
                out[f"lambda_{kind}_{f[:-4]}"] = np.load(os.path.join(d, f))
    return out


def bse_kat() -> dict:
    """The upstream BSE known-answer input (tests/test_four_point.py:46-63, rng 1234) and its outputs."""
    rng = np.random.default_rng(1234)
    nq, o, niw, niv = (4, 4, 1), 2, 3, 3
    shape = (16, o, o, o, o, 2 * niw + 1, 2 * niv, 2 * niv)
    mat = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    beta = 11.0
    fp = FourPoint(mat, SpinChannel.MAGN, nq, 1, 2, True, True, True)
    v1 = deepcopy(fp).invert_and_sum_over_last_vn(beta).mat
    v2 = deepcopy(fp).invert_and_sum_over_last_vn_v2(beta).mat
    # the input is regenerated from default_rng(1234) by the tests; only the outputs are stored
    return {"beta": beta, "v1": v1, "v2": v2}


HF_CONFIGS = ("t1", "t2", "t3")


def hf_fixtures() -> dict:
    """nonlocal_sde.get_hartree_fock (nonlocal_sde.py:31-69) on the configurations' interactions and seeded
    occupations, with the full ordered q list of a single rank."""
    out = {}
    for name in HF_CONFIGS:
        cfg = synthetic.CONFIGS[name]
        inp = synthetic.make_inputs(cfg)
        _setup_config(cfg, inp)
        occ, occ_k = synthetic.make_occupations(cfg)
        config.sys.occ = occ
        config.sys.occ_k = occ_k
        u_loc = LocalInteraction(inp["u"])
        v_full = Interaction(inp["v_q_full"].reshape(*cfg.nk, *inp["v_q_full"].shape[1:]), SpinChannel.NONE,
                             tuple(cfg.nk))
        hartree, fock = nonlocal_sde.get_hartree_fock(u_loc, v_full, config.lattice.q_grid.get_q_list())
        out[f"{name}_u"] = inp["u"]
        out[f"{name}_v_q_full"] = inp["v_q_full"]
        out[f"{name}_nk"] = np.array(cfg.nk)
        out[f"{name}_occ"] = occ
        out[f"{name}_occ_k"] = occ_k
        out[f"{name}_hartree"] = hartree
        out[f"{name}_fock"] = fock
    return out


AT_SIZE_Q = {"c1": 45, "c2": 4, "c3": 2, "c4_bilayer": 2, "c4_single": 4}  # irreducible q whose X is stored
# bosonic indices of X stored where X of one q is large (3 orbitals: 81 x 41 x 80 complex128, 4.3 MB)
AT_SIZE_W = {"c3": (0, 1, 20, 40), "c4_bilayer": (0, 1, 15, 30)}
# through the upstream's q-by-q BSE where v1 would hold every (q, w) matrix at once: 153 x 41 x 720^2 complex128
# (52 GB) for the 3-orbital box, 325 x 31 x 240^2 (9.3 GB) for the bilayer
AT_SIZE_BSE = {"c3": "v3", "c4_bilayer": "v3"}
AT_SIZE_KEYS = ("sigma", "lambda_dens", "lambda_magn", "chi_aux_sum_dens", "chi_aux_sum_magn", "chi_phys_magn")


def input_digest(inp: dict) -> dict:
    """Sums of the seeded inputs, stored beside the at-size outputs so a test can see that it regenerated the
    same inputs (synthetic.make_inputs is deterministic; machines differ at most in the last bits)."""
    return {f"digest_{k}": np.sum(np.asarray(inp[k], dtype=np.complex128))
            for k in ("g_k", "gamma_dens", "gamma_magn", "f_dc", "u", "v_q_irr")}


def run_reference_at_size(name: str) -> dict:
    """The upstream pass at a benchmark configuration's own size (c1: 1 orbital 16x16, niv = niw = 20 with the
    spch lambda-correction; c2: 64x64, niv = niw = 60; c3: 3 orbitals 32x32, niv = niw = 40, N = 720, no
    lambda; the two requests of the batched pair, c4_bilayer: 2 orbitals 48x48, niv = niw = 30, N = 240, and
    c4_single: 1 orbital 32x32, niv = niw = 50, with lambda), in FP64.  Stored: Sigma on the irreducible k points, lambda_d and lambda_m (one orbital), X = sum_nu'
    chi* (at the bosonic indices AT_SIZE_W where given) and (c3, c4) chi_phys_magn for the first AT_SIZE_Q[name]
    irreducible q, and the input digest; the inputs themselves are regenerated from their seed by the tests."""
    full = run_reference_pass(name, variants=False, bse_variant=AT_SIZE_BSE.get(name, "v1"), keep_keys=AT_SIZE_KEYS)
    ref = {k[4:]: v for k, v in full.items() if k.startswith("ref_")}
    inp = synthetic.make_inputs(synthetic.CONFIGS[name])
    nq = AT_SIZE_Q[name]
    w_sel = AT_SIZE_W.get(name)
    pick = (lambda x: x[:nq]) if w_sel is None else (lambda x: x[:nq][..., list(w_sel), :])
    out = {
        "sigma_irr": ref["sigma"][inp["irrk_ind"]],
        "chi_aux_sum_dens_q": pick(ref["chi_aux_sum_dens"]),
        "chi_aux_sum_magn_q": pick(ref["chi_aux_sum_magn"]),
        "chi_phys_magn": ref["chi_phys_magn"] if name in ("c1", "c2") else ref["chi_phys_magn"][:nq],
        "n_q_stored": np.int64(nq),
    }
    if w_sel is not None:
        out["w_stored"] = np.asarray(w_sel, dtype=np.int64)
    for key in ("lambda_dens", "lambda_magn"):
        if key in ref:
            out[key] = ref[key]
    out.update(input_digest(inp))
    return {f"ref_{k}": v for k, v in out.items()}


def main():
    if "--at-size" in sys.argv:
        for name in sys.argv[sys.argv.index("--at-size") + 1:]:
            np.savez_compressed(os.path.join(HERE, f"{name}_size.npz"), **run_reference_at_size(name))
            print("wrote", f"{name}_size.npz")
        return
    if "--only-hf" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "hartree_fock.npz"), **hf_fixtures())
        print("wrote hartree_fock.npz")
        return
    if "--only" in sys.argv:
        for name in sys.argv[sys.argv.index("--only") + 1:]:
            data = run_reference_pass(name)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
            print("wrote", name, sorted(data.keys()))
        return
    np.savez_compressed(os.path.join(HERE, "hartree_fock.npz"), **hf_fixtures())
    for name in ("t1", "t1b", "t2", "t3") + ELIASHBERG_CONFIGS:
        data = run_reference_pass(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print("wrote", name, sorted(data.keys()))
    np.savez_compressed(os.path.join(HERE, "upstream_fixtures.npz"), **upstream_fixtures())
    np.savez_compressed(os.path.join(HERE, "bse_kat.npz"), **bse_kat())
    print("done")


if __name__ == "__main__":
    main()
