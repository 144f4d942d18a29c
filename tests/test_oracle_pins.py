"""Pins the CPU oracle to the upstream code: its own fixtures and its outputs on seeded synthetic inputs."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CONFIGS, load_golden, rel_err
from oracle import ladder as L
from dgamore_b200.kgrid import KGrid

UPSTREAM = "tests/golden/upstream_fixtures.npz"


@pytest.fixture(scope="module")
def upstream():
    import os
    from conftest import REPO

    return dict(np.load(os.path.join(REPO, UPSTREAM)))


def test_bubble_matches_upstream_end_to_end_fixture(upstream):
    # tests/test_data/end_2_end: 2-orbital 4x4, beta=12.5, niw=20, niv_full=30 (core 20, shell 10)
    g = upstream["g_dga"].astype(np.complex128)
    grid = KGrid((4, 4, 1))
    chi0 = L.chi0_q_fft(g, 20, 30, grid.irrk_ind, 12.5)
    ref = upstream["gchi0_q_rank_0"]
    assert chi0.shape == ref.shape
    # the fixture was written in complex64: agreement to single precision
    assert np.max(np.abs(chi0 - ref)) < 2e-6
    inv = L.chi0_inv(L.cut_niv(chi0, 20, 1))
    assert rel_err(inv, upstream["gchi0_q_inv_rank_0"]) < 1e-6


@pytest.mark.parametrize("channel,lam_ref", [("dens", -37.450340), ("magn", 4.328781)])
def test_lambda_spch_matches_upstream_fixture(upstream, channel, lam_ref):
    # tests/test_lambda_correction.py:50-71 (complex64 inputs, as upstream computes them)
    grid = KGrid((4, 4, 1))
    chi = upstream[f"lambda_spch_chi_phys_q_{channel}_before_lambda"]
    loc = L.to_full_niw_range(upstream[f"lambda_spch_chi_{channel}_loc"], 1)
    corrected, lam = L.lambda_correct_single(chi, loc.sum() / 12.5, grid.irrk_count, 12.5, 16)
    assert np.allclose(lam, lam_ref)
    assert np.allclose(corrected, upstream[f"lambda_spch_chi_phys_q_{channel}"])


def test_lambda_sp_matches_upstream_fixture(upstream):
    # tests/test_lambda_correction.py:74-104
    grid = KGrid((4, 4, 1))
    chi_d = L.to_full_niw_range(upstream["lambda_sp_chi_phys_q_dens"], 1)
    loc_d = L.to_full_niw_range(upstream["lambda_sp_chi_dens_loc"], 1).sum()
    loc_m = L.to_full_niw_range(upstream["lambda_sp_chi_magn_loc"], 1).sum()
    target = loc_d + loc_m - 1.0 / 16 * (grid.irrk_count[:, None, None, None, None, None] * chi_d).sum()
    corrected, lam = L.lambda_correct_single(
        upstream["lambda_sp_chi_phys_q_magn_before_lambda"], target / 12.5, grid.irrk_count, 12.5, 16
    )
    assert np.allclose(lam, 4.281153)
    assert np.allclose(corrected, upstream["lambda_sp_chi_phys_q_magn"])


def test_bse_known_answer_matches_upstream():
    # tests/test_four_point.py:46-63 + 480-491: rng 1234, 2 orbitals, niw=niv=3, beta=11, MAGN, 16 q
    import os
    from conftest import REPO

    kat = np.load(os.path.join(REPO, "tests/golden/bse_kat.npz"))
    rng = np.random.default_rng(1234)
    shape = (16, 2, 2, 2, 2, 7, 6, 6)
    mat = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    half = mat[..., 3:, :, :]  # to_half_niw_range
    beta = float(kat["beta"])
    # the KAT matrix is A itself: feed it through bse_matrix-free inversion
    nb, nv = 2, 6
    n = nb * nb * nv
    out1 = np.empty(half.shape[:-1], dtype=np.complex128)
    for q in range(16):
        for w in range(4):
            a = half[q, ..., w, :, :].transpose(0, 1, 4, 3, 2, 5).reshape(n, n)
            x = np.linalg.inv(a).reshape(nb, nb, nv, nb, nb, nv)
            out1[q, ..., w, :] = x.sum(-1).transpose(0, 1, 4, 3, 2) / beta
    assert rel_err(out1, kat["v1"]) < 1e-12
    assert rel_err(kat["v2"], kat["v1"]) < 1e-10


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_oracle_pass_matches_upstream_fp64(name):
    inp, ref = load_golden(name)
    nb = inp["u"].shape[0]
    out = L.sde_pass(inp, do_lambda=(nb == 1))
    for key in (
        "chi0", "chi0_inv", "kernel_dc", "chi_aux_sum_dens", "chi_aux_sum_magn", "vrg_dens", "vrg_magn",
        "chi_phys_dens", "chi_phys_magn", "kernel_dens", "kernel_magn", "kernel", "sigma",
    ):
        assert rel_err(out[key], ref[key]) < 1e-12, key
    if nb == 1:
        assert abs(out["lambdas"]["dens"] - ref["lambda_dens"]) < 1e-10
        assert abs(out["lambdas"]["magn"] - ref["lambda_magn"]) < 1e-10


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_oracle_variants_agree(name):
    """v1 (inverse) and v3 (solve) BSE, FFT and direct bubble / Sigma agree (four_point.py:644-684)."""
    inp, ref = load_golden(name)
    assert rel_err(ref["chi_aux_sum_v3_dens"], ref["chi_aux_sum_dens"]) < 1e-12
    assert rel_err(ref["chi0_direct"], ref["chi0"]) < 1e-12
    assert rel_err(ref["sigma_direct"], ref["sigma"]) < 1e-12
    uv = L.u_as_channel(inp["u"], "magn")[None] + L.v_as_channel(inp["v_q_irr"], "magn")
    a = L.bse_sum(ref["chi0_inv"], inp["gamma_magn"], uv, inp["beta"])
    b = L.bse_sum_solve(ref["chi0_inv"], inp["gamma_magn"], uv, inp["beta"])
    assert rel_err(a, b) < 1e-12


def test_kgrid_irreducible_sizes():
    # 16^2 -> 45, 32^2 -> 153, 64^2 -> 561 under C4v (brillouin_zone.py:349-363)
    assert KGrid((16, 16, 1)).nk_irr == 45
    assert KGrid((32, 32, 1)).nk_irr == 153
    assert KGrid((64, 64, 1)).nk_irr == 561
    g = KGrid((48, 48, 1))
    assert g.irrk_count.sum() == 48 * 48


@pytest.mark.parametrize("name", ("t4e", "t5e", "t3a"))
def test_oracle_eliashberg_matches_upstream_fp64(name):
    """Full vertex in pp notation, chi0pp and the leading singlet/triplet eigenvalues (eliashberg_solver.py)."""
    inp, ref = load_golden(name)
    nb = inp["u"].shape[0]
    niv_pp = int(ref["niv_pp"])
    out = L.sde_pass(inp, do_lambda=(nb == 1))
    fpp = {}
    for ch in ("dens", "magn"):
        uv = L.u_as_channel(inp["u"], ch)[None] + L.v_as_channel(inp["v_q_irr"], ch)
        f = L.full_vertex_q(out["chi0_inv"], inp[f"gamma_{ch}"], uv, out[f"vrg_{ch}"], out[f"chi_phys_{ch}"],
                            inp["beta"], niv_pp)
        fpp[ch] = L.ph_to_pp_w0(f, inp["niw"], niv_pp)
        assert rel_err(fpp[ch], ref[f"f_pp_{ch}"]) < 1e-12
    gam = {"sing": 0.5 * fpp["dens"] - 1.5 * fpp["magn"], "trip": 0.5 * fpp["dens"] + 0.5 * fpp["magn"]}
    chi0pp = L.chi0_pp_full_grid(inp["g_k"], niv_pp)
    assert rel_err(chi0pp.reshape(-1, *chi0pp.shape[3:]), ref["chi0pp"]) < 1e-14
    for ch in ("sing", "trip"):
        assert rel_err(gam[ch], ref[f"gamma_pp_{ch}"]) < 1e-12
        v0 = L.symmetrise_gap(L.d_wave_gap(inp["nk"], nb, niv_pp, ch), inp["irrk_ind"], inp["irrk_inv"])
        rot = (inp["orbital_us"], inp["orbital_sigmas"], inp["orbital_conjs"]) if "orbital_us" in inp else None
        if rot is not None:  # the upstream's auto-mode start vector is not the symmetrised d-wave form
            v0 = np.random.default_rng(3).random(v0.shape) + 0j
        vals, _ = L.eliashberg_eigs(gam[ch], inp["irrk_inv"], inp["nk"], chi0pp, inp["beta"], ch, v0, 4, 1e-12,
                                    rotations=rot)
        assert np.max(np.abs(vals - ref[f"lambdas_{ch}"])) < 1e-9 * max(1.0, np.max(np.abs(vals)))


@pytest.mark.parametrize("name", ("t1", "t2", "t3"))
def test_hartree_fock_oracle_matches_upstream(name):
    """nonlocal_sde.get_hartree_fock run here (tests/golden/make_golden.py) vs the oracle restatement."""
    d = np.load(os.path.join(GOLDEN, "hartree_fock.npz"))
    nk = tuple(int(x) for x in d[f"{name}_nk"])
    v = d[f"{name}_v_q_full"].reshape(*nk, *d[f"{name}_v_q_full"].shape[1:])
    h, f = L.hartree_fock(d[f"{name}_u"], v, d[f"{name}_occ"], d[f"{name}_occ_k"])
    assert rel_err(h, d[f"{name}_hartree"]) < 1e-14
    assert rel_err(f, d[f"{name}_fock"]) < 1e-14
