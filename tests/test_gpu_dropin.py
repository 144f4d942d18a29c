"""The upstream-signature drop-ins (dgamore_b200/dropin.py) against the upstream's own FP64 outputs.

Each test builds the arguments the upstream function receives -- duck-typed stand-ins for its FourPoint /
LocalFourPoint / Interaction / GreensFunction objects and its ``config`` -- from the committed golden fixtures
(tests/golden/make_golden.py ran the upstream to produce them), calls the drop-in with the upstream's argument
list, and compares the result, in the upstream layout, with the upstream's output at the FP64 drop-in bar of
1e-10 relative (the eigenvalues at 1e-9, as the Eliashberg tests).
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10
PASS_CONFIGS = ("t1", "t1b", "t2", "t3", "t4e", "t5e")
LAMBDA_CONFIGS = ("t1", "t1b", "t5e")


class NPoint:
    """Stand-in for an upstream n-point object: ``.mat``, a channel, the half/full bosonic-range flag and the
    layout methods the drop-ins call (here already in the layout the upstream would have converted to)."""

    def __init__(self, mat, channel=None, full_niw_range=False, num_vn_dimensions=1):
        self.mat = np.asarray(mat)
        self.channel = channel
        self.full_niw_range = full_niw_range
        self._num_vn_dimensions = num_vn_dimensions

    @property
    def num_vn_dimensions(self):  # the upstream keeps it in _num_vn_dimensions (local_n_point.py)
        return self._num_vn_dimensions


class FourPointFull(NPoint):
    """A FourPoint with two fermionic dimensions in the full bosonic range [q, o1..o4, w, nu, nu']."""

    def to_half_niw_range(self):
        if self.full_niw_range:
            niw = self.mat.shape[5] // 2
            self.mat = self.mat[..., niw:, :, :]
            self.full_niw_range = False
        return self

    def compress_q_dimension(self):
        return self

    def update_original_shape(self):
        self.updated = True


class Interaction:
    """LocalInteraction / Interaction: ``as_channel`` as dgamore/interaction.py:43-65, 160-182."""

    def __init__(self, mat, local: bool):
        self.mat = np.asarray(mat)
        self.local = local

    def as_channel(self, channel):
        from dgamore_b200.pipeline import u_channel, v_channel

        fn = u_channel if self.local else v_channel
        return NPoint(fn(self.mat, channel))


def _config(inp, **extra):
    from dgamore_b200 import dropin

    n = np.asarray(inp["u"]).shape[0]
    return dropin.namespace_config(inp["beta"], inp["nk"], inp["irrk_ind"], inp["irrk_inv"], inp["irrk_count"], n,
                                   inp["niv_core"], inp["niw"], **extra)


@pytest.fixture(autouse=True)
def fresh_state():
    from dgamore_b200 import dropin

    dropin._state["classes"] = {}
    dropin.set_precision("fp64")
    yield


@pytest.mark.parametrize("name", PASS_CONFIGS)
def test_bubble_fft_and_direct(name):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    cfg = _config(inp)
    dropin.use_config(cfg)
    giwk = NPoint(inp["g_k"])
    niv_full = inp["niv_core"] + inp["niv_shell"]
    got = dropin.create_generalized_chi0_q_fft_auto(None, giwk, inp["niw"], niv_full, cfg.lattice.k_grid,
                                                    inp["beta"], None)
    assert got.kind == "FourPoint" and got.kwargs["has_compressed_q_dimension"]
    assert rel_err(got.mat, ref["chi0"]) < TOL
    q_list = np.array(np.unravel_index(inp["irrk_ind"], inp["nk"])).T
    got = dropin.create_generalized_chi0_q_auto(None, giwk, inp["niw"], niv_full, q_list, cfg.lattice.q_grid,
                                                inp["beta"], None)
    assert rel_err(got.mat, ref["chi0_direct"]) < TOL


@pytest.mark.parametrize("name", ("t4e", "t5e"))
def test_chi0_pp_w0(name):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    cfg = _config(inp)
    dropin.use_config(cfg)
    got = dropin.create_generalized_chi0_q_pp_w0(NPoint(inp["g_k"]), int(ref["niv_pp"]), cfg.lattice.q_grid)
    assert rel_err(got.mat, ref["chi0pp"]) < TOL


def test_four_point_invert_and_sum_method():
    from dgamore_b200 import dropin

    kat = np.load(os.path.join(GOLDEN, "bse_kat.npz"))
    rng = np.random.default_rng(1234)
    shape = (16, 2, 2, 2, 2, 7, 6, 6)
    mat = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for method in ("v1", "v2"):
        fp = FourPointFull(mat, full_niw_range=True, num_vn_dimensions=2)
        out = dropin.invert_and_sum_over_last_vn(fp, float(kat["beta"]))
        assert out is fp and fp.num_vn_dimensions == 1 and fp.updated  # mutates and returns self
        assert rel_err(fp.mat, kat[method]) < TOL
    with pytest.raises(NotImplementedError):
        dropin.invert_and_sum_over_last_vn(FourPointFull(mat[..., 0], num_vn_dimensions=1), 1.0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", PASS_CONFIGS)
def test_auxiliary_chi_sum(name, precision):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    dropin.use_config(_config(inp))
    dropin.set_precision(precision)
    u_loc, v_nonloc = Interaction(inp["u"], True), Interaction(inp["v_q_irr"], False)
    for ch in ("dens", "magn"):
        gamma = NPoint(inp[f"gamma_{ch}"], channel=ch)
        for fn in (dropin.create_auxiliary_chi_r_q_sum_v1,
                   lambda *a: dropin.create_auxiliary_chi_r_q_sum_v3(*a, None)):
            got = fn(gamma, NPoint(ref["chi0_inv"]), u_loc, v_nonloc)
            assert got.channel == ch
            assert rel_err(got.mat, ref[f"chi_aux_sum_{ch}"]) < (TOL if precision == "fp64" else 1e-9), (ch, precision)


def _full_nu(half):
    niv = half.shape[-1]
    full = np.empty(half.shape[:-1] + (2 * niv,), dtype=half.dtype)
    full[..., niv:] = half
    full[..., :niv] = np.conj(half[..., ::-1])
    return full


@pytest.mark.parametrize("name", PASS_CONFIGS)
def test_sigma_from_kernel_fft_and_direct(name):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    cfg = _config(inp)
    dropin.use_config(cfg)
    nk = inp["nk"]
    kernel_full = NPoint(ref["kernel"][inp["irrk_inv"]])  # IBZ -> FBZ (plain gather for these symmetries)
    giwk = NPoint(inp["g_k"])
    sig_r = dropin.calculate_sigma_from_kernel_fft_auto(None, kernel_full, giwk)
    assert sig_r.kind == "SelfEnergy" and sig_r.kwargs == {"full_niv_range": False,
                                                          "has_compressed_q_dimension": True, "calc_smom": False}
    # the caller's ifft over the momentum axes and to_full_niv_range (nonlocal_sde.py:876-879)
    n = sig_r.mat.shape[1]
    k_space = np.fft.ifftn(sig_r.mat.reshape(*nk, n, n, -1), axes=(0, 1, 2)).reshape(sig_r.mat.shape)
    assert rel_err(_full_nu(k_space), ref["sigma"]) < TOL
    full_q = np.array(np.unravel_index(np.arange(int(np.prod(nk))), nk)).T
    sig_k = dropin.calculate_sigma_from_kernel_auto(None, kernel_full, giwk, full_q)
    assert rel_err(sig_k.mat, ref["sigma_direct"]) < TOL
    with pytest.raises(NotImplementedError):
        dropin.calculate_sigma_from_kernel_auto(None, kernel_full, giwk, full_q[::-1])


@pytest.mark.parametrize("name", LAMBDA_CONFIGS)
def test_lambda_correction(name):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    dropin.use_config(_config(inp))
    for ch in ("dens", "magn"):
        half = ref[f"chi_phys_{ch}_before_lambda"].reshape(len(inp["irrk_ind"]), -1)
        full = np.concatenate([np.conj(half[:, :0:-1]), half], axis=1)  # chi(-w) = conj chi(w)
        lam = dropin.find_lambda(full, inp[f"chi_loc_sum_{ch}"])
        assert abs(lam - float(ref[f"lambda_{ch}"])) < TOL * max(1.0, abs(float(ref[f"lambda_{ch}"])))
        chi = NPoint(full[:, None, None, None, None, :], full_niw_range=True)
        out, lam2 = dropin.perform_single_lambda_correction(chi, inp[f"chi_loc_sum_{ch}"])
        assert lam2 == lam
        assert rel_err(out.mat, ref[f"chi_phys_{ch}"]) < TOL


@pytest.mark.parametrize("name", ("t1", "t2", "t3"))
def test_hartree_fock(name):
    from dgamore_b200 import dropin

    d = np.load(os.path.join(GOLDEN, "hartree_fock.npz"))
    nk = tuple(int(x) for x in d[f"{name}_nk"])
    n = d[f"{name}_u"].shape[0]
    nk_tot = int(np.prod(nk))
    cfg = dropin.namespace_config(1.0, nk, np.arange(nk_tot), np.arange(nk_tot), np.ones(nk_tot), n,
                                  occ=d[f"{name}_occ"], occ_k=d[f"{name}_occ_k"])
    dropin.use_config(cfg)
    full_q = np.array(np.unravel_index(np.arange(nk_tot), nk)).T
    hartree, fock = dropin.get_hartree_fock(NPoint(d[f"{name}_u"]), NPoint(d[f"{name}_v_q_full"]), full_q)
    assert rel_err(hartree, d[f"{name}_hartree"]) < TOL
    assert rel_err(fock, d[f"{name}_fock"]) < TOL


@pytest.mark.parametrize("ch", ["sing", "trip"])
@pytest.mark.parametrize("name", ("t4e", "t5e"))
def test_eliashberg_lanczos(name, ch):
    from dgamore_b200 import dropin

    inp, ref = load_golden(name)
    dropin.use_config(_config(inp, n_eig=4, epsilon=1e-12, symmetry="d-wave"))
    lambdas, gaps = dropin.solve_eliashberg_lanczos(NPoint(ref[f"gamma_pp_{ch}"], channel=ch),
                                                    NPoint(ref["chi0pp"]), (0, 1))
    expect = ref[f"lambdas_{ch}"]
    assert np.max(np.abs(np.asarray(lambdas) - expect)) < 1e-9 * max(1.0, np.max(np.abs(expect)))
    n = np.asarray(inp["u"]).shape[0]
    assert len(gaps) == 4 and gaps[0].mat.shape == (*inp["nk"], n, n, 2 * int(ref["niv_pp"]))
