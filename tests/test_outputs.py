"""On-disk outputs in the upstream's conventions (dgamore_b200/outputs.py; CPU).

Self-contained checks of the half/full bosonic range, the unique output folder and the restart readers, plus the
same operations of the upstream itself where its sources are present (through the fixture harness): its
``LocalNPoint.to_full_niw_range`` / ``to_half_niw_range`` and ``nonlocal_sde.get_starting_sigma``.
"""

import os
import sys

import numpy as np
import pytest

from dgamore_b200 import outputs

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def _arr(shape, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_half_and_full_bosonic_range_round_trip():
    half = _arr((3, 2, 2, 2, 2, 5, 6))  # q a b c d w(>=0) nu
    full = outputs.full_niw(half, 1, 1)
    assert full.shape[-2] == 9
    np.testing.assert_array_equal(outputs.half_niw(full, 1, 1), half)
    # F(-w, nu) = conj F(w, -nu): the frequency axes flip together
    np.testing.assert_array_equal(full[..., 0, :], np.conj(half[..., 4, ::-1]))
    # no bosonic axis: unchanged
    sig = _arr((4, 2, 2, 8))
    assert outputs.half_niw(sig, 0, 1) is sig and outputs.full_niw(sig, 0, 1) is sig


def test_output_folder_name_and_uniqueness(tmp_path):
    name = outputs.output_dir_name(1024, 1024, 40, 40, 0)
    assert name == "LDGA_Nk1024_Nq1024_wc40_vc40_vs0"
    p = str(tmp_path / name)
    assert outputs.uniquify_path(p) == p
    os.makedirs(p)
    assert outputs.uniquify_path(p) == p + "_1"
    os.makedirs(p + "_1")
    assert outputs.uniquify_path(p) == p + "_2"


def test_restart_readers(tmp_path):
    out, prev = tmp_path / "out", tmp_path / "prev"
    out.mkdir()
    prev.mkdir()
    default = np.zeros((4, 1, 1, 6), dtype=np.complex128)
    assert outputs.get_starting_sigma(str(out), default)[1] == 0
    assert outputs.get_starting_sigma("", default)[0] is default
    sig = {i: _arr((4, 1, 1, 6), seed=i) for i in (1, 2, 3, 11)}
    outputs.save_sigma_iteration(sig[1], str(prev), 1)
    outputs.save_sigma_iteration(sig[2], str(prev), 2)
    outputs.save_sigma_iteration(sig[3], str(out), 3)
    outputs.save_sigma_iteration(sig[11], str(out), 11)
    np.save(out / "sigma_dga_iteration_x.npy", sig[1])  # not an iteration file
    got, it = outputs.get_starting_sigma(str(out), default)
    assert it == 11
    np.testing.assert_array_equal(got, sig[11])
    last = outputs.read_last_n_sigmas(3, str(out), str(prev))  # numeric order over both folders: 2, 3, 11
    for a, i in zip(last, (2, 3, 11)):
        np.testing.assert_array_equal(a, sig[i])


def _upstream():
    import _ref_harness as harness

    if not os.path.isdir(os.path.join(harness.REFERENCE_ROOT, "dgamore")):
        pytest.skip("the upstream sources are not present")
    harness.install()
    harness.patch_fp64()
    return harness


def test_bosonic_range_matches_the_upstream():
    _upstream()
    from dgamore.local_n_point import LocalNPoint

    half = _arr((2, 2, 2, 2, 4, 6), seed=3)  # a b c d w nu nu' -> here w, nu: num_wn 1, num_vn 1
    obj = LocalNPoint(half.copy(), 4, 1, 1, full_niw_range=False)
    np.testing.assert_array_equal(obj.to_full_niw_range().mat, outputs.full_niw(half, 1, 1))
    np.testing.assert_array_equal(obj.to_half_niw_range().mat, half)


def test_starting_sigma_matches_the_upstream(tmp_path):
    _upstream()
    from dgamore import config, nonlocal_sde
    from dgamore.self_energy import SelfEnergy

    nk = (2, 2, 1)
    config.lattice.nk = nk
    config.sys.beta = 12.5  # the upstream fits Σ's tail moments when it wraps the loaded array
    for i in (2, 7):
        outputs.save_sigma_iteration(_arr((4, 1, 1, 8), seed=i), str(tmp_path), i)
    default = SelfEnergy(_arr((4, 1, 1, 8), seed=9), nk, True, True, False, calc_smom=False)
    theirs, it_theirs = nonlocal_sde.get_starting_sigma(str(tmp_path), default)
    ours, it_ours = outputs.get_starting_sigma(str(tmp_path), default.mat)
    assert it_theirs == it_ours == 7
    np.testing.assert_array_equal(theirs.mat, ours)
    theirs_last = nonlocal_sde.read_last_n_sigmas_from_files(2, str(tmp_path), "")
    for a, b in zip(theirs_last, outputs.read_last_n_sigmas(2, str(tmp_path), "")):
        np.testing.assert_array_equal(a, b)
