"""Self-consistency glue on the device against the upstream run in FP64 (tests/golden/glue.npz, made by
tests/golden/make_golden_glue.py from greens_function.py and self_energy.py).

Bounds: G(k, ν), the tail moments, the fillings and occupations to 1e-12 relative (occupations below 1e-12 are
zeroed by both sides, so they are compared with that absolute slack); μ from the secant search to 1e-9 (both
searches stop at steps below 1e-6 and run on fillings that agree to rounding).
"""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["g1", "g3"])
def case(request):
    d = np.load(os.path.join(GOLDEN, "glue.npz"))
    return {k[3:]: d[k] for k in d.files if k.startswith(request.param + "_")}


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.complex128), device="cuda")


def test_g_full(case):
    from dgamore_b200 import selfconsistency as sc

    g = sc.g_full(_dev(case["sigma"]), _dev(case["ek"]), float(case["mu0"]), float(case["beta"]))
    assert rel_err(g.cpu().numpy(), case["g_full"]) < 1e-12


def test_tail_moments(case):
    from dgamore_b200 import selfconsistency as sc

    m0, m1 = sc.fit_smom(_dev(case["sigma"]), float(case["beta"]))
    assert rel_err(m0, case["smom0"]) < 1e-12 and rel_err(m1, case["smom1"]) < 1e-12


def test_filling_and_mu(case):
    from dgamore_b200 import selfconsistency as sc

    sigma, ek, beta, mu0 = _dev(case["sigma"]), _dev(case["ek"]), float(case["beta"]), float(case["mu0"])
    smom0 = case["smom0"]
    fill = sc.total_fill(mu0, ek, sigma, beta, smom0)
    assert abs(fill - float(case["fill_mu0"])) < 1e-12 * abs(float(case["fill_mu0"]))
    mu = sc.update_mu(mu0, float(case["target"]), ek, sigma, beta, smom0)
    assert abs(mu - float(case["mu_new"])) < 1e-9


def test_occupations(case):
    from dgamore_b200 import selfconsistency as sc

    n_el, occ, occ_k = sc.fill_nonlocal(_dev(case["sigma"]), _dev(case["ek"]), float(case["mu0"]),
                                        float(case["beta"]), case["smom0"])
    assert abs(n_el - float(case["n_el"])) < 1e-12 * abs(float(case["n_el"]))
    assert np.max(np.abs(occ - case["occ"])) < 1e-12 * np.max(np.abs(case["occ"])) + 1e-12
    assert np.max(np.abs(occ_k - case["occ_k"])) < 1e-12 * np.max(np.abs(case["occ_k"])) + 1e-12
