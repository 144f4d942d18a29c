"""GPU parity of the Eliashberg stage against the upstream FP64 outputs (golden fixtures t4e, t5e).

Tolerances: pairing vertices and chi0pp 1e-10 relative; the gap-equation operator against the oracle's
restatement 1e-10; the four leading singlet/triplet eigenvalues 1e-9 relative to the upstream's ARPACK values
(both converged to 1e-12)."""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

ELI = ("t4e", "t5e", "t3a")  # t3a: auto-mode symmetries with per-k orbital rotations


@pytest.fixture(scope="module", params=ELI)
def solver(request):
    from dgamore_b200.eliashberg_solver import EliashbergSolver
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(request.param)
    lp = LadderPass(inp)
    lp.run()
    es = EliashbergSolver(lp)
    torch.cuda.synchronize()
    return request.param, inp, ref, es


def test_pairing_vertices(solver):
    name, inp, ref, es = solver
    assert es.P == int(ref["niv_pp"])
    assert int(es.vertex_status.abs().sum().item()) == 0
    for st, ch in ((0, "sing"), (1, "trip")):
        assert rel_err(es.pairing_vertex_ref_layout(st), ref[f"gamma_pp_{ch}"]) < 1e-10


def test_chi0pp(solver):
    name, inp, ref, es = solver
    n, P = es.lp.sh.n_orb, es.P
    got = es.chi0pp.cpu().numpy().reshape(-1, 2 * P, n, n, n, n).transpose(0, 2, 3, 4, 5, 1)  # k a b c d nu
    assert rel_err(got, ref["chi0pp"]) < 1e-12


@pytest.mark.parametrize("ch", ["sing", "trip"])
def test_gap_operator_matches_oracle(solver, ch):
    from oracle import ladder as L

    name, inp, ref, es = solver
    sh = es.lp.sh
    P = es.P
    st = 0 if ch == "sing" else 1
    chi0pp = L.chi0_pp_full_grid(inp["g_k"], P)
    rot = (inp["orbital_us"], inp["orbital_sigmas"], inp["orbital_conjs"]) if "orbital_us" in inp else None
    g_r, flip, sign = L.eliashberg_operator(ref[f"gamma_pp_{ch}"], inp["irrk_inv"], inp["nk"], chi0pp, sh.beta, ch,
                                            rot)
    rng = np.random.default_rng(5)
    gap = rng.standard_normal((*inp["nk"], sh.n_orb, sh.n_orb, 2 * P)) + 1j * rng.standard_normal(
        (*inp["nk"], sh.n_orb, sh.n_orb, 2 * P))
    expect = L.eliashberg_matvec(g_r, flip, chi0pp, gap, sh.beta, sign)
    got = es.matvec(ch, torch.as_tensor(gap.ravel(), device="cuda")).cpu().numpy().reshape(gap.shape)
    assert rel_err(got, expect) < 1e-10


@pytest.mark.parametrize("ch", ["sing", "trip"])
def test_leading_eigenvalues(solver, ch):
    from dgamore_b200.eliashberg_solver import initial_gap

    name, inp, ref, es = solver
    sh = es.lp.sh
    v0 = initial_gap(sh.nk, sh.n_orb, es.P, ch, "d-wave", inp["irrk_ind"], inp["irrk_inv"])
    if "orbital_us" in inp:  # auto mode: a random start vector (the symmetrised d-wave form assumes no rotations)
        v0 = np.random.default_rng(3).random(v0.shape) + 0j
    vals, vecs, status = es.eigs(ch, 4, 1e-12, v0.ravel())
    assert status == 0
    expect = ref[f"lambdas_{ch}"]
    assert np.max(np.abs(vals - expect)) < 1e-9 * max(1.0, np.max(np.abs(expect)))
    # the leading gap is an eigenvector of the device operator
    x = torch.as_tensor(vecs[0], device="cuda")
    r = es.matvec(ch, x).cpu().numpy() - vals[0] * vecs[0]
    assert np.linalg.norm(r) < 1e-8 * max(1.0, abs(vals[0])) * np.linalg.norm(vecs[0])


@pytest.mark.parametrize("ch", ["sing", "trip"])
def test_leading_eigenvalues_complex64_operator(solver, ch):
    """Gamma(R) stored in complex64 (FP64 products, vectors and normalisation): lambda_max and the next two
    eigenvalues within the stated bound of 1e-6 of the upstream's.  (Further down the spectrum, eigenvalues close
    in real part may come out in another order under the operator's complex64 rounding, so only the leading ones
    are compared.)"""
    from dgamore_b200.eliashberg_solver import EliashbergSolver, initial_gap

    name, inp, ref, es = solver
    sh = es.lp.sh
    es32 = EliashbergSolver(es.lp, precision="mixed")
    assert es32.mat.dtype == torch.complex64
    v0 = initial_gap(sh.nk, sh.n_orb, es32.P, ch, "d-wave", inp["irrk_ind"], inp["irrk_inv"])
    vals, vecs, status = es32.eigs(ch, 4, 1e-9, v0.ravel())
    assert status == 0
    expect = ref[f"lambdas_{ch}"]
    assert np.max(np.abs(vals[:3] - expect[:3])) < 1e-6


@pytest.mark.parametrize("name", ELI)
def test_vertex_fused_into_the_bse(name):
    """A pass built with eliashberg_pp writes the chi* part of the full vertex from its own LU factors; the
    Eliashberg stage then only adds the ladder term.  Pairing vertices equal the separate-kernel path (same
    factors, same order of operations) and the upstream's, the pass's Sigma is unchanged and the buffer is
    consumed by the stage."""
    from dgamore_b200.eliashberg_solver import EliashbergSolver, default_niv_pp
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(name)
    plain = LadderPass(inp)
    sig_plain = plain.run().cpu().numpy()
    es_plain = EliashbergSolver(plain)
    P = default_niv_pp(plain.sh.niw, plain.sh.niv)
    lp = LadderPass(inp, eliashberg_pp=P)
    sig = lp.run().cpu().numpy()
    assert np.array_equal(sig, sig_plain)
    assert lp.f_pp_ready
    es = EliashbergSolver(lp)
    torch.cuda.synchronize()
    assert es.fused and not lp.f_pp_ready
    assert int(es.vertex_status.abs().sum().item()) == 0
    for st, ch in ((0, "sing"), (1, "trip")):
        fused = es.pairing_vertex_ref_layout(st)
        assert rel_err(fused, es_plain.pairing_vertex_ref_layout(st)) < 1e-14
        assert rel_err(fused, ref[f"gamma_pp_{ch}"]) < 1e-10
