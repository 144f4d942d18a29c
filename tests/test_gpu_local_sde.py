"""Device local Schwinger-Dyson equation (dgamore_b200/local_sde.py) against the upstream run and the oracle.

* the four golden cases of tests/golden/local_sde.npz (upstream ``perform_local_schwinger_dyson`` in FP64): all 11
  results to 1e-10 relative, with G2 given in the full and in the half w range;
* the drop-in ``dropin.perform_local_schwinger_dyson`` with a namespace configuration;
* failure paths: an exactly singular G2 raises numpy.linalg.LinAlgError as np.linalg.inv does, a NaN in G2 reaches
  the results and sets DGA_ITEM_NONFINITE without an exception;
* at size: the 3-orbital configuration's box (niv_core = 40, N = 720) on a reduced bosonic range against the
  oracle to 1e-10, and the full box (niw_core = niv_core = 40) through size-independent properties: the vertex
  the inputs were made from comes back (Gamma_r = Gamma_model) and F satisfies F (1 + chi0 Gamma_u / beta^2) =
  Gamma_u, checked with torch matrix products;
* the hand-off to the nonlocal pass on the device: Sigma equal to the pass fed host copies, and to the oracle.
"""

import dataclasses
import types

import numpy as np
import pytest
import torch

from conftest import rel_err
from test_local_sde_oracle import CASES, RESULTS, inputs, load

pytestmark = pytest.mark.gpu


def run_device(*args):
    from dgamore_b200.local_sde import LocalSde

    return LocalSde(*args).run()


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("w_range", ["full", "half"])
def test_local_sde_matches_upstream(case, w_range):
    d = load(case)
    args = list(inputs(d))
    if w_range == "half":
        args[1], args[2] = d["g2_dens_half"], d["g2_magn_half"]
    res = run_device(*args).results()
    for name, r in zip(RESULTS, res):
        assert r.shape == d[name].shape, name
        assert rel_err(r, d[name]) < 1e-10, name


def test_dropin_local_sde_with_namespace_config():
    from dgamore_b200 import dropin

    d = load("l3s")
    g, g2d, g2m, u, beta, niw, niv, sh, occ = inputs(d)
    cfg = types.SimpleNamespace(
        sys=types.SimpleNamespace(beta=beta, occ_dmft=occ),
        box=types.SimpleNamespace(niw_core=niw, niv_core=niv, niv_shell=sh),
        dmft=types.SimpleNamespace(symmetrize_orbitals=[]),
        eliashberg=types.SimpleNamespace(perform_eliashberg=False),
    )
    dropin.use_config(cfg)
    obj = lambda m: types.SimpleNamespace(mat=m)  # noqa: E731
    res = dropin.perform_local_schwinger_dyson(obj(g), obj(g2d), obj(g2m), obj(u))
    assert len(res) == 11
    for name, r in zip(RESULTS, res):
        assert rel_err(r.mat, d[name]) < 1e-10, name
    assert res[0].args[:4] == ("dens", 1, 2, False) and res[2].args[:4] == ("dens", 1, 0, False)
    cfg.dmft.symmetrize_orbitals = [1, 2]
    with pytest.raises(NotImplementedError):
        dropin.perform_local_schwinger_dyson(obj(g), obj(g2d), obj(g2m), obj(u))


def test_singular_g2_raises_linalg_error():
    d = load("l2")
    args = list(inputs(d))
    args[2] = np.zeros_like(args[2])  # magnetic chi = 0: an exact zero pivot
    sde = run_device(*args)
    with pytest.raises(np.linalg.LinAlgError):
        sde.results()


def test_nan_in_g2_is_flagged_not_raised():
    d = load("l1")
    args = list(inputs(d))
    g2d = args[1].copy()
    g2d[0, 0, 0, 0, g2d.shape[4] // 2, 3, 5] = np.nan
    args[1] = g2d
    sde = run_device(*args)
    torch.cuda.synchronize()
    assert int(sde.lu_status[0].item()) & 2  # DGA_ITEM_NONFINITE on the density channel's w = 0 inverse
    res = sde.results()
    assert np.isnan(res[0]).any()
    assert np.isfinite(res[1]).all()  # the magnetic vertex does not depend on G2_dens


def _model_inputs(name: str, niw: int, niv: int, niv_shell: int, seed_offset: int = 0):
    """Inputs of the local SDE made from the synthetic model vertex (tests/golden/make_golden_local.py's
    construction), the dense inverses by torch on the GPU."""
    from dgamore_b200 import synthetic
    from dgamore_b200.kgrid import KGrid
    from oracle import local_sde as osde

    cfg = dataclasses.replace(synthetic.CONFIGS[name], nk=(8, 8, 1), niw=niw, niv=niv, niv_shell=niv_shell)
    rng = np.random.default_rng(cfg.seed + 303 + seed_offset)
    grid = KGrid(cfg.nk, cfg.symmetries)
    ek = synthetic.dispersion(cfg, grid)
    mu = synthetic.find_mu(cfg, ek)
    niv_g = niv + niv_shell + niw + 4
    g = synthetic.g_lattice(ek, synthetic.hubbard_i_sigma(cfg, mu, niv_g), mu, cfg.beta).mean(axis=(0, 1, 2))
    u = synthetic.kanamori_u(cfg)
    beta = cfg.beta
    chi0h = osde.half_niw(osde.local_bubble(g, niw, niv + niv_shell, beta), 2)
    g2s, gammas = [], []
    for ch in ("dens", "magn"):
        u_r = osde.u_as_channel(u, ch)
        gamma = synthetic.gamma_model(cfg, u, ch, rng, niv)
        # chi~_core^-1 per w (dense only through the rank-n^2 U term), then chi = inv(chi~_core^-1 + (Gamma-U)/beta^2)
        c0 = osde.extend_diag(osde.inv_diag(chi0h))
        dense = c0 + u_r[..., None, None, None] / beta**2
        t = torch.from_numpy(osde.to_compound(dense)).cuda()
        s = niv_shell
        nvf = 2 * (niv + niv_shell)
        n2 = u.shape[0] ** 2
        idx = torch.tensor([p * nvf + s + v for p in range(n2) for v in range(2 * niv)], device="cuda")
        tilde = torch.linalg.inv(torch.linalg.inv(t)[:, idx][:, :, idx])
        a = tilde + torch.from_numpy(osde.to_compound((gamma - u_r[..., None, None, None]) / beta**2)).cuda()
        chi = osde.from_compound(torch.linalg.inv(a).cpu().numpy(), u.shape[0], 2 * niv)
        g2 = chi / beta
        if ch == "dens":
            gs = g[..., g.shape[-1] // 2 - niv : g.shape[-1] // 2 + niv]
            g2[:, :, :, :, 0] += 2.0 * gs[:, :, None, None, :, None] * gs[None, None, :, :, None, :]
        g2s.append(osde.full_niw(g2, 3))  # the full w range, as the upstream reads G2
        gammas.append(gamma)
    occ = synthetic.make_occupations(cfg)[0]
    return (g, g2s[0], g2s[1], u, beta, niw, niv, niv_shell, occ), gammas


def test_local_sde_at_the_t2g_box_matches_the_oracle():
    from oracle import local_sde as osde

    args, _ = _model_inputs("c3", 4, 40, 0)
    res = run_device(*args).results()
    ref = osde.perform_local_schwinger_dyson(*args)
    for name, r, o in zip(RESULTS, res, ref):
        assert rel_err(r, o) < 1e-10, name


@pytest.mark.parametrize("name,niw,niv,shell", [("c3", 40, 40, 0), ("c1", 20, 20, 10)])
def test_local_sde_full_box_properties(name, niw, niv, shell):
    args, gammas = _model_inputs(name, niw, niv, shell)
    sde = run_device(*args)
    sde.check()
    beta = args[4]
    for ch in (0, 1):
        assert rel_err(sde.gamma(ch).cpu().numpy(), gammas[ch]) < 1e-9, ch
    # F (1 + chi0 Gamma_u / beta^2) = Gamma_u on every w, in compound form
    n2, nvf, W = sde.n2, sde.nvf, sde.W
    Nf = n2 * nvf
    from oracle import local_sde as osde

    u_np = args[3]
    for ch, cname in ((0, "dens"), (1, "magn")):
        f = torch.from_numpy(osde.to_compound(sde.f(ch).cpu().numpy())).cuda()
        gu = torch.from_numpy(osde.to_compound(osde.pad_with_u(sde.gamma(ch).cpu().numpy(),
                                                               osde.u_as_channel(u_np, cname), niv + shell))).cuda()
        chi0 = sde.bubble().cpu().numpy()
        c0 = torch.from_numpy(osde.to_compound(osde.extend_diag(chi0))).cuda()
        eye = torch.eye(Nf, dtype=torch.complex128, device="cuda")
        lhs = f @ (eye + c0 @ gu / beta**2)
        assert rel_err(lhs.cpu().numpy(), gu.cpu().numpy()) < 1e-10, ch
        assert f.shape == (W, Nf, Nf)


def test_local_results_feed_the_nonlocal_pass_on_the_device():
    """The local equation's vertices reach the nonlocal pass on the device (no .npy hand-off): the pass built from
    LocalSde.nonlocal_inputs gives the same Sigma as the pass built from host copies of the same results, and
    both match the oracle's pass (pinned to the upstream) on those inputs."""
    from dgamore_b200 import synthetic
    from dgamore_b200.local_sde import LocalSde
    from dgamore_b200.pipeline import LadderPass
    from oracle import ladder, local_sde as osde

    cfg = synthetic.CONFIGS["t1"]  # 1 orbital, 4x4, niw = niv = 4, niv_shell = 2, lambda-corrected
    base = synthetic.make_inputs(cfg)
    g_loc = np.asarray(base["g_k"]).mean(axis=(0, 1, 2))
    beta, niw, niv, sh = base["beta"], base["niw"], base["niv_core"], base["niv_shell"]
    u = np.asarray(base["u"])
    chi0h = osde.half_niw(osde.local_bubble(g_loc, niw, niv + sh, beta), 2)
    g2 = []
    for ch in ("dens", "magn"):
        u_r = osde.u_as_channel(u, ch)
        a = osde.chi_tilde_core_inv(chi0h, u_r, beta, niv) + (base[f"gamma_{ch}"] - u_r[..., None, None, None]) / beta**2
        x = osde.inv_dense(a) / beta
        if ch == "dens":
            gs = g_loc[..., g_loc.shape[-1] // 2 - niv : g_loc.shape[-1] // 2 + niv]
            x[:, :, :, :, 0] += 2.0 * gs[:, :, None, None, :, None] * gs[None, None, :, :, None, :]
        g2.append(osde.full_niw(x, 3))
    sde = LocalSde(g_loc, g2[0], g2[1], u, beta, niw, niv, sh, synthetic.make_occupations(cfg)[0]).run()
    dev_inp = sde.nonlocal_inputs(base)
    assert isinstance(dev_inp["gamma_dens"], torch.Tensor) and dev_inp["gamma_dens"].is_cuda
    host_inp = {k: (v.cpu().numpy() if isinstance(v, torch.Tensor) else v) for k, v in dev_inp.items()}
    sig_dev = LadderPass(dev_inp).run().cpu().numpy()
    sig_host = LadderPass(host_inp).run().cpu().numpy()
    assert np.array_equal(sig_dev, sig_host)
    ref = ladder.sde_pass(host_inp)
    assert rel_err(sig_dev, ref["sigma"]) < 1e-10
    assert rel_err(host_inp["gamma_magn"], base["gamma_magn"]) < 1e-10  # the round trip through the local ladder


def test_whole_chain_on_the_device():
    """Local SDE -> nonlocal pass (its vertices handed over on the device) with the Eliashberg vertex fused into the
    FP64 BSE -> leading pairing eigenvalues, equal to the same chain with the separate vertex kernel."""
    from dgamore_b200 import synthetic
    from dgamore_b200.eliashberg_solver import EliashbergSolver, default_niv_pp
    from dgamore_b200.local_sde import LocalSde
    from dgamore_b200.pipeline import LadderPass

    cfg = synthetic.CONFIGS["t4e"]  # 2 orbitals, 6x6, niw = niv = 6
    base = synthetic.make_inputs(cfg)
    lsi, _ = synthetic.local_sde_inputs(cfg)
    sde = LocalSde(*lsi).run()
    inputs = sde.nonlocal_inputs(base)
    P = default_niv_pp(cfg.niw, cfg.niv)
    lp = LadderPass(inputs, eliashberg_pp=P)
    sig = lp.run()
    es = EliashbergSolver(lp, P)
    assert es.fused
    ls, lt, _, _ = es.solve(n_eig=2, tol=1e-10)
    plain = LadderPass({k: (v.clone() if isinstance(v, torch.Tensor) else v) for k, v in inputs.items()})
    sig_plain = plain.run()
    assert torch.equal(sig, sig_plain)
    es_plain = EliashbergSolver(plain, P)
    assert not es_plain.fused
    ls_p, lt_p, _, _ = es_plain.solve(n_eig=2, tol=1e-10)
    assert np.allclose(ls, ls_p, rtol=1e-9) and np.allclose(lt, lt_p, rtol=1e-9)
    assert np.isfinite(ls).all() and np.isfinite(lt).all()
