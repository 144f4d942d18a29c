"""Seeded synthetic inputs for one nonlocal ladder-DGA pass.

The upstream code reads its local vertices from a DMFT impurity solver (w2dynamics HDF5), which has no public
stand-in here.  This module builds inputs with the same shapes, sizes, symmetries and value ranges from a
model, deterministically from a seed:

* dispersion: square lattice t, t', t'' per orbital (``kinetic_one_band_2d_t_tp_tpp``,
  dgamore/hamiltonian.py:188-209), optional on-site inter-orbital hopping (bilayer t_perp);
* local interaction: Kanamori U, J, U' = U - 2J (dgamore/hamiltonian.py:128-186), single band U_0000 = U;
* optional nearest-neighbour density-density V(q) (exercises the V^q terms; zero in the benchmark configs);
* local self-energy: Hubbard-I form, chemical potential by bisection on the filling;
* irreducible local vertex Gamma_r(w, nu, nu') = U_r + a smooth frequency structure built from U_r U_r in the
  compound orbital basis + a seeded complex Gaussian perturbation of relative size 1e-3, symmetrised under
  (nu <-> nu', orbitals abcd -> cdab) as ``symmetrize_v_vp`` (dgamore/local_four_point.py:588-597) and under the
  w=0 conjugation rule F(-w) = conj(flip F(w)) (dgamore/local_n_point.py:218-220);
* local susceptibility in the same asymptotic form the nonlocal pass uses: chi*_loc = (chi0_loc^-1 +
  (Gamma_r - U_r)/beta^2)^-1 and chi_r,loc(w) = [(sum chi*_loc / beta^2)^-1 + U_r]^-1 (dgamore/nonlocal_sde.py:
  85-96 and 167-182 without momentum), giving the lambda-correction targets sum_w chi_r,loc / beta, and the local
  vertex F_magn = beta^2 (chi0^-1 - chi0^-1 chi*_m chi0^-1) used by the double-counting kernel.

Array layouts are the upstream ones (see ``oracle/ladder.py``); everything is complex128.
"""

from __future__ import annotations

from dataclasses import dataclass, field, asdict

import numpy as np

from .kgrid import KGrid, SQUARE_2D


@dataclass
class DgaConfig:
    """One nonlocal DGA parameter point."""

    name: str
    n_bands: int
    nk: tuple
    beta: float
    niw: int
    niv: int
    niv_shell: int = 0
    u: float = 8.0
    j: float = 0.0
    t: tuple = (1.0,)  # nearest-neighbour hopping per orbital (isotropic)
    t_aniso: tuple = ()  # per-orbital (t_x, t_y) nearest-neighbour hoppings; when given, they replace t
    tp: float = 0.0
    tpp: float = 0.0
    t_perp: float = 0.0  # on-site hopping between orbitals 0 and 1 (bilayer)
    v_nn: float = 0.0  # nearest-neighbour density-density interaction
    n: float = 0.85
    seed: int = 0
    symmetries: tuple = SQUARE_2D

    @property
    def niv_full(self) -> int:
        return self.niv + self.niv_shell

    @property
    def niv_g(self) -> int:
        """Fermionic box of G(k): enough for the bubble (niv_full + niw) and the Sigma shift (niw + niv)."""
        return self.niv_full + self.niw + 10

    @property
    def n_compound(self) -> int:
        return self.n_bands**2 * 2 * self.niv

    def to_dict(self) -> dict:
        return asdict(self)


CONFIGS = {
    # plain method, CPU-runnable: 1-orbital square lattice Hubbard
    "c1": DgaConfig("c1", 1, (16, 16, 1), 12.5, 20, 20, 0, u=8.0, t=(1.0,), tp=-0.25, n=0.85, seed=1),
    # FP64 drop-in at scale
    "c2": DgaConfig("c2", 1, (64, 64, 1), 12.5, 60, 60, 0, u=8.0, t=(1.0,), tp=-0.25, n=0.85, seed=2),
    # 3-orbital t2g square lattice, Kanamori U=2.3 J=0.4, per-orbital isotropic hoppings (0.5, 0.5, 0.1)
    "c3": DgaConfig("c3", 3, (32, 32, 1), 20.0, 40, 40, 0, u=2.3, j=0.4, t=(0.5, 0.5, 0.1), n=1.0, seed=3),
    # bilayer 2-orbital Hubbard and a 1-orbital partner
    "c4_bilayer": DgaConfig("c4_bilayer", 2, (48, 48, 1), 15.0, 30, 30, 0, u=6.0, t=(1.0, 1.0), t_perp=0.8, n=1.8, seed=4),
    "c4_single": DgaConfig("c4_single", 1, (32, 32, 1), 12.5, 50, 50, 0, u=8.0, t=(1.0,), tp=-0.25, n=0.85, seed=5),
    # small cases for parity tests
    "t1": DgaConfig("t1", 1, (4, 4, 1), 12.5, 4, 4, 2, u=5.0, t=(1.0,), tp=-0.25, v_nn=0.3, n=0.85, seed=11),
    "t1b": DgaConfig("t1b", 1, (8, 8, 1), 10.0, 6, 6, 0, u=4.0, t=(1.0,), tp=-0.2, n=0.9, seed=12),
    "t2": DgaConfig("t2", 2, (4, 4, 1), 15.0, 2, 3, 1, u=6.0, t=(1.0, 1.0), t_perp=0.8, v_nn=0.2, n=1.8, seed=13),
    "t3": DgaConfig("t3", 3, (4, 4, 1), 20.0, 2, 2, 0, u=2.3, j=0.4, t=(0.5, 0.5, 0.1), n=1.0, seed=14),
    # Eliashberg parity cases (niv_pp = min(niw, niv) // 2 = 3)
    "t4e": DgaConfig("t4e", 2, (6, 6, 1), 15.0, 6, 6, 0, u=6.0, t=(1.0, 1.0), t_perp=0.8, n=1.8, seed=15),
    "t5e": DgaConfig("t5e", 1, (8, 8, 1), 10.0, 6, 6, 0, u=4.0, t=(1.0,), tp=-0.2, n=0.9, seed=16),
    # t2g with the anisotropic d_xz / d_yz hoppings that the square lattice's x <-> y operations exchange: the
    # irreducible wedge and the per-k orbital rotations come from the upstream's symmetry discovery (auto mode)
    "t3a": DgaConfig("t3a", 3, (4, 4, 1), 20.0, 2, 2, 0, u=2.3, j=0.4, t_aniso=((0.5, 0.5), (0.5, 0.1), (0.1, 0.5)),
                     n=1.0, seed=17, symmetries=()),
}


# ----------------------------------------------------------------------------------------------
# model pieces
# ----------------------------------------------------------------------------------------------


def dispersion(cfg: DgaConfig, grid: KGrid) -> np.ndarray:
    """e_k [kx,ky,kz,n,n] for square-lattice hoppings per orbital (isotropic t, or (t_x, t_y) from t_aniso) plus
    an on-site t_perp."""
    kx, ky = np.meshgrid(grid.kx, grid.ky, indexing="ij")
    nb = cfg.n_bands
    ek = np.zeros((*grid.nk, nb, nb), dtype=np.complex128)
    for a in range(nb):
        t = cfg.t[a] if a < len(cfg.t) else cfg.t[-1]
        if cfg.t_aniso:
            tx, ty = cfg.t_aniso[a]
            nn = -2 * (tx * np.cos(kx) + ty * np.cos(ky))
        else:
            nn = -2 * t * (np.cos(kx) + np.cos(ky))
        e = (
            nn
            - 4 * cfg.tp * np.cos(kx) * np.cos(ky)
            - 2 * cfg.tpp * (np.cos(2 * kx) + np.cos(2 * ky))
        )
        ek[..., a, a] = e[..., None]
    if nb >= 2 and cfg.t_perp != 0.0:
        ek[..., 0, 1] = -cfg.t_perp
        ek[..., 1, 0] = -cfg.t_perp
    return ek


def kanamori_u(cfg: DgaConfig) -> np.ndarray:
    """U_abcd with U_llll = U, U_lmml = U_llmm = J, U_lmlm = U - 2J (hamiltonian.py:128-186)."""
    nb = cfg.n_bands
    up = cfg.u - 2 * cfg.j
    u = np.zeros((nb,) * 4, dtype=np.complex128)
    for a in range(nb):
        for b in range(nb):
            for c in range(nb):
                for d in range(nb):
                    if a == b == c == d:
                        u[a, b, c, d] = cfg.u
                    elif (a == d and b == c) or (a == b and c == d):
                        u[a, b, c, d] = cfg.j
                    elif a == c and b == d:
                        u[a, b, c, d] = up
    return u


def nonlocal_v(cfg: DgaConfig, grid: KGrid) -> np.ndarray:
    """V^q_abcd [Nk,n,n,n,n]: density-density NN interaction 2 V (cos qx + cos qy) on U_aabb-type entries."""
    nb = cfg.n_bands
    qx, qy = np.meshgrid(grid.kx, grid.ky, indexing="ij")
    vq = (2 * cfg.v_nn * (np.cos(qx) + np.cos(qy)))[..., None].repeat(grid.nk[2], axis=2).reshape(-1)
    v = np.zeros((grid.nk_tot,) + (nb,) * 4, dtype=np.complex128)
    for a in range(nb):
        for c in range(nb):
            v[:, a, a, c, c] = vq
    return v


def hubbard_i_sigma(cfg: DgaConfig, mu: float, niv: int) -> np.ndarray:
    """Local Hubbard-I self-energy [n,n,2niv]: U n_s + U^2 n_s (1-n_s) / (i nu + mu - U (1 - n_s))."""
    nb = cfg.n_bands
    ns = cfg.n / (2 * nb)
    iv = 1j * np.pi / cfg.beta * (2 * np.arange(-niv, niv) + 1)
    u_eff = cfg.u
    s = u_eff * ns + u_eff**2 * ns * (1 - ns) / (iv + mu - u_eff * (1 - ns))
    sig = np.zeros((nb, nb, 2 * niv), dtype=np.complex128)
    for a in range(nb):
        sig[a, a] = s
    return sig


def g_lattice(ek: np.ndarray, sigma: np.ndarray, mu: float, beta: float) -> np.ndarray:
    """G(k,nu) [kx,ky,kz,n,n,2niv] = [i nu + mu - e_k - Sigma(nu)]^-1 (greens_function.py:125-142)."""
    nb = ek.shape[-1]
    niv = sigma.shape[-1] // 2
    iv = 1j * np.pi / beta * (2 * np.arange(-niv, niv) + 1)
    eye = np.eye(nb)
    mat = (iv[:, None, None] + mu) * eye[None] - ek[..., None, :, :] - np.moveaxis(sigma, -1, 0)[None, None, None]
    g = np.linalg.inv(mat)  # [kx,ky,kz,nu,a,b]
    return np.moveaxis(g, 3, -1)


def filling(ek: np.ndarray, sigma_fn, mu: float, beta: float, niv: int = 400) -> float:
    """Total filling 2 * sum_a n_aa from G(k,nu) with a 1/2 + (1/beta) sum Re G estimate."""
    sig = sigma_fn(mu, niv)
    g = g_lattice(ek, sig, mu, beta)
    gloc = g.mean(axis=(0, 1, 2))
    nb = ek.shape[-1]
    occ = 0.5 + np.sum(np.diagonal(gloc, axis1=0, axis2=1).real, axis=0) / beta
    return float(2 * np.sum(occ)) if nb else 0.0


def find_mu(cfg: DgaConfig, ek: np.ndarray) -> float:
    """Bisection of the filling in mu."""
    lo, hi = -4 * cfg.u - 10, 4 * cfg.u + 10
    fn = lambda m, nv: hubbard_i_sigma(cfg, m, nv)
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        if filling(ek, fn, mid, cfg.beta, 64) < cfg.n:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


# ----------------------------------------------------------------------------------------------
# local vertex model
# ----------------------------------------------------------------------------------------------


def _to_compound_orb(x: np.ndarray) -> np.ndarray:
    """[a,b,c,d,...] -> [(a,b),(d,c),...] matrices."""
    nb = x.shape[0]
    rest = x.shape[4:]
    return np.swapaxes(x, 2, 3).reshape(nb * nb, nb * nb, *rest)


def _from_compound_orb(m: np.ndarray, nb: int) -> np.ndarray:
    rest = m.shape[2:]
    return np.swapaxes(m.reshape(nb, nb, nb, nb, *rest), 2, 3)


def u_channel(u: np.ndarray, channel: str) -> np.ndarray:
    """Channel combination of U (interaction.py:43-65)."""
    u_adcb = np.einsum("abcd->adcb", u)
    return 2 * u - u_adcb if channel == "dens" else -u_adcb


def gamma_model(cfg: DgaConfig, u: np.ndarray, channel: str, rng: np.random.Generator, niv: int) -> np.ndarray:
    """Gamma_r [a,b,c,d,niw+1,2niv,2niv] (see module docstring)."""
    nb, beta, niw = cfg.n_bands, cfg.beta, cfg.niw
    u_r = u_channel(u, channel)
    m = _to_compound_orb(u_r)
    m2 = m @ m
    scale = max(abs(cfg.u), 1e-12)
    nu = np.pi / beta * (2 * np.arange(-niv, niv) + 1)
    om = 2 * np.pi / beta * np.arange(0, niw + 1)
    d1 = (nu[None, :, None] - nu[None, None, :]) / scale
    d2 = (nu[None, :, None] + nu[None, None, :] + om[:, None, None]) / scale
    w = 1.0 / (1.0 + d1**2) + 0.5 / (1.0 + d2**2)  # [w, nu, nu'] real, symmetric under both rules
    sign = 0.3 if channel == "dens" else -0.3
    struct = _from_compound_orb(m2 / scale, nb)  # [a,b,c,d]
    gamma = u_r[..., None, None, None] + sign * struct[..., None, None, None] * w[None, None, None, None]
    noise = rng.standard_normal(gamma.shape) + 1j * rng.standard_normal(gamma.shape)
    gamma = gamma + 1e-3 * scale * noise
    # nu <-> nu' with orbitals abcd -> cdab (local_four_point.py:588-597)
    gamma = 0.5 * (gamma + np.swapaxes(np.einsum("abcd...->cdab...", gamma), -1, -2))
    # w = 0: F(0, nu, nu') = conj F(0, -nu-1, -nu'-1)
    g0 = gamma[..., 0, :, :]
    gamma[..., 0, :, :] = 0.5 * (g0 + np.conj(np.flip(g0, axis=(-1, -2))))
    return gamma


def local_bubble(g_loc: np.ndarray, niw: int, niv: int, beta: float) -> np.ndarray:
    """chi0_loc[a,b,c,d,w>=0,nu] = -beta G_ad(nu) G_cb(nu - w) (bubble_gen.py:21-30), half w range."""
    niv_g = g_loc.shape[-1] // 2
    nb = g_loc.shape[0]
    out = np.empty((nb, nb, nb, nb, niw + 1, 2 * niv), dtype=np.complex128)
    gl = g_loc[..., niv_g - niv : niv_g + niv]
    for iw in range(niw + 1):
        gr = g_loc[..., niv_g - niv - iw : niv_g + niv - iw]
        out[..., iw, :] = -beta * gl[:, None, None, :, :] * np.swapaxes(gr, 0, 1)[None, :, :, None, :]
    return out


def local_chi_and_f(chi0_loc: np.ndarray, gamma: np.ndarray, beta: float, u_r: np.ndarray):
    """Local auxiliary chi* = (chi0^-1 + (Gamma - U_r)/beta^2)^-1, physical chi and F = beta^2 (chi0^-1 - chi0^-1 chi* chi0^-1).

    Returns (chi_r_phys [a,b,c,d,w] = [(sum_{nu nu'} chi*/beta^2)^-1 + U_r]^-1, F_r [a,b,c,d,w,nu,nu']).
    """
    nb = chi0_loc.shape[0]
    w_dim, nv = chi0_loc.shape[4], chi0_loc.shape[5]
    n = nb * nb * nv
    chi_phys = np.empty((nb, nb, nb, nb, w_dim), dtype=np.complex128)
    f = np.empty((nb, nb, nb, nb, w_dim, nv, nv), dtype=np.complex128)
    eye_v = np.eye(nv)
    for iw in range(w_dim):
        c0 = chi0_loc[..., iw, :]  # [a,b,c,d,nu]
        c0_full = c0[..., :, None] * eye_v  # [a,b,c,d,nu,nu']
        c0m = c0_full.transpose(0, 1, 4, 3, 2, 5).reshape(n, n)
        c0inv = np.linalg.inv(c0m)
        gm = (gamma[..., iw, :, :] - u_r[..., None, None]).transpose(0, 1, 4, 3, 2, 5).reshape(n, n)
        chi = np.linalg.inv(c0inv + gm / beta**2)
        fm = beta**2 * (c0inv - c0inv @ chi @ c0inv)
        aux = chi.reshape(nb, nb, nv, nb, nb, nv).sum(axis=(2, 5)) / beta**2  # [o1,o2,o4,o3]
        um = np.swapaxes(u_r, 2, 3).reshape(nb * nb, nb * nb)
        phys = np.linalg.inv(np.linalg.inv(aux.reshape(nb * nb, nb * nb)) + um)
        chi_phys[..., iw] = phys.reshape(nb, nb, nb, nb).transpose(0, 1, 3, 2)
        f[..., iw, :, :] = fm.reshape(nb, nb, nv, nb, nb, nv).transpose(0, 1, 4, 3, 2, 5)
    return chi_phys, f


def pad_with_u(gamma: np.ndarray, u_r: np.ndarray, niv_pad: int) -> np.ndarray:
    """Gamma outside the core box equals U_r (local_four_point.py:652-669), half w range."""
    niv = gamma.shape[-1] // 2
    if niv_pad <= niv:
        return gamma
    out = np.broadcast_to(u_r[..., None, None, None], gamma.shape[:5] + (2 * niv_pad, 2 * niv_pad)).copy()
    d = niv_pad - niv
    out[..., d : d + 2 * niv, d : d + 2 * niv] = gamma
    return out


# ----------------------------------------------------------------------------------------------
# the full input set
# ----------------------------------------------------------------------------------------------


def make_inputs(cfg: DgaConfig | str) -> dict:
    """All inputs of one nonlocal pass for ``cfg`` (deterministic in ``cfg.seed``)."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    rng = np.random.default_rng(cfg.seed)
    grid = KGrid(cfg.nk, cfg.symmetries)
    ek = dispersion(cfg, grid)
    mu = find_mu(cfg, ek)
    sigma = hubbard_i_sigma(cfg, mu, cfg.niv_g)
    g_k = g_lattice(ek, sigma, mu, cfg.beta)
    u = kanamori_u(cfg)
    v_full = nonlocal_v(cfg, grid)
    g_loc = g_k.mean(axis=(0, 1, 2))

    chi0_loc_full = local_bubble(g_loc, cfg.niw, cfg.niv_full, cfg.beta)
    chi0_loc_core = chi0_loc_full[..., cfg.niv_shell : cfg.niv_shell + 2 * cfg.niv]
    out = {
        "config": cfg.to_dict(),
        "beta": cfg.beta,
        "mu": mu,
        "niw": cfg.niw,
        "niv_core": cfg.niv,
        "niv_shell": cfg.niv_shell,
        "nk": grid.nk,
        "irrk_ind": grid.irrk_ind,
        "irrk_inv": grid.irrk_inv,
        "irrk_count": grid.irrk_count,
        "ek": ek,
        "sigma_loc": sigma,
        "g_k": g_k,
        "u": u,
        "v_q_full": v_full,
        "v_q_irr": v_full[grid.irrk_ind],
    }
    for ch in ("dens", "magn"):
        gamma = gamma_model(cfg, u, ch, rng, cfg.niv)
        out[f"gamma_{ch}"] = gamma
        chi_phys, _ = local_chi_and_f(chi0_loc_core, gamma, cfg.beta, u_channel(u, ch))
        full = np.concatenate([np.conj(np.flip(chi_phys[..., 1:], axis=-1)), chi_phys], axis=-1)
        target = complex(full.sum() / cfg.beta)
        if target.real <= 0.0 and cfg.n_bands == 1:
            # (single band: the only case with a lambda-correction) the model vertex drove the local ladder past its instability (a negative local susceptibility
            # sum, which a DMFT susceptibility never has and for which the lambda equation has no root): use
            # the local bubble's sum instead, the susceptibility of the non-interacting local problem
            c0 = chi0_loc_core.sum(axis=-1) / cfg.beta**2  # [a,b,c,d,w]
            c0_full = np.concatenate([np.conj(np.flip(c0[..., 1:], axis=-1)), c0], axis=-1)
            target = complex(c0_full.sum() / cfg.beta)
        out[f"chi_loc_sum_{ch}"] = target
        if ch == "magn":
            g_pad = pad_with_u(gamma, u_channel(u, ch), cfg.niv_full)
            _, f_magn = local_chi_and_f(chi0_loc_full, g_pad, cfg.beta, u_channel(u, ch))
            out["f_magn_loc"] = f_magn
            out["f_dc"] = 2 * np.einsum("abcd...->cbad...", f_magn)
    return out


def make_occupations(cfg: DgaConfig | str, seed_offset: int = 7919) -> tuple[np.ndarray, np.ndarray]:
    """Seeded occupation matrices for the Hartree-Fock term: occ_k [kx, ky, kz, n, n] Hermitian with eigenvalues
    in (0, 1) (a smooth band-like k dependence plus a small seeded perturbation) and occ = its k average, the
    shapes of config.sys.occ_k / config.sys.occ (dgamore/greens_function.py:212-240)."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    rng = np.random.default_rng(cfg.seed + seed_offset)
    nb = cfg.n_bands
    kx = 2 * np.pi * np.arange(cfg.nk[0]) / cfg.nk[0]
    ky = 2 * np.pi * np.arange(cfg.nk[1]) / cfg.nk[1]
    kz = 2 * np.pi * np.arange(cfg.nk[2]) / cfg.nk[2]
    ek = np.cos(kx)[:, None, None] + np.cos(ky)[None, :, None] + 0.5 * np.cos(kz)[None, None, :]
    occ_k = np.zeros((*cfg.nk, nb, nb), dtype=np.complex128)
    for a in range(nb):
        occ_k[..., a, a] = 0.5 - 0.2 * ek * (1.0 + 0.1 * a)
    pert = 0.02 * (rng.standard_normal((*cfg.nk, nb, nb)) + 1j * rng.standard_normal((*cfg.nk, nb, nb)))
    occ_k += 0.5 * (pert + np.conj(np.swapaxes(pert, -1, -2)))
    occ = occ_k.mean(axis=(0, 1, 2))
    return occ, occ_k


def local_sde_inputs(cfg: DgaConfig | str, niw: int | None = None, niv: int | None = None,
                     niv_shell: int | None = None, nk: tuple = (8, 8, 1), seed_offset: int = 303) -> tuple:
    """Inputs of the local Schwinger-Dyson equation (dgamore/local_sde.py:175) made from the model vertex: the
    k-mean of the lattice G, and G2_r such that the equation returns gamma_model in the core box,

        chi_r = [chi~_core^-1 + (Gamma_r - U_r)/beta^2]^-1,  G2_r = chi_r / beta (+ 2 G_ab(nu) G_cd(nu') at w = 0, dens),

    with chi~_core^-1 the shell-corrected bubble term [(chi0^-1 + U_r/beta^2 over the full box)^-1]_core^-1, G2 in
    the full w range.  Returns ((g, g2_dens, g2_magn, u, beta, niw, niv, niv_shell, occ), (gamma_dens, gamma_magn))."""
    import dataclasses

    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    niw = cfg.niw if niw is None else niw
    niv = cfg.niv if niv is None else niv
    niv_shell = cfg.niv_shell if niv_shell is None else niv_shell
    cfg = dataclasses.replace(cfg, nk=nk, niw=niw, niv=niv, niv_shell=niv_shell)
    rng = np.random.default_rng(cfg.seed + seed_offset)
    grid = KGrid(cfg.nk, cfg.symmetries)
    ek = dispersion(cfg, grid)
    mu = find_mu(cfg, ek)
    niv_g = niv + niv_shell + niw + 4
    g = g_lattice(ek, hubbard_i_sigma(cfg, mu, niv_g), mu, cfg.beta).mean(axis=(0, 1, 2))
    u = kanamori_u(cfg)
    beta = cfg.beta
    nb, nvf, nv = cfg.n_bands, 2 * (niv + niv_shell), 2 * niv
    n2 = nb * nb
    chi0 = local_bubble(g, niw, niv + niv_shell, beta)  # [a,b,c,d,w,nu] full box, w >= 0
    c0 = chi0.transpose(4, 5, 0, 1, 3, 2).reshape(niw + 1, nvf, n2, n2)  # [w][nu][(a,b)][(d,c)]
    c0inv = np.linalg.inv(c0)
    g2s, gammas = [], []
    for ch in ("dens", "magn"):
        u_r = u_channel(u, ch)
        uc = _to_compound_orb(u_r)
        # full-box dense chi~^-1 = blockdiag(chi0^-1) + U_r/beta^2 in every (nu, nu') block
        dense = np.broadcast_to(uc[None, None, :, None, :] / beta**2, (niw + 1, nvf, n2, nvf, n2)).copy()
        for v in range(nvf):
            dense[:, v, :, v, :] += c0inv[:, v]
        dense = dense.transpose(0, 2, 1, 4, 3).reshape(niw + 1, n2 * nvf, n2 * nvf)  # rows (p, nu)
        idx = np.array([p * nvf + niv_shell + v for p in range(n2) for v in range(nv)])
        tilde = np.linalg.inv(np.linalg.inv(dense)[:, idx][:, :, idx])
        gamma = gamma_model(cfg, u, ch, rng, niv)
        gm = (gamma - u_r[..., None, None, None]).transpose(4, 0, 1, 5, 3, 2, 6).reshape(niw + 1, n2 * nv, n2 * nv)
        chi = np.linalg.inv(tilde + gm / beta**2)
        g2 = chi.reshape(niw + 1, nb, nb, nv, nb, nb, nv).transpose(1, 2, 5, 4, 0, 3, 6) / beta  # [a,b,c,d,w,nu,nu']
        if ch == "dens":
            gs = g[..., g.shape[-1] // 2 - niv : g.shape[-1] // 2 + niv]
            g2[:, :, :, :, 0] += 2.0 * gs[:, :, None, None, :, None] * gs[None, None, :, :, None, :]
        neg = np.conj(np.flip(g2[:, :, :, :, 1:], axis=(4, 5, 6)))
        g2s.append(np.concatenate([neg, g2], axis=4))
        gammas.append(gamma)
    occ = make_occupations(cfg)[0]
    return (g, g2s[0], g2s[1], u, beta, niw, niv, niv_shell, occ), tuple(gammas)
