"""NumPy restatement of the upstream local Schwinger-Dyson equation (complex128 throughout).

TEST INFRASTRUCTURE ONLY -- the checker, never the product (see ``oracle/__init__.py``).

Follows ``dgamore/local_sde.py:17-217`` (``perform_local_schwinger_dyson`` and the functions it calls) step by
step, including the upstream's own order of inversions, so that it can be compared with the upstream run
(tests/golden/make_golden_local.py) and, as the checker, with the device form.

Layouts are the upstream objects' ``.mat``:

* ``g``      local G(nu)                 [a, b, 2*niv_g]                   full nu range
* ``g2``     G2_r(w, nu, nu')            [a, b, c, d, 2*niw+1, 2*niv, 2*niv] full w range, core box
* ``u``      U_abcd                      [a, b, c, d]
* results    half w range (w >= 0): Gamma_r, gchi_r [a,b,c,d,niw+1,2niv,2niv]; F_r [..,2niv_full,2niv_full];
             vrg_r [a,b,c,d,niw+1,2niv]; chi_r [a,b,c,d,niw+1]; Sigma_loc [1,1,1,a,b,2niv]

The upstream needs an even niw_core: ``pad_with_u`` and ``identity_like`` (``local_four_point.py:652-669,
717-751``) size the bosonic axis of a half-range object as 2 * (len // 2) + 1.
"""

from __future__ import annotations

import numpy as np

from .ladder import filter_small_values, u_as_channel, wn


# ----------------------------------------------------------------------------------------------
# compound indices (local_four_point.py:206-229, 259-288)
# ----------------------------------------------------------------------------------------------


def to_compound(x: np.ndarray) -> np.ndarray:
    """[a,b,c,d,w,nu,nu'] -> [w, (a,b,nu), (d,c,nu')]."""
    n, w_dim, nv = x.shape[0], x.shape[4], x.shape[5]
    return x.transpose(4, 0, 1, 5, 3, 2, 6).reshape(w_dim, n * n * nv, n * n * nv)


def from_compound(m: np.ndarray, n: int, nv: int) -> np.ndarray:
    """[w, (a,b,nu), (d,c,nu')] -> [a,b,c,d,w,nu,nu']."""
    return m.reshape(m.shape[0], n, n, nv, n, n, nv).transpose(1, 2, 5, 4, 0, 3, 6)


def extend_diag(x: np.ndarray) -> np.ndarray:
    """[..., nu] -> [..., nu, nu] on the diagonal (local_n_point.py:163-175)."""
    return x[..., :, None] * np.eye(x.shape[-1])


def inv_diag(x: np.ndarray) -> np.ndarray:
    """Inverse of an object with one nu dimension [a,b,c,d,w,nu]: the compound matrix is block diagonal in nu,
    so the inverse is the per-nu inverse of the [(a,b),(d,c)] blocks (LocalFourPoint.invert,
    local_four_point.py:298-310, with the diagonal extension of :220-221)."""
    n, w_dim, nv = x.shape[0], x.shape[4], x.shape[5]
    blocks = x.transpose(4, 5, 0, 1, 3, 2).reshape(w_dim, nv, n * n, n * n)
    inv = np.linalg.inv(blocks).reshape(w_dim, nv, n, n, n, n)
    return inv.transpose(2, 3, 5, 4, 0, 1)


def inv_orb(x: np.ndarray) -> np.ndarray:
    """Inverse of an object without nu dimensions [a,b,c,d,w] in [(a,b),(d,c)] compound form."""
    n, w_dim = x.shape[0], x.shape[4]
    m = x.transpose(4, 0, 1, 3, 2).reshape(w_dim, n * n, n * n)
    return np.linalg.inv(m).reshape(w_dim, n, n, n, n).transpose(1, 2, 4, 3, 0)


def inv_dense(x: np.ndarray) -> np.ndarray:
    n, nv = x.shape[0], x.shape[5]
    return from_compound(np.linalg.inv(to_compound(x)), n, nv)


def matmul_dense(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    n, nv = x.shape[0], x.shape[5]
    return from_compound(to_compound(x) @ to_compound(y), n, nv)


def half_niw(x: np.ndarray, n_freq_axes: int) -> np.ndarray:
    """w >= 0 part of a full-range object (local_n_point.py:227-240)."""
    axis = x.ndim - n_freq_axes
    n_w = x.shape[axis]
    return np.take(x, np.arange(n_w // 2, n_w), axis=axis)


def full_niw(x: np.ndarray, n_freq_axes: int) -> np.ndarray:
    """Full w range from w >= 0: X(-w) = conj X(w) flipped along every frequency axis (local_n_point.py:191-225)."""
    axes = tuple(range(x.ndim - n_freq_axes, x.ndim))
    w_axis = axes[0]
    neg = np.conj(np.flip(np.take(x, np.arange(1, x.shape[w_axis]), axis=w_axis), axis=axes))
    return np.concatenate([neg, x], axis=w_axis)


# ----------------------------------------------------------------------------------------------
# the local SDE (local_sde.py)
# ----------------------------------------------------------------------------------------------


def local_bubble(g: np.ndarray, niw: int, niv: int, beta: float) -> np.ndarray:
    """chi0[a,b,c,d,w,nu] = -beta G_ad(nu) G_cb(nu - w), full w range, values below 1e-12 in both parts
    set to zero (BubbleGenerator.create_generalized_chi0, bubble_gen.py:20-30)."""
    niv_g = g.shape[-1] // 2
    w = wn(niw)
    v = np.arange(-niv, niv)
    g_left = g[:, None, None, :, None, niv_g - niv : niv_g + niv]
    g_right = np.swapaxes(g, 0, 1)[None, :, :, None, niv_g + v[None, :] - w[:, None]]
    return filter_small_values(-beta * g_left * g_right)


def generalized_chi(g2: np.ndarray, g: np.ndarray, beta: float, niv_core: int, dens: bool) -> np.ndarray:
    """chi = beta G2 (half w range) - 2 beta G_ab(nu) G_cd(nu') at w = 0 in the density channel
    (create_generalized_chi, local_sde.py:17-29)."""
    chi = beta * half_niw(g2, 3)
    if dens:
        niv_g = g.shape[-1] // 2
        gs = g[..., niv_g - niv_core : niv_g + niv_core]
        ggv = gs[:, :, None, None, :, None] * gs[None, None, :, :, None, :]
        chi[:, :, :, :, 0] -= 2.0 * beta * ggv
    return chi


def chi_tilde_core_inv(chi0_half: np.ndarray, u_r: np.ndarray, beta: float, niv_core: int) -> np.ndarray:
    """[(chi0^-1 + U_r/beta^2)^-1 over the full box, cut to the core]^-1 (local_sde.py:49-50).  chi0^-1 comes back
    from ``invert`` with two nu dimensions (block diagonal), so U_r/beta^2 is added to every (nu, nu') entry and
    the result is dense in nu."""
    chi0_inv_full = extend_diag(inv_diag(chi0_half))
    chi_tilde_shell = inv_dense(chi0_inv_full + u_r[..., None, None, None] / beta**2)
    s = chi0_half.shape[-1] // 2 - niv_core
    return inv_dense(chi_tilde_shell[..., s : s + 2 * niv_core, s : s + 2 * niv_core])


def gamma_with_shell(gchi: np.ndarray, chi0_half: np.ndarray, u_r: np.ndarray, beta: float, niv_core: int) -> np.ndarray:
    """Gamma = beta^2 (chi^-1 - chi~_core^-1) + U_r (create_gamma_r_with_shell_correction, local_sde.py:40-51)."""
    return beta**2 * (inv_dense(gchi) - chi_tilde_core_inv(chi0_half, u_r, beta, niv_core)) + u_r[..., None, None, None]


def pad_with_u(gamma: np.ndarray, u_r: np.ndarray, niv_pad: int) -> np.ndarray:
    """Gamma inside the core box, U_r outside it (LocalFourPoint.pad_with_u, local_four_point.py:652-669)."""
    niv = gamma.shape[-1] // 2
    if niv_pad <= niv:
        return gamma.copy()
    out = np.broadcast_to(u_r[..., None, None, None], gamma.shape[:5] + (2 * niv_pad, 2 * niv_pad)).copy()
    d = niv_pad - niv
    out[..., d : d + 2 * niv, d : d + 2 * niv] = gamma
    return out


def full_vertex_from_gamma(gamma: np.ndarray, chi0_half: np.ndarray, u_r: np.ndarray, beta: float, niv_full: int):
    """F = Gamma_u [1 + chi0 Gamma_u / beta^2]^-1 in the full box (create_full_vertex_from_gamma,
    local_sde.py:75-82); chi0 Gamma_u is the per-nu orbital product of local_four_point.py:349-372."""
    gamma_u = pad_with_u(gamma, u_r, niv_full)
    n, w_dim, nv = gamma_u.shape[0], gamma_u.shape[4], gamma_u.shape[5]
    c0g = np.einsum("abcdwv,dcefwvp->abefwvp", chi0_half, gamma_u)
    eye = from_compound(np.broadcast_to(np.eye(n * n * nv), (w_dim, n * n * nv, n * n * nv)).copy(), n, nv)
    return matmul_dense(gamma_u, inv_dense(eye + c0g / beta**2))


def auxiliary_chi(gamma: np.ndarray, chi0_inv_core: np.ndarray, u_r: np.ndarray, beta: float) -> np.ndarray:
    """chi* = (chi0^-1 + (Gamma - U_r)/beta^2)^-1 (create_auxiliary_chi, local_sde.py:54-59)."""
    return inv_dense(extend_diag(chi0_inv_core) + (gamma - u_r[..., None, None, None]) / beta**2)


def vrg(chi_aux: np.ndarray, chi0_inv_core: np.ndarray, beta: float) -> np.ndarray:
    """gamma_r(w, nu) = beta chi0^-1(nu) (sum_nu' chi*(nu, nu') / beta) (create_vrg, local_sde.py:93-99)."""
    aux_sum = chi_aux.sum(axis=-1) / beta
    return beta * np.einsum("abcdwv,dcefwv->abefwv", chi0_inv_core, aux_sum)


def chi_with_shell(aux_sum: np.ndarray, chi0_half: np.ndarray, u_r: np.ndarray, beta: float, niv_core: int):
    """chi_r(w) = ((chi*_sum + chi0_full_sum - chi0_core_sum)^-1 + U_r)^-1 with chi0 sums (1/beta^2) sum_nu chi0
    (create_generalized_chi_with_shell_correction, local_sde.py:62-72)."""
    s = chi0_half.shape[-1] // 2 - niv_core
    full_sum = chi0_half.sum(axis=-1) / beta**2
    core_sum = chi0_half[..., s : s + 2 * niv_core].sum(axis=-1) / beta**2
    return inv_orb(inv_orb(aux_sum + full_sum - core_sum) + u_r[..., None])


def vertex_functions(g2, chi0_half, chi0_inv_core, g, u, beta, niv_core, niv_full, channel):
    """One channel of create_vertex_functions (local_sde.py:102-147): Gamma, chi (shell-corrected), vrg, F, gchi."""
    u_r = u_as_channel(u, channel)
    gchi = generalized_chi(g2, g, beta, niv_core, channel == "dens")
    gamma = gamma_with_shell(gchi, chi0_half, u_r, beta, niv_core)
    f = full_vertex_from_gamma(gamma, chi0_half, u_r, beta, niv_full)
    chi_aux = auxiliary_chi(gamma, chi0_inv_core, u_r, beta)
    vrg_r = vrg(chi_aux, chi0_inv_core, beta)
    aux_sum = chi_aux.sum(axis=(-2, -1)) / beta**2
    chi_r = chi_with_shell(aux_sum, chi0_half, u_r, beta, niv_core)
    return gamma, chi_r, vrg_r, f, gchi


def sigma_loc_vrg(vrg_d, vrg_m, chi_d, chi_m, g, u, occ, beta, niw, niv_core):
    """Sigma_ij(nu) = -1/beta sum U_kjop inner_ilpo(w, nu) G_lk(nu - w) + U_dens_abcd occ_dc with
    inner = [vrg_d - vrg_d U_d chi_d - (vrg_m - vrg_m U_m chi_m)] / 2 over the full w range
    (get_loc_self_energy_vrg, local_sde.py:150-172)."""
    u_d, u_m = u_as_channel(u, "dens"), u_as_channel(u, "magn")

    def dress(v, u_r, chi):
        vu = np.einsum("abijwv,jief->abefwv", v, u_r)
        return v - np.einsum("abcdwv,dcefw->abefwv", vu, chi)

    inner = 0.5 * full_niw(dress(vrg_d, u_d, chi_d) - dress(vrg_m, u_m, chi_m), 2)
    niv_g = g.shape[-1] // 2
    v = np.arange(-niv_core, niv_core)
    g_wv = g[..., niv_g + v[None, :] - wn(niw)[:, None]]
    sigma = -1.0 / beta * np.einsum("kjop,ilpowv,lkwv->ijv", u, inner, g_wv)
    hf = np.einsum("abcd,dc->ab", u_d, occ)[..., None]
    return (hf + sigma)[None, None, None]


def perform_local_schwinger_dyson(g, g2_dens, g2_magn, u, beta, niw, niv_core, niv_shell, occ):
    """perform_local_schwinger_dyson (local_sde.py:175-217) without orbital symmetrisation; returns the upstream's
    11 results in its order: gamma_d, gamma_m, chi_d, chi_m, vrg_d, vrg_m, f_d, f_m, gchi_d, gchi_m, sigma_loc."""
    niv_full = niv_core + niv_shell
    chi0 = local_bubble(g, niw, niv_full, beta)
    chi0_half = half_niw(chi0, 2)
    s = niv_full - niv_core
    chi0_inv_core = inv_diag(chi0_half[..., s : s + 2 * niv_core])
    d = vertex_functions(g2_dens, chi0_half, chi0_inv_core, g, u, beta, niv_core, niv_full, "dens")
    m = vertex_functions(g2_magn, chi0_half, chi0_inv_core, g, u, beta, niv_core, niv_full, "magn")
    sigma = sigma_loc_vrg(d[2], m[2], d[1], m[1], g, u, occ, beta, niw, niv_core)
    return d[0], m[0], d[1], m[1], d[2], m[2], d[3], m[3], d[4], m[4], sigma
