"""NumPy restatement of the upstream ladder-DGA hot path (complex128 throughout).

TEST INFRASTRUCTURE ONLY -- the checker, never the product (see ``oracle/__init__.py``).

Array layouts follow the upstream objects exactly:

* ``g_k``      G(k, nu)            [kx, ky, kz, a, b, 2*niv_g]          full nu range, nu index = n + niv_g
* ``chi0``     chi0(q_irr, w>=0, nu) [q, a, b, c, d, niw+1, 2*niv]      (FourPoint, half w range, one nu)
* ``gamma``    Gamma_r(w>=0, nu, nu') [a, b, c, d, niw+1, 2*niv, 2*niv]  (LocalFourPoint, half w range)
* ``u``        U_abcd              [a, b, c, d]
* ``v_q``      V^q_abcd            [q, a, b, c, d]                      reduced to the q list in use
* compound index of the BSE matrix: row (o1, o2, nu), column (o4, o3, nu')  (four_point.py:216-219)
"""

from __future__ import annotations

import numpy as np
import scipy.fft as sp_fft

# ----------------------------------------------------------------------------------------------
# Matsubara helpers and channel algebra
# ----------------------------------------------------------------------------------------------


def wn(niw: int, only_positive: bool = False) -> np.ndarray:
    """Bosonic indices [-niw, niw] or [0, niw] (matsubara_frequencies.py:21-30)."""
    return np.arange(0, niw + 1) if only_positive else np.arange(-niw, niw + 1)


def vn_values(niv: int, beta: float) -> np.ndarray:
    """Fermionic frequencies (2n+1)pi/beta for n in [-niv, niv) (matsubara_frequencies.py:44-62)."""
    return np.pi / beta * (2 * np.arange(-niv, niv) + 1)


def u_as_channel(u: np.ndarray, channel: str) -> np.ndarray:
    """Local interaction in a spin channel (interaction.py:43-65): dens 2U - U_adcb, magn -U_adcb."""
    u_adcb = np.einsum("abcd->adcb", u)
    if channel == "dens":
        return 2 * u - u_adcb
    if channel == "magn":
        return -u_adcb
    if channel == "sing":
        return u + u_adcb
    if channel == "trip":
        return u - u_adcb
    raise ValueError(channel)


def v_as_channel(v_q: np.ndarray, channel: str) -> np.ndarray:
    """Non-local interaction in a spin channel (interaction.py:160-182): dens 2V, magn 0."""
    if channel == "dens":
        return 2 * v_q
    if channel == "magn":
        return 0 * v_q
    if channel in ("sing", "trip"):
        return v_q.copy()
    raise ValueError(channel)


def filter_small_values(x: np.ndarray, threshold: float = 1e-12) -> np.ndarray:
    """Zeroes entries whose real and imaginary parts are both below threshold (n_point_base.py:205-211)."""
    x = x.copy()
    x[(np.abs(x.real) < threshold) & (np.abs(x.imag) < threshold)] = 0.0
    return x


def to_full_niw_range(x: np.ndarray, n_freq_axes: int) -> np.ndarray:
    """Half (w>=0) to full w range: F(-w) = conj(flip_all_freq_axes F(w)) (local_n_point.py:191-225).

    ``n_freq_axes`` counts the bosonic axis plus the fermionic axes that follow it (all at the end).
    """
    axis = x.ndim - n_freq_axes
    freq_axes = tuple(range(axis, x.ndim))
    pos = x
    src = np.take(x, np.arange(1, x.shape[axis]), axis=axis)
    neg = np.conj(np.flip(src, axis=freq_axes))
    return np.concatenate([neg, pos], axis=axis)


def flip_momentum_axis(x: np.ndarray) -> np.ndarray:
    """F(q) -> F(-q) on a [kx,ky,kz,...] array: roll(flip(., axes 0-2), 1) (n_point_base.py:553-574)."""
    return np.roll(np.flip(x, axis=(0, 1, 2)), shift=1, axis=(0, 1, 2))


# ----------------------------------------------------------------------------------------------
# Green's function
# ----------------------------------------------------------------------------------------------


def g_full(sigma_k: np.ndarray, mu: float, ek: np.ndarray, beta: float) -> np.ndarray:
    """G(k,nu) = [i nu + mu - e_k - Sigma(k,nu)]^-1 per (k, nu) (greens_function.py:125-142).

    sigma_k: [kx,ky,kz,a,b,2niv] (or [1,1,1,a,b,2niv] for a local Sigma), ek: [kx,ky,kz,a,b].
    """
    nb = ek.shape[-1]
    niv = sigma_k.shape[-1] // 2
    eye = np.eye(nb)
    iv = 1j * vn_values(niv, beta)
    mat = (iv[None, None, :] * eye[..., None])[None, None, None] + (mu * eye[:, :, None])[None, None, None]
    mat = mat - ek[..., None] - sigma_k
    return np.linalg.inv(mat.transpose(0, 1, 2, 5, 3, 4)).transpose(0, 1, 2, 4, 5, 3)


# ----------------------------------------------------------------------------------------------
# (a1) bare bubble via FFT over the Brillouin zone
# ----------------------------------------------------------------------------------------------


def chi0_q_fft(g_k: np.ndarray, niw: int, niv: int, irrk_ind: np.ndarray, beta: float) -> np.ndarray:
    """chi0[q_irr,a,b,c,d,w>=0,nu] = -beta/Nk * IFFT_R[G_ad(R,nu) G_cb(-R,nu-w)] (bubble_gen.py:33-69).

    G(R) is the forward FFT of G(k) (n_point_base.py:509-529), G(-R) = flip_momentum_axis(G(R))
    (bubble_gen.py:46-47); the inverse transform is numpy's normalised ifftn (bubble_gen.py:60), and the
    result is filtered at 1e-12 (bubble_gen.py:69).
    """
    nkx, nky, nkz, nb = g_k.shape[0], g_k.shape[1], g_k.shape[2], g_k.shape[3]
    nk_tot = nkx * nky * nkz
    niv_g = g_k.shape[-1] // 2
    cut = niv + niw
    g_cut = g_k[..., niv_g - cut : niv_g + cut]
    g_r = sp_fft.fftn(g_cut, axes=(0, 1, 2))
    g_r_rev = np.swapaxes(flip_momentum_axis(g_r), 3, 4)  # [x,y,z,b,c] holds G_cb(-R)
    start, end = cut - niv, cut + niv
    g_r_core = g_r[..., start:end]
    out = np.zeros((len(irrk_ind), nb, nb, nb, nb, niw + 1, 2 * niv), dtype=np.complex128)
    for iw in range(niw + 1):
        g_vw = g_r_rev[..., start - iw : end - iw]
        prod = g_r_core[:, :, :, :, None, None, :, :] * g_vw[:, :, :, None, :, :, None, :]
        chi_q = np.fft.ifftn(prod, axes=(0, 1, 2)).reshape(nk_tot, nb, nb, nb, nb, 2 * niv)
        out[..., iw, :] = chi_q[irrk_ind]
    out *= -beta / nk_tot
    return filter_small_values(out)


def chi0_pp_w0_q(g_k: np.ndarray, niv_pp: int) -> np.ndarray:
    """chi0pp[k,a,b,c,d,nu] = G_ad(k,nu) conj(G_cb(k,nu)), no -beta (bubble_gen.py:268-279). Returns [Nk,...]."""
    niv_g = g_k.shape[-1] // 2
    g = g_k[..., niv_g - niv_pp : niv_g + niv_pp]
    nk = g.shape[0] * g.shape[1] * g.shape[2]
    g = g.reshape(nk, *g.shape[3:])
    gt = np.swapaxes(g, 1, 2)
    out = g[:, :, None, None, :, :] * np.conj(gt)[:, None, :, :, None, :]
    return filter_small_values(out)


# ----------------------------------------------------------------------------------------------
# (a4) chi0^-1 per (q, w, nu) and frequency sums
# ----------------------------------------------------------------------------------------------


def chi0_inv(chi0: np.ndarray) -> np.ndarray:
    """n^2 x n^2 inverse per (q,w,nu) in the [(o1,o2),(o4,o3)] basis (four_point.py:601-613)."""
    nq, nb, w_dim, nv = chi0.shape[0], chi0.shape[1], chi0.shape[5], chi0.shape[6]
    m = chi0.transpose(0, 5, 6, 1, 2, 4, 3).reshape(nq, w_dim, nv, nb * nb, nb * nb)
    m = np.linalg.inv(m)
    return m.reshape(nq, w_dim, nv, nb, nb, nb, nb).transpose(0, 3, 4, 6, 5, 1, 2)


def cut_niv(x: np.ndarray, niv_cut: int, n_vn: int) -> np.ndarray:
    """Centred cut of the last ``n_vn`` fermionic axes to 2*niv_cut (local_n_point.py:134-154)."""
    niv = x.shape[-1] // 2
    sl = slice(niv - niv_cut, niv + niv_cut)
    if n_vn == 1:
        return x[..., sl]
    return x[..., sl, sl]


def sum_over_all_vn(x: np.ndarray, beta: float, n_vn: int) -> np.ndarray:
    """Sum over the fermionic axes times beta^-n_vn (local_four_point.py:146-177)."""
    axes = (-1,) if n_vn == 1 else (-2, -1)
    return np.sum(x, axis=axes) / beta ** len(axes)


# ----------------------------------------------------------------------------------------------
# (a5) ladder BSE: X = sum_nu' [chi0^-1 + (Gamma_r - U_r - V_r^q)/beta^2]^-1 / beta
# ----------------------------------------------------------------------------------------------


def bse_matrix(chi0_inv_qw: np.ndarray, gamma_w: np.ndarray, uv_q: np.ndarray, beta: float) -> np.ndarray:
    """Compound-index matrix A for one (q, w) (nonlocal_sde.py:85-96 assembled through FourPoint.add).

    chi0_inv_qw: [a,b,c,d,nu]; gamma_w: [a,b,c,d,nu,nu']; uv_q: U_r + V_r^q [a,b,c,d].
    Row (o1,o2,nu), column (o4,o3,nu') as in four_point.py:635.
    """
    nb, nv = gamma_w.shape[0], gamma_w.shape[-1]
    eye = np.eye(nv)
    full = chi0_inv_qw[..., :, None] * eye + gamma_w / beta**2 - uv_q[..., None, None] / beta**2
    n = nb * nb * nv
    return full.transpose(0, 1, 4, 3, 2, 5).reshape(n, n)


def bse_sum(chi0_inv_core: np.ndarray, gamma: np.ndarray, uv_q: np.ndarray, beta: float) -> np.ndarray:
    """Sum over nu' of the auxiliary susceptibility (four_point.py:620-642 via nonlocal_sde.py:85-96).

    chi0_inv_core: [q,a,b,c,d,w,nu]; gamma: [a,b,c,d,w,nu,nu']; uv_q: [q,a,b,c,d] (U_r + V_r^q).
    Returns [q,a,b,c,d,w,nu].
    """
    nq, nb, w_dim, nv = chi0_inv_core.shape[0], chi0_inv_core.shape[1], chi0_inv_core.shape[5], chi0_inv_core.shape[6]
    out = np.empty_like(chi0_inv_core)
    for iq in range(nq):
        for iw in range(w_dim):
            a = bse_matrix(chi0_inv_core[iq, ..., iw, :], gamma[..., iw, :, :], uv_q[iq], beta)
            x = np.linalg.inv(a).reshape(nb, nb, nv, nb, nb, nv)  # [o1,o2,nu,o4,o3,nu']
            out[iq, ..., iw, :] = x.sum(axis=-1).transpose(0, 1, 4, 3, 2) / beta
    return out


def bse_sum_solve(chi0_inv_core: np.ndarray, gamma: np.ndarray, uv_q: np.ndarray, beta: float) -> np.ndarray:
    """Same result through a linear solve with the n^2 selector right-hand sides (four_point.py:644-684)."""
    nq, nb, w_dim, nv = chi0_inv_core.shape[0], chi0_inv_core.shape[1], chi0_inv_core.shape[5], chi0_inv_core.shape[6]
    n = nb * nb * nv
    idx = np.arange(n)
    rhs = np.zeros((n, nb * nb), dtype=np.complex128)
    rhs[idx, (idx // (nb * nv)) * nb + (idx // nv) % nb] = 1.0
    out = np.empty_like(chi0_inv_core)
    for iq in range(nq):
        for iw in range(w_dim):
            a = bse_matrix(chi0_inv_core[iq, ..., iw, :], gamma[..., iw, :, :], uv_q[iq], beta)
            y = np.linalg.solve(a, rhs).reshape(nb, nb, nv, nb, nb)  # [o1,o2,nu,o4,o3]
            out[iq, ..., iw, :] = y.transpose(0, 1, 4, 3, 2) / beta
    return out


def bse_full_inverse(chi0_inv_core: np.ndarray, gamma: np.ndarray, uv_q: np.ndarray, beta: float) -> np.ndarray:
    """Full auxiliary susceptibility chi*[q,a,b,c,d,w,nu,nu'] = A^-1 (nonlocal_sde.py:72-82, four_point.py:615-618)."""
    nq, nb, w_dim, nv = chi0_inv_core.shape[0], chi0_inv_core.shape[1], chi0_inv_core.shape[5], chi0_inv_core.shape[6]
    out = np.empty((nq, nb, nb, nb, nb, w_dim, nv, nv), dtype=np.complex128)
    for iq in range(nq):
        for iw in range(w_dim):
            a = bse_matrix(chi0_inv_core[iq, ..., iw, :], gamma[..., iw, :, :], uv_q[iq], beta)
            x = np.linalg.inv(a).reshape(nb, nb, nv, nb, nb, nv)  # [o1,o2,nu,o4,o3,nu']
            out[iq, ..., iw, :, :] = x.transpose(0, 1, 4, 3, 2, 5)
    return out


# ----------------------------------------------------------------------------------------------
# (a6, a7) three-leg vertex and physical susceptibility with the shell correction
# ----------------------------------------------------------------------------------------------


def vrg(chi0_inv_core: np.ndarray, chi_aux_sum: np.ndarray, beta: float) -> np.ndarray:
    """gamma_r = beta * chi0^-1 @ sum_nu' chi* (nonlocal_sde.py:159-164, einsum of four_point.py:537-541)."""
    return beta * np.einsum("qabcdwv,qdcefwv->qabefwv", chi0_inv_core, chi_aux_sum, optimize=True)


def invert_orbital(x: np.ndarray) -> np.ndarray:
    """n^2 x n^2 inverse of a [q,a,b,c,d,w] object in the [(o1,o2),(o4,o3)] basis (four_point.py:615-618)."""
    nq, nb, w_dim = x.shape[0], x.shape[1], x.shape[5]
    m = x.transpose(0, 5, 1, 2, 4, 3).reshape(nq, w_dim, nb * nb, nb * nb)
    m = np.linalg.inv(m)
    return m.reshape(nq, w_dim, nb, nb, nb, nb).transpose(0, 2, 3, 5, 4, 1)


def chi_phys_shell(
    chi_aux_sum: np.ndarray, chi0_full_sum: np.ndarray, chi0_core_sum: np.ndarray, uv_q: np.ndarray, beta: float
) -> np.ndarray:
    """chi_r(q,w) = [(sum_nu chi*/beta + chi0_full - chi0_core)^-1 + U_r + V_r^q]^-1.

    nonlocal_sde.py:167-182 with the nu sum of nonlocal_sde.py:298.  Inputs [q,a,b,c,d,w(,nu)].
    """
    chi_phys = sum_over_all_vn(chi_aux_sum, beta, 1)
    inner = invert_orbital(chi_phys + chi0_full_sum - chi0_core_sum)
    return invert_orbital(inner + uv_q[..., None])


# ----------------------------------------------------------------------------------------------
# (a13) lambda correction
# ----------------------------------------------------------------------------------------------


def lambda_start(chi_r: np.ndarray) -> float:
    """-min 1/Re chi(q, w=0) (lambda_correction.py:13-18); chi_r [q, 2niw+1]."""
    w0 = chi_r.shape[-1] // 2
    return -np.min(1.0 / chi_r[..., w0].real)  # numpy scalar: float32 for complex64 input, as upstream


def find_lambda(
    chi_r: np.ndarray, chi_loc_sum: complex, irrk_count: np.ndarray, beta: float, nk_tot: int,
    delta: float = 0.1, eps: float = 1e-7, maxiter: int = 1000,
) -> float:
    """Newton iteration with delta halving (lambda_correction.py:28-60); chi_r [q_irr, 2niw+1]."""
    lam0 = lambda_start(chi_r)
    lam = lam0 + delta
    factor = 1 / beta / nk_tot
    for _ in range(maxiter):
        chi_lam = 1.0 / (1.0 / chi_r + lam)
        f = (irrk_count[:, None] * chi_lam).sum() * factor - chi_loc_sum
        fp = -(irrk_count[:, None] * chi_lam**2).sum() * factor
        lam_new = lam - (f / fp).real
        if abs(f.real) < eps:
            return lam_new
        if lam_new < lam:
            delta /= 2
            lam = lam0 + delta
        else:
            lam = lam_new
    return lam


def apply_lambda(chi_r: np.ndarray, lam: float) -> np.ndarray:
    """1 / (1/chi + lambda) (lambda_correction.py:21-25)."""
    return 1.0 / (1.0 / chi_r + lam)


def lambda_correct_single(chi_half: np.ndarray, chi_loc_sum: complex, irrk_count, beta, nk_tot):
    """perform_single_lambda_correction (lambda_correction.py:63-73) for a single-band [q,1,1,1,1,niw+1] chi."""
    full = to_full_niw_range(chi_half, 1)
    mat = full.reshape(full.shape[0], -1)
    lam = find_lambda(mat, chi_loc_sum, irrk_count, beta, nk_tot)
    corrected = apply_lambda(mat, lam)[:, None, None, None, None, :]
    niw = chi_half.shape[-1] - 1
    return corrected[..., niw:], lam


# ----------------------------------------------------------------------------------------------
# (a8, a9) kernels
# ----------------------------------------------------------------------------------------------


def kernel_r(vrg_r: np.ndarray, chi_phys: np.ndarray, uv_q: np.ndarray, channel: str) -> np.ndarray:
    """K_r = U_r @ (gamma - gamma @ U_r @ chi_r [- 2/3 1 in magn]) (nonlocal_sde.py:201-215).

    The products are the einsums of four_point.py:497-501 and 537-541.
    """
    t = np.einsum("qabijwv,qjief->qabefwv", vrg_r, uv_q, optimize=True)
    t = np.einsum("qabcdwv,qdcefw->qabefwv", t, chi_phys, optimize=True)
    k = vrg_r - t
    if channel == "magn":
        nb = k.shape[1]
        ident = np.einsum("ad,bc->abcd", np.eye(nb), np.eye(nb))  # unity in [(o1,o2),(o4,o3)] (four_point.py:732-746)
        k = k - 2.0 / 3.0 * ident[None, ..., None, None]
    return np.einsum("qabij,qjiefwv->qabefwv", uv_q, k, optimize=True)


def sigma_dc_kernel(f_dc: np.ndarray, chi0_full: np.ndarray, u: np.ndarray, beta: float, niv_core: int) -> np.ndarray:
    """K_dc = (U_adcb/beta^2 @ chi0) . F_dc, cut to the core box (nonlocal_sde.py:185-198).

    f_dc: [d,c,e,f,w,nu,nu'] (= 2 F_magn_loc permuted cbad, nonlocal_sde.py:817-820); chi0_full [q,a,b,c,d,w,nu].
    """
    u_adcb = np.einsum("abcd->adcb", u)
    k1 = np.einsum("abij,qjiefwv->qabefwv", u_adcb, chi0_full, optimize=True) / beta**2
    k = np.einsum("qabcdwv,dcefwvp->qabefwp", k1, f_dc, optimize=True)
    return cut_niv(k, niv_core, 1)


# ----------------------------------------------------------------------------------------------
# (a10, a11) IBZ -> FBZ and the Schwinger-Dyson contraction
# ----------------------------------------------------------------------------------------------


def map_to_full_bz(x_irr: np.ndarray, irrk_inv: np.ndarray, rotations=None) -> np.ndarray:
    """x[k] = x_irr[irrk_inv[k]] (n_point_base.py:489-494); with the auto-mode ``rotations`` = (us [Nk][n][n],
    sigmas [Nk], conjs [Nk]) of a four-orbital object [k, a, b, c, d, ...] also
    x_abcd(k) = sigma_k^2 U_ap U*_bq U_cr U*_ds [x_pqrs(k_rep)]^{(*conj_k)} (n_point_base.py:496-504,
    symmetry_reduction.py:791-902)."""
    x = np.take(x_irr, irrk_inv.ravel(), axis=0)
    if rotations is None:
        return x
    us, sigmas, conjs = rotations
    out = np.empty_like(x)
    for k in range(x.shape[0]):
        blk = np.conj(x[k]) if conjs[k] else x[k]
        u = us[k]
        out[k] = sigmas[k] ** 2 * np.einsum("ap,bq,cr,ds,pqrs...->abcd...", u, u.conj(), u, u.conj(), blk)
    return out


def sigma_from_kernel_fft(kernel_full: np.ndarray, g_k: np.ndarray, nk: tuple, beta: float, niv_core: int) -> np.ndarray:
    """Sigma(k, nu) from the full-BZ kernel through real space (nonlocal_sde.py:544-594, 876-879).

    kernel_full: [Nk, a,b,c,d, niw+1, 2*niv_core] (half w, full nu); g_k: [kx,ky,kz,a,b,2niv_g].
    Returns Sigma [Nk, a, b, 2*niv_core] (full nu range, after ifft and to_full_niv_range).
    """
    nkx, nky, nkz = nk
    nk_tot = nkx * nky * nkz
    nb = g_k.shape[3]
    niv_g = g_k.shape[-1] // 2
    g_r = sp_fft.fftn(g_k, axes=(0, 1, 2)).reshape(nk_tot, nb, nb, -1)
    kfull = to_full_niw_range(kernel_full, 2)[..., niv_core:]  # [Nk, abcd, 2niw+1, niv_core]
    niw = (kfull.shape[-2] - 1) // 2
    k_grid = np.conj(kfull).reshape(nkx, nky, nkz, *kfull.shape[1:])
    k_r = np.conj(sp_fft.fftn(k_grid, axes=(0, 1, 2))).reshape(nk_tot, *kfull.shape[1:])
    mat = np.zeros((nk_tot, nb, nb, niv_core), dtype=np.complex128)
    for iw, w in enumerate(range(-niw, niw + 1)):
        g_slice = g_r[..., niv_g - w : niv_g + niv_core - w]
        mat += np.einsum("Radv,Raijdv->Rijv", g_slice, k_r[..., iw, :], optimize=True)
    mat *= -0.5 / beta / nk_tot
    sig = sp_fft.ifftn(mat.reshape(nkx, nky, nkz, nb, nb, niv_core), axes=(0, 1, 2)).reshape(nk_tot, nb, nb, niv_core)
    return np.concatenate([np.conj(np.flip(sig, axis=-1)), sig], axis=-1)  # self_energy.py:109-120


def sigma_from_kernel_direct(kernel_full: np.ndarray, g_k: np.ndarray, nk: tuple, beta: float, niv_core: int) -> np.ndarray:
    """Direct q-loop variant (nonlocal_sde.py:430-469): Sigma_ij(k,nu) = -1/(2 beta Nq) sum_q,w G_ad(k+q,nu-w) K_aijd."""
    nkx, nky, nkz = nk
    nk_tot = nkx * nky * nkz
    nb = g_k.shape[3]
    niv_g = g_k.shape[-1] // 2
    kfull = to_full_niw_range(kernel_full, 2)[..., niv_core:]
    niw = (kfull.shape[-2] - 1) // 2
    mat = np.zeros((nkx, nky, nkz, nb, nb, niv_core), dtype=np.complex128)
    qs = np.array(np.unravel_index(np.arange(nk_tot), (nkx, nky, nkz))).T
    kx, ky, kz = np.arange(nkx), np.arange(nky), np.arange(nkz)
    for iq, q in enumerate(qs):
        gq = g_k[((kx + q[0]) % nkx)[:, None, None], ((ky + q[1]) % nky)[None, :, None], ((kz + q[2]) % nkz)[None, None, :]]
        for iw, w in enumerate(range(-niw, niw + 1)):
            g_slice = gq[..., niv_g - w : niv_g + niv_core - w]
            mat += np.einsum("xyzadv,aijdv->xyzijv", g_slice, kfull[iq, ..., iw, :], optimize=True)
    mat *= -0.5 / beta / nk_tot
    sig = mat.reshape(nk_tot, nb, nb, niv_core)
    return np.concatenate([np.conj(np.flip(sig, axis=-1)), sig], axis=-1)


# ----------------------------------------------------------------------------------------------
# One nonlocal SDE pass (bubble -> BSE in dens/magn -> vertex -> lambda -> kernel -> Sigma)
# ----------------------------------------------------------------------------------------------


def hartree_fock(u: np.ndarray, v_full: np.ndarray, occ: np.ndarray, occ_k: np.ndarray):
    """Hartree and Fock terms (nonlocal_sde.get_hartree_fock, dgamore/nonlocal_sde.py:31-69) with the full,
    ordered q list of one rank:

        hartree[a,b] = 2 sum_cd (U + V_(q=0))[a,b,c,d] occ[d,c]                        (nonlocal_sde.py:45)
        fock[k,a,b]  = -1/Nq sum_q sum_cd (U + V_q)[a,b,c,d] occ_k[k+q][d,c]          (nonlocal_sde.py:52-68)

    (the upstream pairs the permuted interaction uq[:, a, d, c, b] = (U + V_q)[a, b, c, d] with
    np.roll(occ_k, -q), i.e. occ_k at k + q).  v_full: [kx, ky, kz, a, b, c, d]; occ_k: [kx, ky, kz, n, n].
    Returns hartree [1, n, n, 1] and fock [Nk, n, n, 1] as the upstream does."""
    nk = occ_k.shape[:3]
    nb = occ.shape[0]
    hartree = 2.0 * np.einsum("abcd,dc->ab", u + v_full[0, 0, 0], occ)
    nk_tot = int(np.prod(nk))
    fock = np.zeros((nk_tot, nb, nb), dtype=np.result_type(v_full, occ_k))
    for qx in range(nk[0]):
        for qy in range(nk[1]):
            for qz in range(nk[2]):
                w = u + v_full[qx, qy, qz]
                occ_shift = np.roll(occ_k, (-qx, -qy, -qz), axis=(0, 1, 2)).reshape(nk_tot, nb, nb)
                fock += np.einsum("abcd,kdc->kab", w, occ_shift)
    fock *= -1.0 / nk_tot
    return hartree[None, ..., None], fock[..., None]


def sde_pass(inp: dict, do_lambda: bool = True) -> dict:
    """One pass of the hot path of nonlocal_sde.calculate_self_energy_q (nonlocal_sde.py:786-879).

    ``inp`` keys: g_k [kx,ky,kz,n,n,2niv_g], beta, niw, niv_core, niv_shell, nk (tuple), irrk_ind, irrk_inv,
    irrk_count, u [n,n,n,n], v_q_irr [q_irr,n,n,n,n], gamma_dens, gamma_magn [n,n,n,n,niw+1,2niv,2niv],
    f_dc [n,n,n,n,niw+1,2niv_full,2niv_full], chi_loc_sum_dens/magn (complex, lambda targets 'spch').
    Returns the intermediate and final arrays keyed by name.
    """
    beta, niw, niv_core, niv_shell = inp["beta"], inp["niw"], inp["niv_core"], inp["niv_shell"]
    niv_full = niv_core + niv_shell
    out = {}
    chi0 = chi0_q_fft(inp["g_k"], niw, niv_full, inp["irrk_ind"], beta)
    out["chi0"] = chi0
    k_total = -sigma_dc_kernel(inp["f_dc"], chi0, inp["u"], beta, niv_core)
    out["kernel_dc"] = -k_total
    chi0_full_sum = sum_over_all_vn(chi0, beta, 1) / beta
    chi0_core = cut_niv(chi0, niv_core, 1)
    chi0_core_inv = chi0_inv(chi0_core)
    out["chi0_inv"] = chi0_core_inv
    chi0_core_sum = sum_over_all_vn(chi0_core, beta, 1) / beta
    lambdas = {}
    for ch, factor in (("dens", 1.0), ("magn", 3.0)):
        uv = u_as_channel(inp["u"], ch)[None] + v_as_channel(inp["v_q_irr"], ch)
        aux = bse_sum(chi0_core_inv, inp[f"gamma_{ch}"], uv, beta)
        out[f"chi_aux_sum_{ch}"] = aux
        g3 = vrg(chi0_core_inv, aux, beta)
        out[f"vrg_{ch}"] = g3
        chi_phys = chi_phys_shell(aux, chi0_full_sum, chi0_core_sum, uv, beta)
        out[f"chi_phys_{ch}_before_lambda"] = chi_phys
        if do_lambda:
            chi_phys, lam = lambda_correct_single(
                chi_phys, inp[f"chi_loc_sum_{ch}"], inp["irrk_count"], beta, int(np.prod(inp["nk"]))
            )
            lambdas[ch] = lam
        out[f"chi_phys_{ch}"] = chi_phys
        k_r = kernel_r(g3, chi_phys, uv, ch)
        out[f"kernel_{ch}"] = k_r
        k_total = k_total + factor * k_r
    out["lambdas"] = lambdas
    out["kernel"] = k_total
    rot = (inp["orbital_us"], inp["orbital_sigmas"], inp["orbital_conjs"]) if "orbital_us" in inp else None
    k_full = map_to_full_bz(k_total, inp["irrk_inv"], rot)
    out["sigma"] = sigma_from_kernel_fft(k_full, inp["g_k"], tuple(inp["nk"]), beta, niv_core)
    return out


# ----------------------------------------------------------------------------------------------
# (a14, a15) Eliashberg: full vertex, PH -> PP (w = 0), pairing vertex and the pairing-kernel eigen-solve
# ----------------------------------------------------------------------------------------------


def full_vertex_q(chi0_inv_core, gamma, uv_q, vrg_r, chi_phys, beta, niv_pp):
    """F_r(q,w) = beta^2 (chi0^-1 - chi0^-1 chi* chi0^-1) + U_r g g - U_r chi_r U_r g g, cut to the pp box.

    eliashberg_solver.py:175-204 (create_full_vertex_q_r_v2) with chi* the full auxiliary susceptibility
    (nonlocal_sde.py:72-82), the products of four_point.py:442-588 and the nu-cut of local_n_point.py:134-154.
    Inputs as in ``sde_pass``; chi_phys [q,a,b,c,d,w] is the (lambda-corrected) physical susceptibility.
    Returns [q,a,b,c,d,w,2niv_pp,2niv_pp] (half w range).
    """
    chi_star = bse_full_inverse(chi0_inv_core, gamma, uv_q, beta)  # [q,abcd,w,nu,nu']
    nv = chi0_inv_core.shape[-1]
    eye = np.eye(nv)
    d_full = chi0_inv_core[..., :, None] * eye  # [q,abcd,w,nu,nu'] diagonal in nu
    t = np.einsum("qabcdwv,qdcefwvp->qabefwvp", chi0_inv_core, chi_star, optimize=True)
    t = np.einsum("qabcdwvp,qdcefwp->qabefwvp", t, chi0_inv_core, optimize=True)
    f1 = beta**2 * (d_full - t)
    gg = np.einsum("qabcdwv,qdcefwp->qabefwvp", vrg_r, vrg_r, optimize=True)
    ugg = np.einsum("qabij,qjiefwvp->qabefwvp", uv_q, gg, optimize=True)
    uc = np.einsum("qabij,qjiefw->qabefw", uv_q, chi_phys, optimize=True)
    ucu = np.einsum("qabijw,qjief->qabefw", uc, uv_q, optimize=True)
    ucugg = np.einsum("qabcdw,qdcefwvp->qabefwvp", ucu, gg, optimize=True)
    f = f1 + ugg - ucugg
    return cut_niv(f, niv_pp, 2)


def ph_to_pp_w0(f_half, niw, niv_pp):
    """Full vertex to the modified pp notation at w = 0 (eliashberg_solver.py:44-75).

    f_half: [q,a,b,c,d,w>=0,2niv_pp,2niv_pp] (pp box) -> [q,a,b,c,d,2niv_pp,2niv_pp];
    F_pp[nu, nu'] = -F_full[w = nu - nu'][nu][-nu'-1] with F(-w) = conj(flip F(w)).
    """
    nv = 2 * niv_pp
    vn = np.arange(-niv_pp, niv_pp)
    omega = vn[:, None] - vn[None, :]
    full = to_full_niw_range(f_half[..., : niw + 1, :, :], 3)
    full = np.flip(full, axis=-1)
    out = np.zeros(f_half.shape[:-3] + (nv, nv), dtype=np.complex128)
    for idx, w in enumerate(range(-niw, niw + 1)):
        mask = omega == w
        out[..., mask] = -full[..., idx, :, :][..., mask]
    return out


def chi0_pp_full_grid(g_k, niv_pp):
    """chi0pp[kx,ky,kz,a,b,c,d,nu] decompressed (bubble_gen.py:268-279 then decompress_q_dimension)."""
    nk = g_k.shape[:3]
    c = chi0_pp_w0_q(g_k, niv_pp)
    return c.reshape(*nk, *c.shape[1:])


def eliashberg_matvec(gamma_r_signed, gamma_flip, chi0pp, gap, beta, sign):
    """One application of the linearised gap equation (eliashberg_solver.py:420-428).

    gamma_r_signed: sign * FFT_q Gamma_pp(q) [x,y,z,a,b,c,d,nu,nu']; gamma_flip its flipped form
    (flip_momentum_axis, flip nu', permute abcd->adcb); chi0pp [x,y,z,a,b,c,d,nu]; gap [x,y,z,a,b,nu].
    """
    nk_tot = int(np.prod(gap.shape[:3]))
    norm = 0.5 / nk_tot / beta
    gap_gg = np.fft.fftn(np.einsum("xyzabcdv,xyzcdv->xyzabv", chi0pp, gap, optimize=True), axes=(0, 1, 2))
    gap_gg_flipped = np.roll(np.flip(gap_gg, axis=(0, 1, 2)), shift=1, axis=(0, 1, 2))
    new = np.einsum("xyzacbdvp,xyzcdp->xyzabv", gamma_r_signed, gap_gg, optimize=True) + sign * np.einsum(
        "xyzacbdvp,xyzcdp->xyzabv", gamma_flip, gap_gg_flipped, optimize=True
    )
    return np.fft.ifftn(norm * new, axes=(0, 1, 2))


def eliashberg_operator(gamma_pp_irr, irrk_inv, nk, chi0pp, beta, channel, rotations=None):
    """Gamma(R) and its flipped form for the matvec (eliashberg_solver.py:392-400); gamma_pp_irr [q_irr,...];
    ``rotations``: the auto-mode per-k orbital rotations of the IBZ -> FBZ map (map_to_full_bz)."""
    sign = 1 if channel == "sing" else -1
    full = map_to_full_bz(gamma_pp_irr, irrk_inv, rotations).reshape(*nk, *gamma_pp_irr.shape[1:])
    g_r = sign * sp_fft.fftn(full, axes=(0, 1, 2))
    flip = flip_momentum_axis(g_r)
    flip = np.flip(flip, axis=-1)
    flip = np.einsum("xyzabcd...->xyzadcb...", flip)
    return g_r, flip, sign


def eliashberg_eigs(gamma_pp_irr, irrk_inv, nk, chi0pp, beta, channel, v0, n_eig=4, tol=1e-10, rotations=None):
    """Leading eigenvalues via ARPACK eigsh(which='LA') as eliashberg_solver.py:430-452."""
    import scipy.sparse.linalg as spla

    g_r, flip, sign = eliashberg_operator(gamma_pp_irr, irrk_inv, nk, chi0pp, beta, channel, rotations)
    shape = v0.shape

    def mv(x):
        return eliashberg_matvec(g_r, flip, chi0pp, x.reshape(shape), beta, sign).ravel()

    dim = int(np.prod(shape))
    op = spla.LinearOperator((dim, dim), matvec=mv, dtype=np.complex128)
    vals, vecs = spla.eigsh(op, k=n_eig, tol=tol, v0=v0.ravel(), which="LA", maxiter=10000)
    order = np.argsort(vals)[::-1]
    return vals[order], vecs[:, order]


def d_wave_gap(nk, n_bands, niv_pp, channel):
    """Initial gap of symmetry 'd-wave' (eliashberg_solver.py:339-372): -cos kx + cos ky, even (singlet) or odd in nu."""
    kx = np.linspace(0, 2 * np.pi, nk[0], endpoint=False)
    ky = np.linspace(0, 2 * np.pi, nk[1], endpoint=False)
    nv = 2 * niv_pp
    gap = np.zeros((*nk, n_bands, n_bands, nv), dtype=np.complex128)
    sym = -np.cos(kx)[:, None, None] + np.cos(ky)[None, :, None]
    gap[..., niv_pp:] = np.repeat(sym[:, :, :, None, None, None], niv_pp, axis=-1)
    if channel == "sing":
        gap[..., :niv_pp] = gap[..., niv_pp:]
    else:
        gap[..., :niv_pp] = -gap[..., niv_pp:]
    return gap


def symmetrise_gap(gap, irrk_ind, irrk_inv):
    """gap[k] = gap[irrk_ind][irrk_inv] (eliashberg_solver.py:408-410)."""
    nk = gap.shape[:3]
    flat = gap.reshape(int(np.prod(nk)), *gap.shape[3:])
    return flat[irrk_ind][irrk_inv].reshape(gap.shape)
