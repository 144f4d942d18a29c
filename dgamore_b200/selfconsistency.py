"""Self-consistency glue of the ladder loop: the lattice Green's function, filling and occupations, the
chemical-potential search, the self-energy's tail moments and the mixing of successive self-energies.

The per-(k, ν) work — an n×n inverse for every momentum and frequency — runs on the device
(``csrc/glue.cu``: ``dga_g_full_c128``, ``dga_fill_sums_c128``, ``dga_sigma_kmean_c128``); what is left per step
is host logic on n×n matrices and short vectors, as in the upstream:

=====================================  =====================================================================
function                               upstream
=====================================  =====================================================================
``g_full``                             ``GreensFunction.get_g_full`` (dgamore/greens_function.py:110-124)
``total_fill`` / ``update_mu``         ``get_total_fill``, ``root_fun``, ``update_mu`` (greens_function.py:20-82)
``fill_nonlocal``                      ``GreensFunction.get_fill_nonlocal`` (greens_function.py:212-240)
``fit_smom``                           ``SelfEnergy.fit_smom`` (self_energy.py:51-75)
``apply_mixing``                       ``apply_mixing_strategy`` (nonlocal_sde.py:979-1151): linear, Pulay, Anderson
=====================================  =====================================================================

Layouts: Σ and G [Nk][n][n][2 niv] complex128 (compressed k, ν = (2m+1)π/β, m = −niv .. niv−1), e_k
[Nk][n][n] complex128 (the upstream's [kx, ky, kz, n, n] flattened), on the device as torch tensors.

``update_mu`` finds the root of total_fill(μ) − target with the secant method that
``scipy.optimize.newton`` uses when no derivative is given (start μ0 and μ0·(1 + 1e-4) ± 1e-4, step to the root
of the line through the last two points, stop when a step is below tol, at most maxiter steps; returns NaN
where the upstream's search raises), so that the μ it returns is the upstream's.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call
from .outputs import read_last_n_sigmas

C128 = torch.complex128


def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _s() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def vn(niv: int, beta: float) -> np.ndarray:
    """Fermionic Matsubara frequencies ν_m = (2m+1)π/β, m = −niv .. niv−1 (matsubara_frequencies.py)."""
    return (2 * np.arange(-niv, niv) + 1) * np.pi / beta


def _shape(sigma: torch.Tensor) -> tuple[int, int, int]:
    nk, n, _, nv = sigma.shape
    return nk, n, nv // 2


def g_full(sigma: torch.Tensor, ek: torch.Tensor, mu: float, beta: float) -> torch.Tensor:
    """G(k, ν) = [iν + μ − e_k − Σ(k, ν)]⁻¹ for every (k, ν) on the device."""
    nk, n, niv = _shape(sigma)
    g = torch.empty_like(sigma)
    call("dga_g_full_c128", _p(sigma), _p(ek), n, nk, niv, float(mu), float(beta), _p(g), _s())
    return g


def fit_smom(sigma: torch.Tensor, beta: float) -> tuple[np.ndarray, np.ndarray]:
    """The first two tail moments of Σ from its k-average over the last max(4, ⌊0.2 niv⌋) positive frequencies:
    mom0 = mean Re Σ, mom1 = mean Im Σ·ν (self_energy.py:51-75)."""
    nk, n, niv = _shape(sigma)
    n_fit = max(4, int(0.2 * niv))
    out = torch.empty((n, n, n_fit), dtype=C128, device=sigma.device)
    call("dga_sigma_kmean_c128", _p(sigma), n, nk, 2 * niv, 2 * niv - n_fit, n_fit, _p(out), _s())
    fitdata = out.cpu().numpy()
    nu = vn(niv, beta)[2 * niv - n_fit:]
    return np.mean(fitdata.real, axis=-1), np.mean(fitdata.imag * nu[None, None, :], axis=-1)


def _rho(h: np.ndarray) -> np.ndarray:
    """Fermi function of β(h − μ) through its eigen-decomposition, evaluated without overflow
    (greens_function.py:41-49, 222-229); h: [..., n, n] (already β(h − μ))."""
    eigenvals, eigenvecs = np.linalg.eig(h)
    rho_diag = np.empty_like(eigenvals)
    mask = eigenvals > 0
    rho_diag[mask] = np.exp(-eigenvals[mask]) / (1 + np.exp(-eigenvals[mask]))
    rho_diag[~mask] = 1 / (1 + np.exp(eigenvals[~mask]))
    n = h.shape[-1]
    rho_diag = np.einsum("...i,ij->...ij", rho_diag, np.eye(n))
    return eigenvecs @ rho_diag @ np.linalg.inv(eigenvecs)


def _sums(sigma: torch.Tensor, ek: torch.Tensor, mu: float, beta: float, smom0: np.ndarray):
    nk, n, niv = _shape(sigma)
    s0 = torch.as_tensor(np.ascontiguousarray(np.real(smom0), dtype=np.float64), device=sigma.device)
    s_k = torch.empty((nk, n, n), dtype=torch.float64, device=sigma.device)
    t_k = torch.empty_like(s_k)
    call("dga_fill_sums_c128", _p(sigma), _p(ek), _p(s0), n, nk, niv, float(mu), float(beta), _p(s_k), _p(t_k), _s())
    return s_k, t_k


def total_fill(mu: float, ek: torch.Tensor, sigma: torch.Tensor, beta: float, smom0: np.ndarray,
               hloc: np.ndarray | None = None) -> float:
    """Total filling 2 tr[ρ_loc + Σ_ν Re(G_loc(ν) − G_model(ν))/β] with G_model = [iν + μ − h_loc − s0]⁻¹ and
    ρ_loc the Fermi function of β(Re h_loc + s0 − μ) (greens_function.py:20-52)."""
    nk, n, niv = _shape(sigma)
    if hloc is None:
        hloc = ek.mean(dim=0).cpu().numpy()
    s_k, _ = _sums(sigma, ek, mu, beta, smom0)
    g_loc_sum = s_k.mean(dim=0).cpu().numpy()
    eye = np.eye(n)
    iv = 1j * vn(niv, beta)
    mat = iv[:, None, None] * eye[None] + mu * eye[None] - hloc[None] - smom0[None]
    g_model_sum = np.sum(np.linalg.inv(mat).real, axis=0)
    rho_loc = _rho(beta * (hloc.real + smom0 - mu * eye))
    occ = rho_loc + (g_loc_sum - g_model_sum) / beta
    return 2.0 * np.trace(occ).real


def _secant(f, x0: float, tol: float = 1e-6, maxiter: int = 50) -> float:
    """Secant root search as scipy.optimize.newton without fprime (published algorithm; rtol 0)."""
    p0 = x0
    eps = 1e-4
    p1 = x0 * (1 + eps) + (eps if x0 >= 0 else -eps)
    q0, q1 = f(p0), f(p1)
    if abs(q1) < abs(q0):
        p0, p1, q0, q1 = p1, p0, q1, q0
    for _ in range(maxiter):
        if q1 == q0:
            return (p1 + p0) / 2.0
        if abs(q1) > abs(q0):
            p = (-q0 / q1 * p1 + p0) / (1 - q0 / q1)
        else:
            p = (-q1 / q0 * p0 + p1) / (1 - q1 / q0)
        if abs(p - p1) <= tol:
            return p
        p0, q0 = p1, q1
        p1 = p
        q1 = f(p1)
    raise RuntimeError("secant search did not converge")


def update_mu(mu0: float, target_filling: float, ek: torch.Tensor, sigma: torch.Tensor, beta: float,
              smom0: np.ndarray) -> float:
    """μ with total_fill(μ) = target_filling (greens_function.py:63-82); NaN where the search fails."""
    hloc = ek.mean(dim=0).cpu().numpy()
    try:
        mu = _secant(lambda m: total_fill(m, ek, sigma, beta, smom0, hloc) - target_filling, mu0, tol=1e-6)
    except RuntimeError:
        return np.nan
    return float(np.real(mu))


def fill_nonlocal(sigma: torch.Tensor, ek: torch.Tensor, mu: float, beta: float,
                  smom0: np.ndarray) -> tuple[float, np.ndarray, np.ndarray]:
    """(n, occ [n][n], occ_k [Nk][n][n]): occ_k = ρ_k + Σ_ν Re(G(k, ν) − G_model(k, ν))/β with
    G_model(k) = [iν + μ − e_k − s0]⁻¹ and ρ_k the Fermi function of β(Re e_k + s0 − μ)
    (greens_function.py:212-240)."""
    nk, n, niv = _shape(sigma)
    s_k, t_k = _sums(sigma, ek, mu, beta, smom0)
    ek_h = ek.cpu().numpy()
    rho_k = _rho(beta * (ek_h.real + smom0[None] - mu * np.eye(n)[None]))
    occ_k = rho_k + (s_k - t_k).cpu().numpy() / beta
    occ_k.real[np.abs(occ_k) < 1e-12] = 0.0
    occ_mean = np.mean(occ_k, axis=0)
    occ_mean.real[np.abs(occ_mean) < 1e-12] = 0.0
    return 2.0 * np.trace(occ_mean).real, occ_mean, occ_k


def apply_mixing(strategy: str, sigma_new: np.ndarray, sigma_old: np.ndarray, sigma_dmft: np.ndarray,
                 current_iter: int, n_hist: int, alpha: float, niv_core: int, output_path: str,
                 previous_sc_path: str = "") -> np.ndarray:
    """The next self-energy from this iteration's result (nonlocal_sde.py:979-1151): linear mixing
    α Σ_new + (1 − α) Σ_old, or, once current_iter > n_hist, Pulay or Anderson extrapolation over the last n_hist
    self-energies written by earlier iterations (``sigma_dga_iteration_{N}.npy``) inside the core frequency
    window.  Arrays [Nk][n][n][2 niv]; sigma_dmft [1][n][n][2 niv] or [n][n][2 niv]."""
    s = strategy.lower()
    if s in ("pulay", "anderson") and current_iter > n_hist:
        last = read_last_n_sigmas(n_hist, output_path, previous_sc_path)
        dmft = np.asarray(sigma_dmft).reshape(1, *sigma_new.shape[1:])
        dmft_stacked = np.tile(dmft, (sigma_new.shape[0], 1, 1, 1))
        niv = sigma_new.shape[-1] // 2
        sl = slice(niv - niv_core, niv + niv_core)
        proposals = [x[..., sl] for x in [dmft_stacked] + last]
        results = [x[..., sl] for x in last + [sigma_new]]
        shape = results[-1].shape
        n_total = int(np.prod(shape))
        flat = lambda x: x.reshape(-1)
        ri = lambda z: np.concatenate([z.real, z.imag])
        if s == "pulay":
            r_matrix = np.zeros((2 * n_total, n_hist))
            f_matrix = np.zeros_like(r_matrix)
            for i in range(n_hist):
                pd = flat(proposals[-1 - i]) - flat(proposals[-2 - i])
                r_matrix[:, i] = ri(pd)
                rd = flat(results[-1 - i]) - flat(results[-2 - i])
                f_matrix[:, i] = ri(rd) - r_matrix[:, i]
            f_i = ri(flat(results[-1]) - flat(proposals[-1]))
            norm_f = np.linalg.norm(f_i)
            u, sv, vh = np.linalg.svd(f_matrix, full_matrices=False)
            cutoff = 1e-5 * (sv[0] if sv.size else 1.0)
            mask = sv > cutoff
            if not np.any(mask):
                return alpha * sigma_new + (1 - alpha) * sigma_old
            coeffs = vh[mask].T @ ((u[:, mask].T @ f_i) / sv[mask])
            update = alpha * f_i - (r_matrix + alpha * f_matrix) @ coeffs
            norm_u = np.linalg.norm(update)
            if norm_f > 0 and norm_u > 10.0 * norm_f:
                update *= 10.0 * norm_f / norm_u
            update = update[:n_total] + 1j * update[n_total:]
            out = sigma_new.copy()
            out[..., sl] = flat(proposals[-1]).reshape(shape) + update.reshape(shape)
            return out
        # Anderson
        f_curr = flat(results[-1]) - flat(proposals[-1])
        f_vec = ri(f_curr)
        norm_f = np.linalg.norm(f_vec)
        dx_cols, df_cols = [], []
        for i in range(n_hist):
            dx_cols.append(ri(flat(proposals[-1 - i]) - flat(proposals[-2 - i])))
            df_i = flat(results[-1 - i]) - flat(proposals[-1 - i])
            df_im1 = flat(results[-2 - i]) - flat(proposals[-2 - i])
            df_cols.append(ri(df_i - df_im1))
        dx_matrix = np.column_stack(dx_cols)
        df_matrix = np.column_stack(df_cols)
        try:
            u, sv, vh = np.linalg.svd(df_matrix, full_matrices=False)
            cutoff = 1e-5 * (sv[0] if len(sv) > 0 else 1.0)
            mask = sv > cutoff
            if not np.any(mask):
                raise np.linalg.LinAlgError("all singular values below the cutoff")
            s_reg = sv[mask] / (sv[mask] ** 2 + cutoff**2)
            coeffs = vh[mask].T @ (s_reg * (u[:, mask].T @ f_vec))
        except np.linalg.LinAlgError:
            return alpha * sigma_new + (1 - alpha) * sigma_old
        x_n = flat(proposals[-1])
        x_and = ri(x_n) + f_vec - (dx_matrix + df_matrix) @ coeffs
        x_and = x_and[:n_total] + 1j * x_and[n_total:]
        candidate = (1 - alpha) * x_n + alpha * x_and.reshape(-1)
        update = candidate - x_n
        norm_u = np.linalg.norm(update)
        if norm_f > 0 and norm_u > 3.0 * norm_f:
            candidate = x_n + update * (3.0 * norm_f / norm_u)
        out = sigma_new.copy()
        out[..., sl] = candidate.reshape(shape)
        return out
    return alpha * sigma_new + (1 - alpha) * sigma_old
