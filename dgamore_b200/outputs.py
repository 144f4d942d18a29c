"""On-disk outputs of a nonlocal pass in the upstream's file conventions, and the restart readers that use them.

The upstream writes its results as ``.npy`` arrays named after the quantity (``LocalNPoint.save``,
``dgamore/local_n_point.py:296-303``), always in the half bosonic range (ω ≥ 0; the negative frequencies follow
from F(−ω) = conj(flip F(ω)), ``local_n_point.py:191-240``):

=============================================  ============================================  =====================
file                                           content                                       upstream
=============================================  ============================================  =====================
``sigma_dga_iteration_{N}.npy``                Σ(k, ν) [Nk, n, n, 2 niv] (compressed k)      nonlocal_sde.py:923-925
``chi_phys_q_{dens,magn}.npy``                 χ_r(q, ω) after λ [q, a, b, c, d, ω ≥ 0]       nonlocal_sde.py:321
``gchi0_q_rank_0.npy``                         χ0 [q, a, b, c, d, ω ≥ 0, ν_full]             nonlocal_sde.py:812
``mu_history.npy``                             μ per iteration                               nonlocal_sde.py:973
eliashberg: ``vrg_q_{ch}_rank_0.npy``          γ_r [q, a, b, c, d, ω ≥ 0, ν]                  nonlocal_sde.py:292-295
eliashberg: ``gchi_aux_q_{ch}_sum_rank_0.npy``  χ_r(q, ω) (the same array as chi_phys_q)       nonlocal_sde.py:330-334
eliashberg: ``gchi0_q_inv_rank_0.npy``         χ0⁻¹ in the core box [q, a, b, c, d, ω ≥ 0, ν]  nonlocal_sde.py:833
=============================================  ============================================  =====================

The output folder is ``LDGA_Nk{Nk}_Nq{Nq}_wc{niw}_vc{niv}_vs{shell}`` made unique by a numeric suffix
(``dga_io.py:19-31, 101-107``).  A later run restarts from the highest ``sigma_dga_iteration_{N}.npy`` of a
folder (``get_starting_sigma``, ``nonlocal_sde.py:676-696``) and its Pulay mixing reads the last n of them from
the output folder and a previous run's folder (``read_last_n_sigmas``, ``nonlocal_sde.py:699-716``).

Everything here is host-side numpy on arrays copied from the device after a pass; nothing is computed.
"""

from __future__ import annotations

import glob
import os
import re

import numpy as np

_SIGMA_RE = re.compile(r"sigma_dga_iteration_(\d+)\.npy$")
CHANNELS = ("dens", "magn")


def output_dir_name(nk_tot: int, nq_tot: int, niw_core: int, niv_core: int, niv_shell: int) -> str:
    """The upstream's output folder name (dga_io.py:101-107)."""
    return f"LDGA_Nk{nk_tot}_Nq{nq_tot}_wc{niw_core}_vc{niv_core}_vs{niv_shell}"


def uniquify_path(path: str) -> str:
    """``path``, or ``path_1``, ``path_2`` ... (before the extension) if it exists (dga_io.py:19-31)."""
    stem, ext = os.path.splitext(path)
    counter = 1
    while os.path.exists(path):
        path = f"{stem}_{counter}{ext}"
        counter += 1
    return path


def half_niw(mat: np.ndarray, num_wn: int, num_vn: int) -> np.ndarray:
    """Full bosonic range [-niw, niw] -> ω ≥ 0 on the first frequency axis (local_n_point.py:227-240)."""
    if num_wn == 0:
        return mat
    axis = mat.ndim - (num_wn + num_vn)
    n = mat.shape[axis]
    return np.take(mat, np.arange(n // 2, n), axis=axis)


def full_niw(mat: np.ndarray, num_wn: int, num_vn: int) -> np.ndarray:
    """ω ≥ 0 -> the full range, F(−ω) = conj(F(ω) flipped along every frequency axis) (local_n_point.py:191-225)."""
    if num_wn == 0:
        return mat
    axis = mat.ndim - (num_wn + num_vn)
    freq_axes = tuple(range(axis, mat.ndim))
    n = mat.shape[axis]
    neg = np.take(mat, np.arange(1, n), axis=axis)
    neg = np.conj(np.flip(neg, axis=freq_axes))
    return np.concatenate([neg, mat], axis=axis)


def save_npoint(mat: np.ndarray, output_dir: str, name: str, num_wn: int = 0, num_vn: int = 0,
                full_niw_range: bool = False) -> str:
    """``np.save(output_dir/name.npy)`` in the half bosonic range, as ``LocalNPoint.save`` (local_n_point.py:296-303)."""
    if full_niw_range:
        mat = half_niw(mat, num_wn, num_vn)
    path = os.path.join(output_dir, f"{name}.npy")
    np.save(path, np.ascontiguousarray(mat), allow_pickle=False)
    return path


def save_sigma_iteration(sigma: np.ndarray, output_dir: str, iteration: int) -> str:
    """Σ [Nk, n, n, 2 niv] as ``sigma_dga_iteration_{iteration}.npy`` (nonlocal_sde.py:923-925)."""
    return save_npoint(sigma, output_dir, f"sigma_dga_iteration_{iteration}")


def _sigma_files(*dirs: str) -> list[tuple[int, str]]:
    found = []
    for d in dirs:
        if d and os.path.exists(d):
            for f in glob.glob(os.path.join(d, "sigma_dga_iteration_*.npy")):
                m = _SIGMA_RE.search(f)
                if m:
                    found.append((int(m.group(1)), f))
    return sorted(found, key=lambda x: x[0])


def get_starting_sigma(output_path: str, default_sigma: np.ndarray) -> tuple[np.ndarray, int]:
    """The highest-numbered Σ of a previous run's folder and its iteration, or (default_sigma, 0) when the folder
    is unset, missing or holds none (nonlocal_sde.py:676-696)."""
    if not output_path or not os.path.exists(output_path):
        return default_sigma, 0
    files = _sigma_files(output_path)
    if not files:
        return default_sigma, 0
    it = files[-1][0]
    return np.load(os.path.join(output_path, f"sigma_dga_iteration_{it}.npy")), it


def read_last_n_sigmas(n: int, output_path: str = "./", previous_sc_path: str = "./") -> list[np.ndarray]:
    """The last n Σ by iteration number over the output folder and a previous run's folder
    (nonlocal_sde.py:699-716)."""
    files = _sigma_files(output_path, previous_sc_path if previous_sc_path else "")
    return [np.load(f) for _, f in files[-n:]]


def save_pass(lp, output_dir: str, iteration: int, eliashberg_dir: str | None = None,
              mu_history: list[float] | None = None) -> list[str]:
    """Writes the files the upstream's pass writes from a LadderPass after ``run()``: Σ of this iteration and
    χ_phys of both channels in ``output_dir``; χ0 when the pass kept it; with ``eliashberg_dir`` the Eliashberg
    hand-off (γ when kept, χ_r, χ0⁻¹); ``mu_history.npy`` when given.  Returns the paths written."""
    import torch

    torch.cuda.synchronize()
    os.makedirs(output_dir, exist_ok=True)
    written = [save_sigma_iteration(lp.sigma.cpu().numpy(), output_dir, iteration)]
    chi_r = lp.chi_lam if getattr(lp, "do_lambda", False) else lp.chi_phys
    for ch, name in enumerate(CHANNELS):
        written.append(save_npoint(lp.chi_phys_ref_layout(chi_r, ch), output_dir, f"chi_phys_q_{name}"))
    if getattr(lp, "chi0", None) is not None:
        written.append(save_npoint(lp.chi0_ref_layout(), output_dir, "gchi0_q_rank_0"))
    if eliashberg_dir is not None:
        os.makedirs(eliashberg_dir, exist_ok=True)
        for ch, name in enumerate(CHANNELS):
            if getattr(lp, "gamma3", None) is not None:
                written.append(save_npoint(lp.orbmat_ref_layout(lp.gamma3[ch]), eliashberg_dir,
                                           f"vrg_q_{name}_rank_0"))
            written.append(save_npoint(lp.chi_phys_ref_layout(chi_r, ch), eliashberg_dir,
                                       f"gchi_aux_q_{name}_sum_rank_0"))
        written.append(save_npoint(lp.orbmat_ref_layout(lp.chi0_inv), eliashberg_dir, "gchi0_q_inv_rank_0"))
    if mu_history is not None:
        path = os.path.join(output_dir, "mu_history.npy")
        np.save(path, np.asarray(mu_history, dtype=np.float64), allow_pickle=False)
        written.append(path)
    return written
