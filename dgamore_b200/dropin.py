"""Drop-in replacements for the upstream hot-path entry points, with the upstream's Python signatures.

``install()`` patches them into the imported upstream ``dgamore`` package (module attributes and class methods,
which is how the upstream itself calls them), so ``nonlocal_sde.calculate_self_energy_q`` and
``eliashberg_solver.solve`` run unchanged with the libdga_b200 kernels underneath; ``uninstall()`` restores the
originals.  The functions can also be called directly.

=================================================  ==================================================
upstream entry point                               device path
=================================================  ==================================================
BubbleGenerator.create_generalized_chi0_q_fft_auto  G(k) -> G(R) plane DFTs, bubble kernel
  (dgamore/bubble_gen.py:117-144)
BubbleGenerator.create_generalized_chi0_q_auto      the same kernels evaluated on an explicit q list
  (bubble_gen.py:225-253)
BubbleGenerator.create_generalized_chi0_q_pp_w0     dga_eli_chi0pp_c128
  (bubble_gen.py:268-279)
FourPoint.invert_and_sum_over_last_vn(_v2)          dga_invert_sum_dense_c128 (four_point.invert_and_sum...)
  (four_point.py:620-684)
nonlocal_sde.create_auxiliary_chi_r_q_sum_v1/v2/v3  structured BSE (dga_bse_solve_sum_c128 or the mixed form)
  (nonlocal_sde.py:85-156)                          from Gamma_r, chi0^-1, U_r + V_r^q: no [q,w,nu,nu'] array
nonlocal_sde.calculate_sigma_from_kernel_fft_auto   dga_sigma_rspace_c128 (R-space, nu >= 0)
  (nonlocal_sde.py:650-674)
nonlocal_sde.calculate_sigma_from_kernel_auto       dga_sigma_c128 on the full-zone kernel
  (nonlocal_sde.py:517-541)
nonlocal_sde.get_hartree_fock (nonlocal_sde.py:31-69)  dga_hartree_fock_c128
lambda_correction.find_lambda,                      dga_lambda_c128
  perform_single_lambda_correction (:28-73)
eliashberg_solver.solve_eliashberg_lanczos (:376-471)  device gap-equation matvec + Krylov-Schur
local_sde.perform_local_schwinger_dyson             local_sde.LocalSde: local bubble, batched dense LU,
  (local_sde.py:175-217)                            the BSE at q = 0, local Sigma kernels
=================================================  ==================================================

Arguments are the upstream's objects, duck-typed: a function reads only ``.mat`` and the metadata the original
reads (``.channel``, ``.niv``, ``.num_vn_dimensions``, the ``to_half_niw_range`` / ``compress_q_dimension``
layout methods where the original calls them) and the ``config`` values the original reads (``config.sys.beta``,
``config.lattice.q_grid``, ``config.box.niv_core`` ...).  ``install`` records the upstream ``config`` module and
result classes; ``use_config`` / ``use_classes`` set them for direct calls without the upstream package, in which
case results are ``Result`` records carrying the same ``.mat`` and constructor arguments.  Errors mirror the
originals: ``NotImplementedError`` for a FourPoint without two fermionic dimensions, ``numpy.linalg.LinAlgError``
for an exactly singular matrix; the library's own failures raise ``DgaError``.

Scope: one process and one GPU, as the device schedule has no inter-rank exchange.  The distributors the upstream
passes are used only as it uses them with one rank (``scatter`` of the bubble is applied when present); a
``my_full_q_list`` that is not the whole zone in row-major order is rejected.
"""

from __future__ import annotations

import ctypes
import types

import numpy as np
import torch

from . import four_point as _fp
from ._lib import call, lib, ll_array
from .eliashberg_solver import initial_gap, krylov_schur
from .pipeline import compound_orb, twiddles

C128 = torch.complex128

_state = {"config": None, "classes": {}, "precision": "fp64", "patched": []}


# ------------------------------------------------------------------------------------------------
# configuration, result classes, precision
# ------------------------------------------------------------------------------------------------
class Result:
    """Stand-in for an upstream n-point object when the upstream classes are not registered: ``.mat`` plus the
    constructor arguments the upstream would have received (``kind``, ``args``, ``kwargs``)."""

    def __init__(self, kind: str, mat, *args, **kwargs):
        self.kind, self.mat, self.args, self.kwargs = kind, mat, args, kwargs
        self.channel = kwargs.get("channel", args[0] if args else None)

    def filter_small_values(self, threshold: float = 1e-12):
        self.mat[(np.abs(self.mat.real) < threshold) & (np.abs(self.mat.imag) < threshold)] = 0.0
        return self


def use_config(config) -> None:
    """Sets the configuration object the drop-ins read (the upstream's ``dgamore.config`` module, or any
    namespace with the same ``sys`` / ``lattice`` / ``box`` / ``eliashberg`` attributes)."""
    _state["config"] = config


def use_classes(**classes) -> None:
    """Registers result classes by upstream name (FourPoint, SelfEnergy, GapFunction, SpinChannel,
    FrequencyNotation)."""
    _state["classes"].update(classes)


def set_precision(precision: str) -> None:
    """'fp64' (the drop-in form, parity with the upstream to 1e-10) or 'mixed' (complex64 LU on the tensor cores
    with FP64 refinement) for the structured BSE."""
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    _state["precision"] = precision


def _cfg():
    cfg = _state["config"]
    if cfg is None:
        raise RuntimeError("no configuration: call dropin.install() or dropin.use_config(config) first")
    return cfg


def _make(kind: str, mat, *args, **kwargs):
    cls = _state["classes"].get(kind)
    return cls(mat, *args, **kwargs) if cls is not None else Result(kind, mat, *args, **kwargs)


def _enum(kind: str, name: str):
    cls = _state["classes"].get(kind)
    return getattr(cls, name) if cls is not None else name.lower()


def _channel_name(channel) -> str:
    return str(getattr(channel, "value", channel)).lower()


# ------------------------------------------------------------------------------------------------
# device helpers
# ------------------------------------------------------------------------------------------------
def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _s() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(x, dtype=C128) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128 if dtype == C128 else None)).to("cuda")


def _g_k(giwk) -> tuple[torch.Tensor, int, tuple, int]:
    """G(k, nu) of a GreensFunction as [Nk][n][n][2 niv] on the device, with niv, the grid and n_bands."""
    mat = np.asarray(giwk.mat)
    nk = tuple(int(x) for x in mat.shape[:3])
    n = mat.shape[3]
    g = _dev(mat.reshape(int(np.prod(nk)), n, n, mat.shape[-1]))
    return g, mat.shape[-1] // 2, nk, n


def _g_r(g_k: torch.Tensor, niv_g: int, nu_first: int, n_slots: int, nk: tuple, n: int) -> torch.Tensor:
    """out[t][a][b][R] = sum_k G(k)[a][b][nu_first + t] e^{-ikR} (n_point_base.py:509-529)."""
    nk_tot = int(np.prod(nk))
    nvg2 = 2 * niv_g
    if niv_g + nu_first < 0 or niv_g + nu_first + n_slots > nvg2:
        raise ValueError("the Green's function does not hold the fermionic frequencies this stage needs")
    out = torch.empty((n_slots, n, n, nk_tot), dtype=C128, device="cuda")
    base = g_k[..., niv_g + nu_first:]
    tw = _dev(twiddles(nk, -1))
    call("dga_dft_planes_c128", _p(base), 1, nvg2, n * n * nvg2, _p(out), n * n * nk_tot, nk_tot, 1, n * n,
         n_slots * n * n, nk[0], nk[1], nk[2], _p(tw), 1.0, _s())
    return out


def _bubble(giwk, niw: int, niv: int, q_list: np.ndarray, nk: tuple, beta: float) -> np.ndarray:
    """chi0[q, a, b, c, d, w >= 0, nu] = -beta/Nk sum_k G_ad(k, nu) G_cb(k - q, nu - w), filtered at 1e-12."""
    g_k, niv_g, g_nk, n = _g_k(giwk)
    if tuple(g_nk) != tuple(nk):
        raise ValueError(f"momentum grids differ: G on {g_nk}, bubble on {tuple(nk)}")
    g_r = _g_r(g_k, niv_g, -niv - niw, 2 * niv + niw, nk, n)
    q = torch.from_numpy(np.ascontiguousarray(np.asarray(q_list).reshape(-1, 3), dtype=np.int32)).to("cuda")
    Q, W, nv = q.shape[0], niw + 1, 2 * niv
    out = torch.empty((Q, n, n, n, n, W, nv), dtype=C128, device="cuda")
    strides = [n**4 * W * nv, nv, 1, n**3 * W * nv, n**2 * W * nv, n * W * nv, W * nv]  # q w nu a b c d
    tw_inv = _dev(twiddles(nk, +1))
    call("dga_bubble_c128", _p(g_r), n, niv, niw, nk[0], nk[1], nk[2], _p(q), Q, _p(tw_inv), float(beta), _p(out),
         ll_array(strides), _s())
    return out.cpu().numpy()


# ------------------------------------------------------------------------------------------------
# bubble_gen
# ------------------------------------------------------------------------------------------------
def create_generalized_chi0_q_fft_auto(mpi_dist_irrk, giwk, niw: int, niv: int, k_grid, beta: float, logger=None):
    """BubbleGenerator.create_generalized_chi0_q_fft_auto (bubble_gen.py:117-144): chi0 on the irreducible q of
    ``k_grid``, half bosonic range, compressed q."""
    nk = tuple(int(x) for x in k_grid.nk)
    q_list = np.array(np.unravel_index(np.asarray(k_grid.irrk_ind), nk)).T
    mat = _bubble(giwk, int(niw), int(niv), q_list, nk, beta)
    if mpi_dist_irrk is not None and hasattr(mpi_dist_irrk, "scatter"):
        mat = mpi_dist_irrk.scatter(mat)
    return _make("FourPoint", mat, _enum("SpinChannel", "NONE"), k_grid.nk, 1, 1, full_niw_range=False,
                 has_compressed_q_dimension=True)


def create_generalized_chi0_q_auto(mpi_distributor, giwk, niw: int, niv: int, q_list, q_grid, beta: float,
                                   logger=None):
    """BubbleGenerator.create_generalized_chi0_q_auto (bubble_gen.py:225-253): chi0 for an explicit list of q
    points (integer grid coordinates), half bosonic range, compressed q."""
    nk = tuple(int(x) for x in q_grid.nk)
    mat = _bubble(giwk, int(niw), int(niv), np.asarray(q_list), nk, beta)
    return _make("FourPoint", mat, _enum("SpinChannel", "NONE"), q_grid.nk, 1, 1, full_niw_range=False,
                 has_compressed_q_dimension=True)


def create_generalized_chi0_q_pp_w0(giwk, niv_pp: int, q_grid):
    """BubbleGenerator.create_generalized_chi0_q_pp_w0 (bubble_gen.py:268-279):
    chi0pp[k, a, b, c, d, nu] = G_ad(k, nu) conj(G_cb(k, nu)) (no factor -beta), PP notation."""
    g_k, niv_g, nk, n = _g_k(giwk)
    nk_tot, P, n2 = int(np.prod(nk)), int(niv_pp), n * n
    if P > niv_g:
        raise ValueError("niv_pp exceeds the Green's function's frequency box")
    out = torch.empty((nk_tot, 2 * P, n2, n2), dtype=C128, device="cuda")
    call("dga_eli_chi0pp_c128", _p(g_k), n, niv_g, P, nk_tot, _p(out), _s())
    mat = out.cpu().numpy().reshape(nk_tot, 2 * P, n, n, n, n).transpose(0, 2, 3, 4, 5, 1)
    mat = np.ascontiguousarray(mat)
    return _make("FourPoint", mat, _enum("SpinChannel", "NONE"), q_grid.nk, 0, 1, True, True, True,
                 _enum("FrequencyNotation", "PP")).filter_small_values()


# ------------------------------------------------------------------------------------------------
# four_point
# ------------------------------------------------------------------------------------------------
def invert_and_sum_over_last_vn(self, beta: float):
    """FourPoint.invert_and_sum_over_last_vn / _v2 (four_point.py:620-684): mutates and returns ``self`` with
    mat = sum_nu' [A^-1] / beta and one fermionic dimension."""
    if self.num_vn_dimensions != 2:
        raise NotImplementedError("Method only implemented for objects with two fermionic frequency dimensions.")
    if hasattr(self, "to_half_niw_range"):
        self.to_half_niw_range()
    if hasattr(self, "compress_q_dimension"):
        self.compress_q_dimension()
    self.mat = _fp.invert_and_sum_over_last_vn(np.asarray(self.mat), beta)
    self._num_vn_dimensions = 1
    if hasattr(self, "update_original_shape"):
        self.update_original_shape()
    return self


# ------------------------------------------------------------------------------------------------
# nonlocal_sde: structured BSE, Sigma, Hartree-Fock
# ------------------------------------------------------------------------------------------------
def _bse_structured(gamma, chi0_inv, uv, beta: float, precision: str) -> np.ndarray:
    """sum_nu' [chi0^-1 + (Gamma - U - V)/beta^2]^-1 / beta for one channel.  gamma [n,n,n,n,W,nv,nv] (half w
    range), chi0_inv [Q,n,n,n,n,W,nv], uv [Q,n,n,n,n] (U_r + V_r^q); returns [Q,n,n,n,n,W,nv]."""
    n, W, nv, Q = gamma.shape[0], gamma.shape[4], gamma.shape[5], chi0_inv.shape[0]
    n2, niv, N = n * n, nv // 2, n * n * nv
    if chi0_inv.shape[1:] != (n, n, n, n, W, nv) or uv.shape != (Q, n, n, n, n):
        raise ValueError(f"inconsistent shapes: Gamma {gamma.shape}, chi0^-1 {chi0_inv.shape}, U+V {uv.shape}")
    g = _dev(gamma)
    gamma_cm = torch.empty((1, W, N, N), dtype=C128, device="cuda")
    call("dga_strided_copy_c128", _p(g), _p(gamma_cm), 7, ll_array(g.shape), ll_array(list(g.stride())),
         ll_array([n * nv, nv, nv * N, n * nv * N, N * N, 1, N]), 1.0, _s())
    c0 = _dev(np.asarray(chi0_inv).transpose(0, 5, 6, 1, 2, 4, 3).reshape(Q, W, nv, n2, n2))
    uvd = _dev(compound_orb(np.asarray(uv))[None])
    work = torch.tensor([(0, q, w) for w in range(W) for q in range(Q)], dtype=torch.int32, device="cuda")
    n_items = work.shape[0]
    out = torch.empty((1, Q, W, N, n2), dtype=C128, device="cuda")
    status = torch.zeros(n_items, dtype=torch.int32, device="cuda")
    inv_beta2 = 1.0 / beta**2
    L = lib()
    if precision == "mixed":
        iters = torch.zeros(n_items, dtype=torch.int32, device="cuda")
        sb = int(L.dga_bse_mixed_scratch_bytes(N, n2, n_items))
        scratch = torch.empty(sb // 16 + 1, dtype=C128, device="cuda")
        call("dga_bse_solve_sum_mixed_c128", n, niv, W, Q, 1, beta, inv_beta2, _p(gamma_cm), _p(c0), _p(uvd),
             _p(work), n_items, 6, 1e-10, _p(out), _p(status), _p(iters), _p(scratch), scratch.numel() * 16, _s())
        grid = min(n_items, 148)
        rs = torch.empty(grid * (N * N + N * n2) + 1, dtype=C128, device="cuda")
        call("dga_bse_resolve_fp64_c128", n, niv, W, Q, 1, beta, inv_beta2, _p(gamma_cm), _p(c0), _p(uvd), _p(work),
             n_items, _p(out), _p(status), grid, _p(rs), rs.numel() * 16, _s())
    else:
        sb = int(L.dga_bse_scratch_bytes(N, n2, n_items))
        scratch = torch.empty(sb // 16 + 1, dtype=C128, device="cuda")
        call("dga_bse_solve_sum_c128", n, niv, W, Q, 1, beta, inv_beta2, _p(gamma_cm), _p(c0), _p(uvd), _p(work),
             n_items, _p(out), _p(status), _p(scratch), scratch.numel() * 16, _s())
    st = status.cpu().numpy()
    if np.any(st & 1):
        raise np.linalg.LinAlgError("Singular matrix")
    if np.any(st):
        from ._lib import DgaError

        raise DgaError(f"BSE items flagged (status bits {int(np.bitwise_or.reduce(st))}): non-finite or unconverged")
    x = out[0].cpu().numpy().reshape(Q, W, n, n, nv, n, n)  # q w o1 o2 nu o4 o3
    return np.ascontiguousarray(x.transpose(0, 2, 3, 6, 5, 1, 4))


def _half_w(obj):
    if getattr(obj, "full_niw_range", False) and hasattr(obj, "to_half_niw_range"):
        obj = obj.to_half_niw_range()
    return obj


def create_auxiliary_chi_r_q_sum_v1(gamma_r, gchi0_q_inv, u_loc, v_nonloc):
    """nonlocal_sde.create_auxiliary_chi_r_q_sum_v1 (nonlocal_sde.py:85-96): sum_nu' chi*_r(q, w, nu, nu') of the
    channel of ``gamma_r`` for every q of ``gchi0_q_inv`` (half bosonic range, compressed q), solved on the
    device from the structured form -- the [q, w, nu, nu'] matrix the upstream broadcasts is never formed."""
    cfg = _cfg()
    ch = gamma_r.channel
    g = _half_w(gamma_r)
    c0 = _half_w(gchi0_q_inv)
    if hasattr(c0, "compress_q_dimension"):
        c0 = c0.compress_q_dimension()
    c0m = np.asarray(c0.mat)
    n = c0m.shape[1]
    Q = c0m.shape[0]
    u = np.asarray(u_loc.as_channel(ch).mat).reshape(n, n, n, n)
    v = np.asarray(v_nonloc.as_channel(ch).mat).reshape(-1, n, n, n, n)
    if v.shape[0] != Q:
        raise ValueError(f"V(q) holds {v.shape[0]} q points, chi0^-1 {Q}")
    x = _bse_structured(np.asarray(g.mat), c0m, u[None] + v, float(cfg.sys.beta), _state["precision"])
    return _make("FourPoint", x, ch, cfg.lattice.nq, 1, 1, False, has_compressed_q_dimension=True)


def create_auxiliary_chi_r_q_sum_v2(gamma_r, gchi0_q_inv, u_loc, v_nonloc, mpi_dist_irrq):
    """nonlocal_sde.create_auxiliary_chi_r_q_sum_v2 (nonlocal_sde.py:99-126): the same result per q."""
    return create_auxiliary_chi_r_q_sum_v1(gamma_r, gchi0_q_inv, u_loc, v_nonloc)


def create_auxiliary_chi_r_q_sum_v3(gamma_r, gchi0_q_inv, u_loc, v_nonloc, mpi_dist_irrq):
    """nonlocal_sde.create_auxiliary_chi_r_q_sum_v3 (nonlocal_sde.py:129-156): the same result per q."""
    return create_auxiliary_chi_r_q_sum_v1(gamma_r, gchi0_q_inv, u_loc, v_nonloc)


def _sigma_inputs(kernel, giwk, cfg):
    k = _half_w(kernel)
    if hasattr(k, "compress_q_dimension"):
        k = k.compress_q_dimension()
    km = np.asarray(k.mat)  # [q, a, i, j, d, w, nu]
    Q, n, W, nv = km.shape[0], km.shape[1], km.shape[5], km.shape[6]
    kd = _dev(km.transpose(0, 5, 6, 1, 2, 4, 3).reshape(Q, W, nv, n * n, n * n))
    g_k, niv_g, nk, gn = _g_k(giwk)
    niv, niw = nv // 2, W - 1
    g_r = _g_r(g_k, niv_g, -niw, niv + 2 * niw, nk, n)
    return kd, g_r, Q, n, niv, niw, nk


def calculate_sigma_from_kernel_fft_auto(mpi_distributor, kernel, giwk):
    """nonlocal_sde.calculate_sigma_from_kernel_fft_auto (nonlocal_sde.py:650-674): Sigma in R space for nu >= 0
    from the full-zone kernel, returned like the original (the caller applies ifft().to_full_niv_range())."""
    cfg = _cfg()
    kd, g_r, Q, n, niv, niw, nk = _sigma_inputs(kernel, giwk, cfg)
    nk_tot = int(np.prod(nk))
    if Q != nk_tot:
        raise ValueError(f"the kernel holds {Q} q points, not the full zone of {nk_tot}")
    gather = torch.arange(nk_tot, dtype=torch.int32, device="cuda")
    chunks = 1
    sb = int(lib().dga_sigma_scratch_bytes(n, niv, nk_tot, chunks))
    scratch = torch.empty(sb // 16 + 1, dtype=C128, device="cuda")
    out = torch.empty((niv, n * n, nk_tot), dtype=C128, device="cuda")
    tw_inv = _dev(twiddles(nk, +1))
    call("dga_sigma_rspace_c128", _p(kd), _p(g_r), n, niv, niw, Q, nk[0], nk[1], nk[2], _p(gather), _p(tw_inv),
         float(cfg.sys.beta), chunks, _p(out), _p(scratch), scratch.numel() * 16, _s())
    mat = np.ascontiguousarray(out.cpu().numpy().reshape(niv, n, n, nk_tot).transpose(3, 1, 2, 0))
    return _make("SelfEnergy", mat, cfg.lattice.nk, full_niv_range=False, has_compressed_q_dimension=True,
                 calc_smom=False)


def calculate_sigma_from_kernel_auto(mpi_distributor, kernel, giwk, my_full_q_list):
    """nonlocal_sde.calculate_sigma_from_kernel_auto (nonlocal_sde.py:517-541): Sigma(k, nu) over the full
    fermionic range from the full-zone kernel (the direct form; the same sums through real space here)."""
    cfg = _cfg()
    kd, g_r, Q, n, niv, niw, nk = _sigma_inputs(kernel, giwk, cfg)
    nk_tot = int(np.prod(nk))
    full = np.array(np.unravel_index(np.arange(nk_tot), nk)).T
    if Q != nk_tot or not np.array_equal(np.asarray(my_full_q_list).reshape(-1, 3), full):
        raise NotImplementedError("the device Sigma needs the whole q zone in row-major order on one rank")
    gather = torch.arange(nk_tot, dtype=torch.int32, device="cuda")
    chunks = 1
    sb = int(lib().dga_sigma_scratch_bytes(n, niv, nk_tot, chunks))
    scratch = torch.empty(sb // 16 + 1, dtype=C128, device="cuda")
    out = torch.empty((nk_tot, n, n, 2 * niv), dtype=C128, device="cuda")
    tw_inv = _dev(twiddles(nk, +1))
    call("dga_sigma_c128", _p(kd), _p(g_r), n, niv, niw, Q, nk[0], nk[1], nk[2], _p(gather), _p(tw_inv),
         float(cfg.sys.beta), chunks, _p(out), _p(scratch), scratch.numel() * 16, _s())
    return _make("SelfEnergy", out.cpu().numpy(), cfg.lattice.nk, True, True)


def get_hartree_fock(u_loc, v_nonloc, q_list):
    """nonlocal_sde.get_hartree_fock (nonlocal_sde.py:31-69): (hartree [1,n,n,1], fock [Nk,n,n,1]) from
    config.sys.occ and config.sys.occ_k, on the whole q zone in row-major order."""
    cfg = _cfg()
    nk = tuple(int(x) for x in cfg.lattice.nk)
    nk_tot = int(np.prod(nk))
    u = np.asarray(u_loc.mat)
    n = u.shape[0]
    full = np.array(np.unravel_index(np.arange(nk_tot), nk)).T
    if not np.array_equal(np.asarray(q_list).reshape(-1, 3), full):
        raise NotImplementedError("the device Fock term needs the whole q zone in row-major order on one rank")
    v = np.asarray(v_nonloc.mat).reshape(nk_tot, n, n, n, n)
    occ = np.asarray(cfg.sys.occ).reshape(n, n)
    occ_k = np.asarray(cfg.sys.occ_k).reshape(nk_tot, n, n)
    hartree = torch.empty((n, n), dtype=C128, device="cuda")
    fock = torch.empty((nk_tot, n, n), dtype=C128, device="cuda")
    ud, vd, od, okd = _dev(u), _dev(v.reshape(nk_tot, -1)), _dev(occ), _dev(occ_k)
    call("dga_hartree_fock_c128", _p(ud), _p(vd), _p(od), _p(okd), n, nk[0], nk[1], nk[2], _p(hartree), _p(fock),
         ctypes.c_void_p(0), 0, _s())
    return hartree.cpu().numpy()[None, ..., None], fock.cpu().numpy()[..., None]


# ------------------------------------------------------------------------------------------------
# lambda_correction
# ------------------------------------------------------------------------------------------------
def _lambda(chi_half: np.ndarray, target: complex, delta: float, eps: float, maxiter: int):
    cfg = _cfg()
    qg = cfg.lattice.q_grid
    chi = _dev(chi_half)
    Q, W = chi.shape
    weights = torch.as_tensor(np.asarray(qg.irrk_count, dtype=np.int64), device="cuda")
    tgt = torch.tensor([complex(target)], dtype=C128, device="cuda")
    lam = torch.zeros(1, dtype=torch.float64, device="cuda")
    its = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    chi_out = torch.empty_like(chi)
    call("dga_lambda_c128", _p(chi), Q, W, 1, _p(weights), _p(tgt), float(cfg.sys.beta), float(qg.nk_tot),
         float(delta), float(eps), int(maxiter), _p(lam), _p(its), _p(status), _p(chi_out), _s())
    return float(lam.item()), chi_out.cpu().numpy()


def find_lambda(chi_r_mat: np.ndarray, chi_r_loc_sum: complex, delta: float = 0.1, eps: float = 1e-7,
                maxiter: int = 1000) -> float:
    """lambda_correction.find_lambda (lambda_correction.py:28-60) for chi_r [q_irr, 2 niw + 1] over the full
    bosonic range, which the upstream passes with chi(-w) = conj chi(w): the device iteration reads the w >= 0
    half and returns the same lambda."""
    chi = np.asarray(chi_r_mat)
    niw = chi.shape[-1] // 2
    return _lambda(chi.reshape(-1, chi.shape[-1])[:, niw:], chi_r_loc_sum, delta, eps, maxiter)[0]


def perform_single_lambda_correction(chi_r, chi_r_loc_sum: complex):
    """lambda_correction.perform_single_lambda_correction (lambda_correction.py:63-73): returns (chi_r corrected,
    irreducible q, half bosonic range; lambda).  Like the original it works on ``chi_r`` itself."""
    if hasattr(chi_r, "to_full_niw_range"):
        chi_r = chi_r.to_full_niw_range()
    if hasattr(chi_r, "compress_q_dimension"):
        chi_r = chi_r.compress_q_dimension()
    full = np.asarray(chi_r.mat).reshape(np.asarray(chi_r.mat).shape[0], -1)
    niw = full.shape[-1] // 2
    lam, chi_half = _lambda(full[:, niw:], chi_r_loc_sum, 0.1, 1e-7, 1000)
    if hasattr(chi_r, "to_half_niw_range"):
        chi_r = chi_r.to_half_niw_range()
    chi_r.mat = chi_half[:, None, None, None, None, :]
    return chi_r, lam


# ------------------------------------------------------------------------------------------------
# local_sde
# ------------------------------------------------------------------------------------------------
def perform_local_schwinger_dyson(g_dmft, g2_dens, g2_magn, u_loc):
    """local_sde.perform_local_schwinger_dyson (local_sde.py:175-217) on the device (``local_sde.LocalSde``):
    returns gamma_d, gamma_m, chi_d, chi_m, vrg_d, vrg_m, f_d, f_m, gchi_d, gchi_m (LocalFourPoint, half w range)
    and sigma_loc (SelfEnergy), reading config.sys.beta / occ_dmft, config.box.niw_core / niv_core / niv_shell
    and, like the original, saving the local bubble as ``gchi0_loc`` when config.eliashberg.perform_eliashberg.
    Orbital symmetrisation (config.dmft.symmetrize_orbitals) raises NotImplementedError."""
    from .local_sde import LocalSde
    from .outputs import save_npoint

    cfg = _cfg()
    dmft = getattr(cfg, "dmft", None)
    if dmft is not None and len(getattr(dmft, "symmetrize_orbitals", []) or []) > 0:
        raise NotImplementedError("orbital symmetrisation of the local vertices is not part of the device form")
    box = cfg.box
    sde = LocalSde(np.asarray(g_dmft.mat), np.asarray(g2_dens.mat), np.asarray(g2_magn.mat), np.asarray(u_loc.mat),
                   cfg.sys.beta, box.niw_core, box.niv_core, box.niv_shell, cfg.sys.occ_dmft).run()
    res = sde.results()
    eli = getattr(cfg, "eliashberg", None)
    if eli is not None and getattr(eli, "perform_eliashberg", False):
        save_npoint(sde.bubble().cpu().numpy(), cfg.output.output_path, "gchi0_loc")
    dens, magn = _enum("SpinChannel", "DENS"), _enum("SpinChannel", "MAGN")
    n_vn = (2, 2, 0, 0, 1, 1, 2, 2, 2, 2)
    chans = (dens, magn) * 5
    four = [_make("LocalFourPoint", m, c, 1, nv, False) for m, c, nv in zip(res[:10], chans, n_vn)]
    return (*four, _make("SelfEnergy", res[10]))


# ------------------------------------------------------------------------------------------------
# eliashberg_solver
# ------------------------------------------------------------------------------------------------
class PairingOperator:
    """The linearised gap-equation operator of one channel on the device (eliashberg_solver.py:392-428), from the
    irreducible pairing vertex [Q, a, b, c, d, nu, nu'] and chi0pp [Nk, a, b, c, d, nu] in the upstream layouts."""

    def __init__(self, gamma_pp_irr: np.ndarray, chi0pp: np.ndarray, nk: tuple, irrk_inv, beta: float, sign: float):
        Q, n, nvp = gamma_pp_irr.shape[0], gamma_pp_irr.shape[1], gamma_pp_irr.shape[5]
        self.n, self.P, self.nk, self.beta, self.sign = n, nvp // 2, tuple(int(x) for x in nk), float(beta), float(sign)
        M = n * n * nvp
        self.M = M
        nk_tot = int(np.prod(self.nk))
        # Mat[(a,b,nu)][(c,d,nu')] = Gamma[a,c,b,d](nu,nu') (the device pairing-vertex layout)
        mat_irr = _dev(np.asarray(gamma_pp_irr).transpose(0, 1, 3, 5, 2, 4, 6).reshape(Q, M, M))
        self.tw_fwd, self.tw_inv = _dev(twiddles(self.nk, -1)), _dev(twiddles(self.nk, +1))
        gather = torch.as_tensor(np.asarray(irrk_inv, dtype=np.int32), device="cuda")
        self.mat = torch.empty((nk_tot, M, M), dtype=C128, device="cuda")
        call("dga_dft_planes_gather_c128", _p(mat_irr), 1, 0, M * M, _p(self.mat), 1, 0, M * M, 1, M * M, self.nk[0],
             self.nk[1], self.nk[2], _p(self.tw_fwd), self.sign, _p(gather), _s())
        self.chi0pp = _dev(np.asarray(chi0pp).reshape(nk_tot, n, n, n, n, nvp).transpose(0, 5, 1, 2, 3, 4)
                           .reshape(nk_tot, nvp, n * n, n * n))
        self.scratch = torch.empty(int(lib().dga_eli_matvec_scratch_bytes(n, self.P, nk_tot)) // 16 + 1, dtype=C128,
                                   device="cuda")
        self.dim = nk_tot * M

    def __call__(self, x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        call("dga_eli_matvec_c128", _p(self.mat), _p(self.chi0pp), _p(x), self.n, self.P, self.nk[0], self.nk[1],
             self.nk[2], _p(self.tw_fwd), _p(self.tw_inv), self.beta, self.sign, _p(out), _p(self.scratch), self.scratch.numel() * 16, _s())
        return out


def solve_eliashberg_lanczos(gamma_r_pp, gchi0_q0_pp, ranks=(0, 0)):
    """eliashberg_solver.solve_eliashberg_lanczos (eliashberg_solver.py:376-471): the config.eliashberg.n_eig
    leading eigenvalues (descending) and gap functions of the channel of ``gamma_r_pp`` (irreducible q,
    compressed, PP notation) with ``gchi0_q0_pp`` (full zone, compressed), to config.eliashberg.epsilon."""
    cfg = _cfg()
    qg = cfg.lattice.q_grid
    ch = _channel_name(gamma_r_pp.channel)
    sign = 1.0 if ch == "sing" else -1.0
    g = np.asarray(gamma_r_pp.mat)
    g = g.reshape(-1, *g.shape[-6:])
    nk = tuple(int(x) for x in qg.nk)
    op = PairingOperator(g, np.asarray(gchi0_q0_pp.mat), nk, qg.irrk_inv, float(cfg.sys.beta), sign)
    n, P = op.n, op.P
    symmetry = (getattr(cfg.eliashberg, "symmetry", None) or "random").lower()
    gap0 = initial_gap(nk, n, P, ch, symmetry, qg.irrk_ind, qg.irrk_inv)
    n_eig = int(cfg.eliashberg.n_eig)
    out = torch.empty(op.dim, dtype=C128, device="cuda")
    x0 = torch.as_tensor(gap0.ravel(), device="cuda")
    vals, vecs, status = krylov_schur(lambda v: op(v.contiguous(), out), x0, n_eig, float(cfg.eliashberg.epsilon))
    if status:
        raise RuntimeError("the Krylov-Schur iteration did not converge (ArpackNoConvergence in the upstream)")
    gap_shape = nk + (n, n, 2 * P)
    gaps = [_make("GapFunction", v.reshape(gap_shape), gamma_r_pp.channel, nk) for v in vecs]
    return vals, gaps


# ------------------------------------------------------------------------------------------------
# install / uninstall
# ------------------------------------------------------------------------------------------------
PATCHES = [
    ("bubble_gen", "BubbleGenerator", "create_generalized_chi0_q_fft_auto", create_generalized_chi0_q_fft_auto, True),
    ("bubble_gen", "BubbleGenerator", "create_generalized_chi0_q_auto", create_generalized_chi0_q_auto, True),
    ("bubble_gen", "BubbleGenerator", "create_generalized_chi0_q_pp_w0", create_generalized_chi0_q_pp_w0, True),
    ("four_point", "FourPoint", "invert_and_sum_over_last_vn", invert_and_sum_over_last_vn, False),
    ("four_point", "FourPoint", "invert_and_sum_over_last_vn_v2", invert_and_sum_over_last_vn, False),
    ("nonlocal_sde", None, "create_auxiliary_chi_r_q_sum_v1", create_auxiliary_chi_r_q_sum_v1, False),
    ("nonlocal_sde", None, "create_auxiliary_chi_r_q_sum_v2", create_auxiliary_chi_r_q_sum_v2, False),
    ("nonlocal_sde", None, "create_auxiliary_chi_r_q_sum_v3", create_auxiliary_chi_r_q_sum_v3, False),
    ("nonlocal_sde", None, "calculate_sigma_from_kernel_fft_auto", calculate_sigma_from_kernel_fft_auto, False),
    ("nonlocal_sde", None, "calculate_sigma_from_kernel_auto", calculate_sigma_from_kernel_auto, False),
    ("nonlocal_sde", None, "get_hartree_fock", get_hartree_fock, False),
    ("lambda_correction", None, "find_lambda", find_lambda, False),
    ("lambda_correction", None, "perform_single_lambda_correction", perform_single_lambda_correction, False),
    ("eliashberg_solver", None, "solve_eliashberg_lanczos", solve_eliashberg_lanczos, False),
    ("local_sde", None, "perform_local_schwinger_dyson", perform_local_schwinger_dyson, False),
]


def install(package: str = "dgamore", precision: str = "fp64") -> list:
    """Patches the device drop-ins into the imported upstream package and registers its config and classes.
    Returns the list of (owner, name, original) it replaced; ``uninstall()`` puts them back."""
    import importlib

    lib()  # no CPU fallback: fail before patching anything if the library is missing
    set_precision(precision)
    mods = {m: importlib.import_module(f"{package}.{m}") for m in
            ("bubble_gen", "four_point", "nonlocal_sde", "lambda_correction", "eliashberg_solver", "self_energy",
             "gap_function", "n_point_base", "local_sde", "local_four_point")}
    use_config(importlib.import_module(f"{package}.config"))
    use_classes(FourPoint=mods["four_point"].FourPoint, SelfEnergy=mods["self_energy"].SelfEnergy,
                GapFunction=mods["gap_function"].GapFunction, SpinChannel=mods["n_point_base"].SpinChannel,
                LocalFourPoint=mods["local_four_point"].LocalFourPoint,
                FrequencyNotation=mods["n_point_base"].FrequencyNotation)
    replaced = []
    for mod, cls, name, fn, static in PATCHES:
        owner = getattr(mods[mod], cls) if cls else mods[mod]
        original = owner.__dict__[name] if cls else getattr(owner, name)
        setattr(owner, name, staticmethod(fn) if static else fn)
        replaced.append((owner, name, original))
    _state["patched"] = replaced
    return replaced


def uninstall() -> None:
    """Restores the upstream functions that ``install`` replaced."""
    for owner, name, original in reversed(_state["patched"]):
        setattr(owner, name, original)
    _state["patched"] = []


def namespace_config(beta: float, nk: tuple, irrk_ind, irrk_inv, irrk_count, n_bands: int, niv_core: int = 0,
                     niw_core: int = 0, occ=None, occ_k=None, n_eig: int = 1, epsilon: float = 1e-6,
                     symmetry: str | None = None):
    """A minimal stand-in for the upstream ``config`` with the values the drop-ins read (for direct calls)."""
    nk = tuple(int(x) for x in nk)
    q_grid = types.SimpleNamespace(nk=nk, nk_tot=int(np.prod(nk)), irrk_ind=np.asarray(irrk_ind),
                                   irrk_inv=np.asarray(irrk_inv), irrk_count=np.asarray(irrk_count))
    return types.SimpleNamespace(
        sys=types.SimpleNamespace(beta=float(beta), n_bands=int(n_bands), occ=occ, occ_k=occ_k),
        lattice=types.SimpleNamespace(nk=nk, nq=nk, q_grid=q_grid, k_grid=q_grid),
        box=types.SimpleNamespace(niv_core=int(niv_core), niw_core=int(niw_core)),
        eliashberg=types.SimpleNamespace(n_eig=int(n_eig), epsilon=float(epsilon), symmetry=symmetry),
    )
