"""Device-resident nonlocal ladder-DGA pass on one B200.

One pass replays the hot path of ``nonlocal_sde.calculate_self_energy_q`` (dgamore/nonlocal_sde.py:786-879)
entirely on the device, with every stage a libdga_b200 kernel enqueued on one CUDA stream:

    G(k) --DFT--> G(R) --bubble--> chi0(q_irr, w, nu) --prep--> chi0^-1, nu sums
    chi0, F_dc --dc GEMM--> K_dc
    chi0^-1, Gamma_r(w), U_r + V_r^q --BSE (dens, magn)--> X = sum_nu' chi* / beta
    X --shell correction--> chi_r(q, w) --lambda (single band)--> chi_r^lambda
    chi0^-1, X, chi_r --assembly--> K = -K_dc + K_d + 3 K_m
    K, G(R) --Sigma contraction + inverse DFT--> Sigma(k, nu)

Inputs stay resident between passes (``LadderPass.upload``), so a pass needs only the device-side work;
``run_e2e`` adds the host->device copy of G(k) and the device->host copy of Sigma.  PyTorch is used for
device memory and the stream only.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import call, lib, ll_array

C128 = torch.complex128


def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _s() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def twiddles(nk: tuple, sign: int) -> np.ndarray:
    """e^{sign 2 pi i m / n} for each axis, concatenated (x, y, z), in FP64."""
    parts = [np.exp(sign * 2j * np.pi * np.arange(n) / n) for n in nk]
    return np.concatenate(parts).astype(np.complex128)


def _resident(x, dev) -> torch.Tensor:
    """A complex128 input on the device: a device tensor (the local equation's results, local_sde.LocalSde) as it
    is, host arrays copied once."""
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=C128).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).to(dev)


def compound_orb(x: np.ndarray) -> np.ndarray:
    """[..., a, b, c, d] -> [..., (a,b), (d,c)] compound orbital matrices."""
    nb = x.shape[-1]
    return np.swapaxes(x, -1, -2).reshape(*x.shape[:-4], nb * nb, nb * nb)


def u_channel(u: np.ndarray, channel: str) -> np.ndarray:
    """Local interaction in a spin channel (dgamore/interaction.py:43-65)."""
    u_adcb = np.einsum("abcd->adcb", u)
    return 2 * u - u_adcb if channel == "dens" else -u_adcb


def v_channel(v: np.ndarray, channel: str) -> np.ndarray:
    """Non-local interaction in a spin channel (dgamore/interaction.py:160-182)."""
    return 2 * v if channel == "dens" else 0 * v


@dataclass
class PassShapes:
    n_orb: int
    nk: tuple
    beta: float
    niw: int
    niv: int
    niv_shell: int
    n_q: int
    niv_g: int
    rotated: bool = False  # auto-mode symmetries with orbital rotations in the IBZ -> FBZ map
    wedge: bool = False  # Sigma through the irreducible wedge of real space (dga_sigma_wedge_c128)

    @property
    def n2(self):
        return self.n_orb * self.n_orb

    @property
    def W(self):
        return self.niw + 1

    @property
    def nv(self):
        return 2 * self.niv

    @property
    def nvf(self):
        return 2 * (self.niv + self.niv_shell)

    @property
    def N(self):
        return self.n2 * self.nv

    @property
    def nk_tot(self):
        return int(np.prod(self.nk))

    @property
    def n_solves(self) -> int:
        """(q, w) ladder solves of one pass: irreducible q x (niw+1) x 2 channels."""
        return self.n_q * self.W * 2

    @classmethod
    def from_inputs(cls, inp: dict) -> "PassShapes":
        u = np.asarray(inp["u"])
        g_k = inp["g_k"]
        return cls(
            n_orb=u.shape[0], nk=tuple(int(x) for x in inp["nk"]), beta=float(inp["beta"]), niw=int(inp["niw"]),
            niv=int(inp["niv_core"]), niv_shell=int(inp["niv_shell"]), n_q=len(inp["irrk_ind"]),
            niv_g=np.shape(g_k)[-1] // 2, rotated=needs_rotation(inp),
            wedge=not needs_rotation(inp) and inversion_shares_representatives(inp["irrk_inv"], inp["nk"]),
        )


def inversion_shares_representatives(irrk_inv, nk) -> bool:
    """True when every point and its inverse -k (per axis modulo the grid) map to the same irreducible point, the
    condition of the wedge form of the Sigma contraction."""
    inv = np.asarray(irrk_inv).reshape(tuple(int(x) for x in nk))
    neg = inv[tuple(np.ix_(*[(-np.arange(n)) % n for n in inv.shape]))]
    return bool(np.array_equal(inv, neg))


def star_sums(irrk_ind, irrk_inv, nk) -> np.ndarray:
    """S[q_irr][r] = sum over the points q with irrk_inv[q] = q_irr of e^{+i q R_r}, R_r = the point irrk_ind[r], from
    the per-axis twiddles e^{+2 pi i m / n} (the s_star operand of dga_sigma_wedge_c128)."""
    nk = tuple(int(x) for x in nk)
    tw = [np.exp(2j * np.pi * np.arange(n) / n) for n in nk]
    k = np.array(np.unravel_index(np.arange(int(np.prod(nk))), nk)).T  # [Nk][3]
    r = np.array(np.unravel_index(np.asarray(irrk_ind), nk)).T  # [Q][3]
    phase = np.ones((len(k), len(r)), dtype=np.complex128)
    for ax in range(3):
        phase *= tw[ax][(k[:, ax:ax + 1] * r[None, :, ax]) % nk[ax]]
    s = np.zeros((len(r), len(r)), dtype=np.complex128)
    np.add.at(s, np.asarray(irrk_inv).ravel(), phase)
    return s


def needs_rotation(inp: dict) -> bool:
    """True when the inputs carry auto-mode orbital rotations (``orbital_us``, ``orbital_conjs``) that are not all
    the identity without conjugation (KGrid.specify_auto_symmetries, brillouin_zone.py:365-449)."""
    if "orbital_us" not in inp:
        return False
    us = np.asarray(inp["orbital_us"])
    conjs = np.asarray(inp["orbital_conjs"], dtype=bool)
    return bool(conjs.any()) or not np.array_equal(us, np.broadcast_to(np.eye(us.shape[-1]), us.shape))


_ALLOC_GRAIN = 512  # the caching allocator's block granularity


def _blk(nbytes: int) -> int:
    return -(-int(nbytes) // _ALLOC_GRAIN) * _ALLOC_GRAIN


def device_sm_count() -> int:
    """SMs of the current CUDA device (the library's cached query); 148, the B200's count, without a GPU."""
    if torch.cuda.is_available():
        return int(lib().dga_device_sm_count())
    return 148


def sigma_chunks_for(sh: PassShapes, sm_count: int | None = None) -> int:
    """(nu, i, j, w-chunk) CTAs of the Sigma contraction: at least four waves of its two resident CTAs per SM
    (8 CTAs per SM in all: 1,184 on a 148-SM B200), so that the last wave's tail is short (the 3-orbital 32x32
    pass has 360 (nu, i, j) units: 4 chunks)."""
    sms = device_sm_count() if sm_count is None else int(sm_count)
    base = sh.niv * sh.n2
    return max(1, min(2 * sh.niw + 1, -(-(8 * sms) // base)))


def estimate_device_bytes(sh: PassShapes, precision: str = "fp64", keep_intermediates: bool = True,
                          own_bse_scratch: bool = False) -> int:
    """HBM held by a LadderPass of these shapes (resident inputs + work buffers), computed without a GPU.

    Mirrors the allocations of ``LadderPass.__init__``; with ``own_bse_scratch`` False (the serving path) the
    BSE scratch is not counted because the batch launch brings its own."""
    c = 16
    n, n2, W, Q, nv, nvf, N, nk = sh.n_orb, sh.n2, sh.W, sh.n_q, sh.nv, sh.nvf, sh.N, sh.nk_tot
    Nf = n2 * nvf
    n_items = 2 * Q * W
    tw = sum(sh.nk) * c
    chunks = sigma_chunks_for(sh)
    sizes = [
        Q * 3 * 4, nk * 4, Q * 8, tw, tw,                      # q_irr, irrk_inv, irrk_count, twiddles
        2 * Q * n2 * n2 * c, n2 * n2 * c, 2 * c,               # uv, u_perm, targets
        2 * W * N * N * c, W * Nf * Nf * c,                    # gamma_cm, F_dc
        nk * n * n * 2 * sh.niv_g * c, n_items * 3 * 4,        # G(k), work
        (nvf + sh.niw) * n * n * nk * c, (sh.niv + 2 * sh.niw) * n * n * nk * c,  # G(R) slots
        Q * W * nvf * n2 * n2 * c, Q * W * nv * n2 * n2 * c,   # chi0, chi0^-1
        Q * W * n2 * n2 * c, Q * W * n2 * n2 * c,              # nu sums
        Q * W * nv * n2 * n2 * c,                              # K_dc
        (Q * W * 2 * (nvf // 2) * n2 * n2 * c) // c * c + c,  # dc scratch
        2 * Q * W * N * n2 * c, n_items * 4, n_items * 4,      # X, status, iters
        2 * Q * W * n2 * n2 * c, 2 * Q * W * n2 * n2 * c,      # chi_phys, chi_lam
        2 * 8, 2 * 4, 4 * 4,                                   # lambdas, iterations, status
        Q * W * nv * n2 * n2 * c,                              # K
        (chunks * sh.niv * n2 * nk * c * 2 + (W * nv * n2 * n2 * Q * c if sh.wedge else 0)) // c * c + c,  # Sigma scratch
        nk * n * n * 2 * sh.niv * c,                           # Sigma
    ]
    if sh.wedge:
        sizes.append(Q * Q * c)  # star sums
    if sh.rotated:
        sizes += [nk * n * n * c, nk * 8, nk, nk * 4, nk * W * nv * n2 * n2 * c]  # U_k, sigma_k, conj_k, map, K(FBZ)
    if keep_intermediates:
        sizes.append(2 * Q * W * nv * n2 * n2 * c)
    if own_bse_scratch:
        raise ValueError("the BSE scratch of a standalone pass depends on the GPU's occupancy; count it separately")
    return sum(_blk(x) for x in sizes)


class LadderPass:
    """Resident inputs, work buffers and the kernel sequence of one nonlocal pass."""

    def __init__(self, inp: dict, device: str = "cuda", do_lambda: bool | None = None, sigma_chunks: int | None = None,
                 keep_intermediates: bool = True, precision: str = "fp64", refine_tol: float = 1e-10,
                 refine_max_iter: int = 6, resolve_grid: int = 148, own_bse_scratch: bool = True,
                 eliashberg_pp: int | None = None):
        lib()  # fail loudly before anything else if the CUDA library is missing
        self.dev = torch.device(device)
        g_k = np.asarray(inp["g_k"])
        u = np.asarray(inp["u"], dtype=np.complex128)
        n_orb = u.shape[0]
        self.sh = PassShapes.from_inputs(inp)
        sh = self.sh
        nk = sh.nk
        if sh.niv_g < sh.niv + sh.niv_shell + sh.niw:
            raise ValueError("G(k) must hold at least niv_full + niw fermionic frequencies")
        self.do_lambda = (n_orb == 1) if do_lambda is None else bool(do_lambda)
        if self.do_lambda and n_orb != 1:
            raise NotImplementedError("the lambda-correction is single-band only (dgamore/DGAmore.py:501-508)")
        self.keep = keep_intermediates
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        self.precision = precision
        self.refine_tol = float(refine_tol)
        self.refine_max_iter = int(refine_max_iter)
        dev = self.dev
        beta = sh.beta
        # ---------------- host-side preparation (once per request) ----------------
        irr = np.asarray(inp["irrk_ind"])
        self.irrk_ind_host = irr
        q_list = np.array(np.unravel_index(irr, nk)).T.astype(np.int32)
        self.q_irr = torch.from_numpy(np.ascontiguousarray(q_list)).to(dev)
        self.irrk_inv = torch.from_numpy(np.asarray(inp["irrk_inv"], dtype=np.int32)).to(dev)
        # auto-mode symmetries (KGrid.specify_auto_symmetries): per-k orbital rotations of the IBZ -> FBZ map
        self.rot_us = self.rot_sigmas = self.rot_conjs = self.rot_ident = self.k_full = None
        if sh.rotated:
            us = np.asarray(inp["orbital_us"], dtype=np.complex128).reshape(sh.nk_tot, n_orb, n_orb)
            conjs = np.asarray(inp["orbital_conjs"], dtype=bool).ravel()
            sig = np.asarray(inp.get("orbital_sigmas", np.ones(len(conjs))), dtype=np.float64).ravel()
            self.rot_us = torch.from_numpy(np.ascontiguousarray(us)).to(dev)
            self.rot_sigmas = torch.from_numpy(np.ascontiguousarray(sig)).to(dev)
            self.rot_conjs = torch.from_numpy(conjs.astype(np.uint8)).to(dev)
            self.rot_ident = torch.arange(sh.nk_tot, dtype=torch.int32, device=dev)
            self.k_full = torch.empty((sh.nk_tot, sh.W, sh.nv, sh.n2, sh.n2), dtype=C128, device=dev)
        self.irrk_count = torch.from_numpy(np.asarray(inp["irrk_count"], dtype=np.int64)).to(dev)
        self.tw_fwd = torch.from_numpy(twiddles(nk, -1)).to(dev)
        self.tw_inv = torch.from_numpy(twiddles(nk, +1)).to(dev)
        v_irr = np.asarray(inp["v_q_irr"], dtype=np.complex128)
        uv = np.stack([compound_orb(v_channel(v_irr, ch) + u_channel(u, ch)[None]) for ch in ("dens", "magn")])
        self.uv = torch.from_numpy(np.ascontiguousarray(uv)).to(dev)
        u_perm = np.einsum("abcd->adcb", u) * (1.0 / beta**2)
        self.u_perm = torch.from_numpy(np.ascontiguousarray(compound_orb(u_perm))).to(dev)
        self.inv_beta2 = 1.0 / beta**2
        self.targets = torch.tensor(
            [complex(inp.get("chi_loc_sum_dens", 0)), complex(inp.get("chi_loc_sum_magn", 0))], dtype=C128, device=dev
        )
        # Gamma_r (upstream layout) -> column-major compound [ch][W][N][N]
        n, nv, W, N = sh.n_orb, sh.nv, sh.W, sh.N
        self.gamma_cm = torch.empty((2, W, N, N), dtype=C128, device=dev)
        for ich, ch in enumerate(("dens", "magn")):
            g_ref = _resident(inp[f"gamma_{ch}"], dev)
            src_strides = list(g_ref.stride())
            dst = self.gamma_cm[ich]
            # dims (a, b, c, d, w, nu, nu')
            dst_strides = [n * nv, nv, nv * N, n * nv * N, N * N, 1, N]
            call("dga_strided_copy_c128", _p(g_ref), _p(dst), 7, ll_array(g_ref.shape), ll_array(src_strides),
                 ll_array(dst_strides), 1.0, _s())
        # F_dc (upstream [d,c,e,f,w,nu,nu']) -> row-major compound [W][Nf][Nf]
        nvf = sh.nvf
        Nf = sh.n2 * nvf
        f_ref = _resident(inp["f_dc"], dev)
        self.fdc = torch.empty((W, Nf, Nf), dtype=C128, device=dev)
        call("dga_strided_copy_c128", _p(f_ref), _p(self.fdc), 7, ll_array(f_ref.shape), ll_array(list(f_ref.stride())),
             ll_array([n * nvf * Nf, nvf * Nf, nvf, n * nvf, Nf * Nf, Nf, 1]), 1.0, _s())
        del f_ref
        # resident G(k) and work list
        self.g_k = torch.from_numpy(np.ascontiguousarray(g_k, dtype=np.complex128).reshape(sh.nk_tot, n, n, -1)).to(dev)
        work = [(ch, q, w) for w in range(W) for ch in range(2) for q in range(sh.n_q)]
        self.work = torch.tensor(work, dtype=torch.int32, device=dev)
        self.n_items = len(work)
        # ---------------- work buffers ----------------
        Q, n2, nk_tot = sh.n_q, sh.n2, sh.nk_tot
        self.t_bubble = nvf + sh.niw
        self.g_r_bubble = torch.empty((self.t_bubble, n, n, nk_tot), dtype=C128, device=dev)
        self.t_sigma = sh.niv + 2 * sh.niw
        self.g_r_sigma = torch.empty((self.t_sigma, n, n, nk_tot), dtype=C128, device=dev)
        self.chi0 = torch.empty((Q, W, nvf, n2, n2), dtype=C128, device=dev)
        self.chi0_inv = torch.empty((Q, W, nv, n2, n2), dtype=C128, device=dev)
        self.full_sum = torch.empty((Q, W, n2, n2), dtype=C128, device=dev)
        self.core_sum = torch.empty((Q, W, n2, n2), dtype=C128, device=dev)
        self.k_dc = torch.empty((Q, W, nv, n2, n2), dtype=C128, device=dev)
        self.dc_scratch = torch.empty(
            int(lib().dga_dc_scratch_bytes(n, sh.niv + sh.niv_shell, W, Q)) // 16 + 1, dtype=C128, device=dev
        )
        self.X = torch.empty((2, Q, W, N, n2), dtype=C128, device=dev)
        self.bse_status = torch.zeros(self.n_items, dtype=torch.int32, device=dev)
        self.own_bse_scratch = bool(own_bse_scratch)
        self.tuning = None
        if not self.own_bse_scratch:
            # the BSE runs in a batch launch (serving.solve_bse_batch) that brings its own scratch
            self.bse_scratch = self.mixed_scratch = None
        elif precision == "fp64" and eliashberg_pp:
            self.bse_scratch_bytes = int(lib().dga_bse_eli_scratch_bytes(N, n2, self.n_items))
        elif precision == "fp64":
            self.bse_scratch_bytes = int(lib().dga_bse_scratch_bytes(N, n2, self.n_items))
        else:
            # mixed solve + a small FP64 grid for the status-driven re-solve of unconverged items
            self.resolve_grid = int(resolve_grid)
            self.mixed_scratch_bytes = int(lib().dga_bse_mixed_scratch_bytes(N, n2, self.n_items))
            self.bse_scratch_bytes = self.resolve_grid * (N * N + N * n2) * 16
            self.mixed_scratch = torch.empty(self.mixed_scratch_bytes // 16 + 1, dtype=C128, device=dev)
        if self.own_bse_scratch:
            self.bse_scratch = torch.empty(self.bse_scratch_bytes // 16 + 1, dtype=C128, device=dev)
        self.bse_iters = torch.zeros(self.n_items, dtype=torch.int32, device=dev)
        self.chi_phys = torch.empty((2, Q, W, n2, n2), dtype=C128, device=dev)
        self.chi_lam = torch.empty((2, Q, W, n2, n2), dtype=C128, device=dev)
        self.lambdas = torch.zeros(2, dtype=torch.float64, device=dev)
        self.lambda_iters = torch.zeros(2, dtype=torch.int32, device=dev)
        self.status = torch.zeros(4, dtype=torch.int32, device=dev)
        self.K = torch.empty((Q, W, nv, n2, n2), dtype=C128, device=dev)
        self.gamma3 = torch.empty((2, Q, W, nv, n2, n2), dtype=C128, device=dev) if keep_intermediates else None
        # Eliashberg vertex fused into the FP64 BSE: the items w < 2 niv_pp also write the chi* part of the full
        # vertex in the pp box from their own LU factors (eliashberg_solver.EliashbergSolver adds the ladder term)
        self.eli_P = int(eliashberg_pp) if eliashberg_pp else 0
        self.f_pp = None
        if self.eli_P:
            if precision != "fp64" or not own_bse_scratch or not keep_intermediates:
                raise ValueError("the fused Eliashberg vertex needs the FP64 BSE, its own scratch and the three-leg vertex")
            if 2 * self.eli_P > W or self.eli_P > sh.niv:
                raise ValueError(f"eliashberg_pp={self.eli_P} needs 2 niv_pp <= niw + 1 and niv_pp <= niv")
            mb = n2 * 2 * self.eli_P
            self.f_pp = torch.empty((2, Q, 2 * self.eli_P, mb, mb), dtype=C128, device=dev)
        self.f_pp_ready = False  # f_pp holds the chi* part of this pass's vertex (the fused BSE ran last)
        if sigma_chunks is None:
            sigma_chunks = sigma_chunks_for(sh)
        self.sigma_chunks = sigma_chunks
        self.sigma_tile = 1  # wedge GEMM tile (dga_sigma_wedge_c128; autotune.tune_sigma picks it per shape)
        if sh.wedge:
            self.s_star = torch.from_numpy(star_sums(inp["irrk_ind"], inp["irrk_inv"], sh.nk)).to(dev)
            self.sigma_scratch_bytes = int(lib().dga_sigma_wedge_scratch_bytes(n, sh.niv, sh.niw, sh.n_q, nk_tot,
                                                                               sigma_chunks))
        else:
            self.s_star = None
            self.sigma_scratch_bytes = int(lib().dga_sigma_scratch_bytes(n, sh.niv, nk_tot, sigma_chunks))
        self.sigma_scratch = torch.empty(self.sigma_scratch_bytes // 16 + 1, dtype=C128, device=dev)
        self.sigma = torch.empty((nk_tot, n, n, 2 * sh.niv), dtype=C128, device=dev)
        self.g_k_host = torch.from_numpy(np.ascontiguousarray(g_k, dtype=np.complex128).reshape(sh.nk_tot, n, n, -1)).pin_memory()
        self.sigma_host = torch.empty(self.sigma.shape, dtype=C128).pin_memory()

    # ------------------------------------------------------------------------------------------
    def _g_transform(self, out: torch.Tensor, nu_first: int, n_slots: int):
        """out[t][a][b][R] = sum_k G(k)[a][b][nu_first + t] e^{-ikR} (forward transform, n_point_base.py:509-529)."""
        sh = self.sh
        n, nvg2 = sh.n_orb, 2 * sh.niv_g
        base = self.g_k[..., sh.niv_g + nu_first :]
        nx, ny, nz = sh.nk
        call("dga_dft_planes_c128", _p(base), 1, nvg2, n * n * nvg2, _p(out), n * n * sh.nk_tot, sh.nk_tot, 1,
             n * n, n_slots * n * n, nx, ny, nz, _p(self.tw_fwd), 1.0, _s())

    def bubble(self):
        sh = self.sh
        n, n2, W, nvf = sh.n_orb, sh.n2, sh.W, sh.nvf
        self._g_transform(self.g_r_bubble, -(nvf // 2) - sh.niw, self.t_bubble)
        strides = [W * nvf * n2 * n2, nvf * n2 * n2, n2 * n2, n * n2, n2, 1, n]  # q w nu a b c d
        nx, ny, nz = sh.nk
        call("dga_bubble_c128", _p(self.g_r_bubble), n, nvf // 2, sh.niw, nx, ny, nz, _p(self.q_irr), sh.n_q,
             _p(self.tw_inv), sh.beta, _p(self.chi0), ll_array(strides), _s())

    def chi0_prep(self):
        sh = self.sh
        call("dga_chi0_prep_c128", _p(self.chi0), sh.n_orb, sh.niv, sh.niv_shell, sh.W, sh.n_q, sh.beta,
             _p(self.chi0_inv), _p(self.full_sum), _p(self.core_sum), _p(self.status), _s())

    def dc_kernel(self):
        sh = self.sh
        call("dga_dc_kernel_c128", _p(self.chi0), _p(self.u_perm), _p(self.fdc), sh.n_orb, sh.niv, sh.niv_shell, sh.W,
             sh.n_q, _p(self.k_dc), _p(self.dc_scratch), self.dc_scratch.numel() * 16, _s())

    def set_tuning(self, choice, wait_limit: int = 0) -> None:
        """Uses the launch choice (kernel, ctas_per_sm) of dga_bse_tuning for this pass's BSE (see autotune.py).

        ``wait_limit`` (polls, 0 = the library default) bounds each wait of the mixed kernels on a bulk copy or
        a tensor-core tile inside an item; an item whose wait runs out is flagged DGA_ITEM_WAIT_TIMEOUT and
        re-solved in FP64."""
        from ._lib import BseTuning

        t = BseTuning(kernel=int(choice[0]), ctas_per_sm=int(choice[1]), wait_limit=int(wait_limit))
        sh = self.sh
        mixed = 1 if self.precision == "mixed" else 0
        nbytes = int(lib().dga_bse_tuned_scratch_bytes(sh.N, sh.n2, self.n_items, mixed, ctypes.byref(t)))
        if nbytes == 0:
            raise ValueError(f"tuning {tuple(choice)} cannot run N={sh.N} in {self.precision}")
        self.tuning = t
        self.mixed_scratch = None
        if mixed:
            self.tuned_scratch = torch.empty(nbytes // 16 + 1, dtype=C128, device=self.dev)
        else:
            # the FP64 form reuses its own scratch when it is large enough
            if self.bse_scratch is None or self.bse_scratch.numel() * 16 < nbytes:
                self.bse_scratch = torch.empty(nbytes // 16 + 1, dtype=C128, device=self.dev)
            self.tuned_scratch = self.bse_scratch

    def bse(self):
        sh = self.sh
        if not self.own_bse_scratch:
            raise RuntimeError("this pass was built without BSE scratch: run its BSE through serving.solve_bse_batch")
        self.f_pp_ready = False
        if self.tuning is not None:
            mixed = 1 if self.precision == "mixed" else 0
            call("dga_bse_solve_sum_tuned_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2,
                 _p(self.gamma_cm), _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, mixed,
                 self.refine_max_iter, self.refine_tol, _p(self.X), _p(self.bse_status), _p(self.bse_iters),
                 ctypes.byref(self.tuning), _p(self.tuned_scratch), self.tuned_scratch.numel() * 16, _s())
            if mixed:
                call("dga_bse_resolve_fp64_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2,
                     _p(self.gamma_cm), _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, _p(self.X),
                     _p(self.bse_status), self.resolve_grid, _p(self.bse_scratch), self.bse_scratch.numel() * 16,
                     _s())
            return
        if self.precision == "mixed":
            call("dga_bse_solve_sum_mixed_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2,
                 _p(self.gamma_cm), _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, self.refine_max_iter,
                 self.refine_tol, _p(self.X), _p(self.bse_status), _p(self.bse_iters), _p(self.mixed_scratch),
                 self.mixed_scratch.numel() * 16, _s())
            call("dga_bse_resolve_fp64_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2,
                 _p(self.gamma_cm), _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, _p(self.X),
                 _p(self.bse_status), self.resolve_grid, _p(self.bse_scratch), self.bse_scratch.numel() * 16, _s())
            return
        if self.eli_P:
            call("dga_bse_solve_sum_eli_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2,
                 _p(self.gamma_cm), _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, self.eli_P,
                 2 * self.eli_P, _p(self.X), _p(self.f_pp), _p(self.bse_status), _p(self.bse_scratch),
                 self.bse_scratch.numel() * 16, _s())
            self.f_pp_ready = True
            return
        call("dga_bse_solve_sum_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, self.inv_beta2, _p(self.gamma_cm),
             _p(self.chi0_inv), _p(self.uv), _p(self.work), self.n_items, _p(self.X), _p(self.bse_status),
             _p(self.bse_scratch), self.bse_scratch.numel() * 16, _s())

    def chi_phys_stage(self):
        sh = self.sh
        call("dga_chi_phys_c128", _p(self.X), _p(self.uv), _p(self.full_sum), _p(self.core_sum), sh.n_orb, sh.niv,
             sh.W, sh.n_q, 2, sh.beta, _p(self.chi_phys), _p(self.status), _s())

    def lambda_stage(self):
        sh = self.sh
        if not self.do_lambda:
            return self.chi_phys
        call("dga_lambda_c128", _p(self.chi_phys), sh.n_q, sh.W, 2, _p(self.irrk_count), _p(self.targets), sh.beta,
             float(sh.nk_tot), 0.1, 1e-7, 1000, _p(self.lambdas), _p(self.lambda_iters), _p(self.status[1:]),
             _p(self.chi_lam), _s())
        return self.chi_lam

    def kernel_stage(self, chi_r: torch.Tensor):
        sh = self.sh
        call("dga_kernel_assembly_c128", _p(self.chi0_inv), _p(self.X), _p(self.uv), _p(chi_r), _p(self.k_dc),
             sh.n_orb, sh.niv, sh.W, sh.n_q, sh.beta, _p(self.K),
             _p(self.gamma3) if self.gamma3 is not None else ctypes.c_void_p(0), _s())

    def sigma_stage(self):
        sh = self.sh
        self._g_transform(self.g_r_sigma, -sh.niw, self.t_sigma)
        nx, ny, nz = sh.nk
        if sh.wedge:
            call("dga_sigma_wedge_c128", _p(self.K), _p(self.g_r_sigma), sh.n_orb, sh.niv, sh.niw, sh.n_q, nx, ny, nz,
                 _p(self.irrk_inv), _p(self.s_star), _p(self.tw_inv), sh.beta, self.sigma_chunks, self.sigma_tile,
                 _p(self.sigma),
                 _p(self.sigma_scratch), self.sigma_scratch.numel() * 16, _s())
            return
        kern, n_q, inv = self.K, sh.n_q, self.irrk_inv
        if sh.rotated:
            # K(q) over the full zone with each point's orbital rotation, then the contraction without a gather
            n, n2, W, nv = sh.n_orb, sh.n2, sh.W, sh.nv
            call("dga_fbz_rotate_c128", _p(self.K), _p(self.irrk_inv), sh.nk_tot, _p(self.rot_us), _p(self.rot_sigmas),
                 _p(self.rot_conjs), n, ll_array([n * n2, n2, 1, n]), n2 * n2, W * nv, 0, 1, W * nv * n2 * n2,
                 _p(self.k_full), _s())
            kern, n_q, inv = self.k_full, sh.nk_tot, self.rot_ident
        call("dga_sigma_c128", _p(kern), _p(self.g_r_sigma), sh.n_orb, sh.niv, sh.niw, n_q, nx, ny, nz,
             _p(inv), _p(self.tw_inv), sh.beta, self.sigma_chunks, _p(self.sigma), _p(self.sigma_scratch),
             self.sigma_scratch.numel() * 16, _s())

    def set_occupations(self, occ: np.ndarray, occ_k: np.ndarray, v_q_full: np.ndarray, u: np.ndarray) -> None:
        """Adds the Hartree-Fock term to Sigma at the end of every pass (nonlocal_sde.py:782-784, 884), from
        config.sys.occ [n][n], config.sys.occ_k [kx,ky,kz,n,n], V(q) over the full grid [Nq][n][n][n][n] and U."""
        dev, sh = self.dev, self.sh
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).to(dev)
        self.hf_u = up(u)
        self.hf_v = up(np.asarray(v_q_full).reshape(sh.nk_tot, -1))
        self.hf_occ = up(occ)
        self.hf_occ_k = up(np.asarray(occ_k).reshape(sh.nk_tot, sh.n_orb, sh.n_orb))
        self.hartree = torch.empty((sh.n_orb, sh.n_orb), dtype=C128, device=dev)
        self.fock = torch.empty((sh.nk_tot, sh.n_orb, sh.n_orb), dtype=C128, device=dev)

    def hartree_fock_stage(self):
        if getattr(self, "hf_occ", None) is None:
            return
        sh = self.sh
        nx, ny, nz = sh.nk
        call("dga_hartree_fock_c128", _p(self.hf_u), _p(self.hf_v), _p(self.hf_occ), _p(self.hf_occ_k), sh.n_orb,
             nx, ny, nz, _p(self.hartree), _p(self.fock), _p(self.sigma), 2 * sh.niv, _s())

    def pre_bse(self):
        """Stages before the BSE: G(R), bubble, double-counting kernel, chi0^-1 and the nu sums."""
        self.status.zero_()
        self.bubble()
        self.dc_kernel()
        self.chi0_prep()

    def post_bse(self):
        """Stages after the BSE: chi_r with shell correction, lambda, kernel assembly, Sigma."""
        self.chi_phys_stage()
        chi_r = self.lambda_stage()
        self.kernel_stage(chi_r)
        self.sigma_stage()
        self.hartree_fock_stage()
        return self.sigma

    def run(self):
        """One device pass over the resident inputs (no host transfers, no synchronisation).  The three phases are
        NVTX ranges (dga.pre_bse, dga.bse, dga.post_bse) for timeline profilers; they cost nothing without one."""
        with torch.cuda.nvtx.range("dga.pre_bse"):
            self.pre_bse()
        with torch.cuda.nvtx.range("dga.bse"):
            self.bse()
        with torch.cuda.nvtx.range("dga.post_bse"):
            return self.post_bse()

    def capture(self) -> "torch.cuda.CUDAGraph":
        """Captures one device pass into a CUDA graph (``replay`` then re-runs all its kernels with one launch).

        Runs the pass once eagerly first, so that kernel attributes and module loading happen outside the
        capture.  The graph reads and writes this pass's own buffers: refresh ``g_k`` in place between replays."""
        self.run()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            self.run()
        torch.cuda.synchronize()
        self.graph = g
        return g

    def replay(self) -> torch.Tensor:
        self.graph.replay()
        return self.sigma

    def run_e2e(self) -> np.ndarray:
        """Host G(k) in, host Sigma(k, nu) out: H2D copy, one pass, D2H copy (synchronises)."""
        self.g_k.copy_(self.g_k_host, non_blocking=True)
        if getattr(self, "graph", None) is not None:
            self.graph.replay()
        else:
            self.run()
        self.sigma_host.copy_(self.sigma, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.sigma_host.numpy()

    def kernels_per_pass(self) -> int:
        """Library kernel launches of one ``run()``: the G(R) transform, bubble, double counting (2), chi0^-1 and
        sums (2); the BSE (mixed: solve + FP64 re-solve); chi_phys, lambda (single band), kernel assembly; the
        Sigma stage's G(R) transform and contraction (wedge: GEMM, partial sums, reduction, inverse transform,
        full-nu; otherwise the partial sums in place of the GEMM and partial sums, after the rotated expansion of K
        when there is one); the Hartree-Fock term when occupations are set."""
        n = 6 + (2 if self.precision == "mixed" else 1) + 2 + (1 if self.do_lambda else 0)
        n += 1 + (5 if self.sh.wedge else 4 + (1 if self.sh.rotated else 0))
        n += 1 if getattr(self, "hf_occ", None) is not None else 0
        return n

    def device_bytes(self) -> int:
        """HBM held by this pass's device tensors, in caching-allocator blocks."""
        return sum(_blk(t.numel() * t.element_size()) for t in vars(self).values()
                   if isinstance(t, torch.Tensor) and t.is_cuda)

    @property
    def h2d_bytes(self) -> int:
        return self.g_k_host.numel() * 16

    @property
    def d2h_bytes(self) -> int:
        return self.sigma_host.numel() * 16

    # ------------------------------------------------------------------------------------------
    # conversions of device intermediates to the upstream layouts (for tests)
    # ------------------------------------------------------------------------------------------
    def chi0_ref_layout(self) -> np.ndarray:
        """[Q][W][nvf][(a,b)][(d,c)] -> [q,a,b,c,d,w,nu]."""
        sh = self.sh
        n = sh.n_orb
        x = self.chi0.cpu().numpy().reshape(sh.n_q, sh.W, sh.nvf, n, n, n, n)  # q w v a b d c
        return x.transpose(0, 3, 4, 6, 5, 1, 2)

    def orbmat_ref_layout(self, t: torch.Tensor) -> np.ndarray:
        """[Q][W][nv][(a,b)][(d,c)] -> [q,a,b,c,d,w,nu]."""
        sh = self.sh
        n = sh.n_orb
        x = t.cpu().numpy().reshape(t.shape[0], t.shape[1], t.shape[2], n, n, n, n)
        return x.transpose(0, 3, 4, 6, 5, 1, 2)

    def x_ref_layout(self, ch: int) -> np.ndarray:
        """X[ch][Q][W][(o1,o2,nu)][(o4,o3)] -> [q,o1,o2,o3,o4,w,nu]."""
        sh = self.sh
        n = sh.n_orb
        x = self.X[ch].cpu().numpy().reshape(sh.n_q, sh.W, n, n, sh.nv, n, n)  # q w o1 o2 nu o4 o3
        return x.transpose(0, 2, 3, 6, 5, 1, 4)

    def chi_phys_ref_layout(self, t: torch.Tensor, ch: int) -> np.ndarray:
        """[2][Q][W][(a,b)][(d,c)] -> [q,a,b,c,d,w]."""
        sh = self.sh
        n = sh.n_orb
        x = t[ch].cpu().numpy().reshape(sh.n_q, sh.W, n, n, n, n)
        return x.transpose(0, 2, 3, 5, 4, 1)
