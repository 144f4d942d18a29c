"""Device-resident local Schwinger-Dyson equation (upstream ``dgamore/local_sde.py:17-217``).

``LocalSde`` runs ``perform_local_schwinger_dyson`` for one atom on the GPU: the local bubble, the generalized
susceptibilities of both channels, the irreducible vertex Gamma_r with the shell correction, the full vertex F_r
over the full box, the auxiliary susceptibility's nu' sum (the ladder BSE at q = 0), the three-leg vertex, the
shell-corrected local susceptibility and the local self-energy.  Its results stay on the device in the layouts
the nonlocal pass reads (``gamma_cm`` is the column-major compound Gamma_r of ``dga_bse_solve_sum_c128``), so the
local vertices reach the nonlocal pass without the upstream's ``.npy`` hand-off (``DGAmore.py:257-277``); the
upstream-layout arrays are produced on request.

Every computation is a libdga_b200 kernel (csrc/local_sde.cu, the dense LU of csrc/bse.cu and the nonlocal
pass's BSE, chi_phys and three-leg-vertex entries at q = 0); the only host arithmetic is the channel
combination of the n^4 interaction tensor.  An exactly singular matrix raises ``numpy.linalg.LinAlgError`` as the
upstream's ``np.linalg.inv`` does; NaN inputs propagate to the results as they do there.

The upstream needs an even niw_core (``pad_with_u`` and ``identity_like`` size the bosonic axis of a half-range
object as 2 * (len // 2) + 1); this form takes any niw_core.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, lib, ll_array
from .pipeline import compound_orb, u_channel

C128 = torch.complex128
DENSE_RHS = 16


def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _s() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=C128).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).to(dev)


def _cols(n_rhs: int) -> int:
    return (n_rhs + DENSE_RHS - 1) // DENSE_RHS * DENSE_RHS


class LocalSde:
    """perform_local_schwinger_dyson (local_sde.py:175-217) of one atom, device resident.

    g: local G [n, n, 2 niv_g]; g2_dens, g2_magn: [n, n, n, n, n_w, 2 niv_core, 2 niv_core] in the full
    (n_w = 2 niw_core + 1) or half (n_w = niw_core + 1) w range; u: U_abcd [n, n, n, n]; occ: [n, n]
    (config.sys.occ_dmft).  Orbital symmetrisation (config.dmft.symmetrize_orbitals) is not part of this form.
    """

    def __init__(self, g, g2_dens, g2_magn, u, beta: float, niw_core: int, niv_core: int, niv_shell: int, occ,
                 device="cuda"):
        lib()  # no CPU fallback
        self.dev = torch.device(device)
        u_np = np.asarray(u.cpu() if isinstance(u, torch.Tensor) else u, dtype=np.complex128)
        self.n = n = u_np.shape[0]
        self.n2 = n2 = n * n
        self.beta = float(beta)
        self.niw, self.niv, self.niv_shell = int(niw_core), int(niv_core), int(niv_shell)
        self.W = self.niw + 1
        self.nv, self.nvf = 2 * self.niv, 2 * (self.niv + self.niv_shell)
        self.N, self.Nf = n2 * self.nv, n2 * self.nvf
        self.g = _dev(g, self.dev)
        self.niv_g = self.g.shape[-1] // 2
        if self.g.shape != (n, n, 2 * self.niv_g):
            raise ValueError(f"g must be [n, n, 2 niv_g], got {tuple(self.g.shape)}")
        if self.niv_g < self.niv + self.niv_shell + self.W:
            raise ValueError(f"G holds {self.niv_g} positive frequencies; the bubble needs niv_core + niv_shell + "
                             f"niw_core + 1 = {self.niv + self.niv_shell + self.W}")
        self.g2 = []
        for g2 in (g2_dens, g2_magn):
            t = _dev(g2, self.dev)
            n_w = t.shape[4]
            if t.shape[:4] != (n,) * 4 or t.shape[5:] != (self.nv, self.nv) or n_w not in (2 * self.niw + 1, self.W):
                raise ValueError(f"G2 of shape {tuple(t.shape)} does not match n={n}, niw_core={self.niw}, "
                                 f"niv_core={self.niv}")
            self.g2.append(t)
        self.u = _dev(u_np, self.dev)
        self.occ = _dev(occ, self.dev)
        uv = np.stack([compound_orb(u_channel(u_np, ch)) for ch in ("dens", "magn")])  # [2][n2][n2]
        self.uv = torch.from_numpy(np.ascontiguousarray(uv)).to(self.dev)
        self._ran = False

    # ------------------------------------------------------------------ the pass
    def run(self) -> "LocalSde":
        """Launches the whole equation on the device (no synchronisation), inside the NVTX range dga.local_sde."""
        with torch.cuda.nvtx.range("dga.local_sde"):
            return self._run()

    def _run(self) -> "LocalSde":
        n, n2, W, N, Nf, nv, nvf = self.n, self.n2, self.W, self.N, self.Nf, self.nv, self.nvf
        dev, beta = self.dev, self.beta
        M = 2 * W
        # local bubble over the full box (half w range) and its inverse / sums over the core box
        self.chi0 = torch.empty((W, nvf, n2, n2), dtype=C128, device=dev)
        call("dga_local_bubble_c128", _p(self.g), n, self.niv_g, W, self.niv + self.niv_shell, beta, _p(self.chi0),
             _s())
        self.chi0_inv = torch.empty((1, W, nv, n2, n2), dtype=C128, device=dev)
        self.full_sum = torch.empty((1, W, n2, n2), dtype=C128, device=dev)
        self.core_sum = torch.empty((1, W, n2, n2), dtype=C128, device=dev)
        self.flags = torch.zeros(4, dtype=torch.int32, device=dev)
        call("dga_chi0_prep_c128", _p(self.chi0), n, self.niv, self.niv_shell, W, 1, beta, _p(self.chi0_inv),
             _p(self.full_sum), _p(self.core_sum), _p(self.flags), _s())
        # generalized susceptibilities (create_generalized_chi) and their inverses
        self.chi_cm = torch.empty((2, W, N, N), dtype=C128, device=dev)
        for ch, g2 in enumerate(self.g2):
            n_w = g2.shape[4]
            w0 = self.niw if n_w == 2 * self.niw + 1 else 0
            call("dga_local_chi_c128", _p(g2), n, self.niv, W, w0, n_w, _p(self.g), self.niv_g, beta,
                 1 if ch == 0 else 0, _p(self.chi_cm[ch]), _s())
        lu = self.chi_cm.clone()
        piv = torch.empty((M, N), dtype=torch.int32, device=dev)
        self.lu_status = torch.zeros(M, dtype=torch.int32, device=dev)
        call("dga_lu_batched_c128", _p(lu), N, M, N * N, _p(piv), _p(self.lu_status), _s())
        cols = _cols(N)
        chi_inv = torch.empty((M, cols, N), dtype=C128, device=dev)
        call("dga_lu_solve_batched_c128", _p(lu), _p(piv), N, M, N * N, None, 0, 0, 0, N, _p(chi_inv), cols * N,
             _p(self.lu_status), _s())
        del lu
        # irreducible vertex with the shell correction (create_gamma_r_with_shell_correction)
        self.ucorr = torch.empty((2, W, n2, n2), dtype=C128, device=dev)
        self.ucorr_status = torch.zeros(M, dtype=torch.int32, device=dev)
        call("dga_local_ucorr_c128", _p(self.uv), _p(self.full_sum), _p(self.core_sum), n, W, _p(self.ucorr),
             _p(self.ucorr_status), _s())
        self.gamma_cm = torch.empty((2, W, N, N), dtype=C128, device=dev)
        call("dga_local_gamma_c128", _p(chi_inv), cols * N, _p(self.chi0_inv), _p(self.ucorr), n, self.niv, W, beta,
             _p(self.gamma_cm), _s())
        del chi_inv
        # full vertex over the full box (create_full_vertex_from_gamma): F^T = (1 + chi0 Gamma_u / beta^2)^-T Gamma_u^T.
        # It depends on Gamma_r only, like the BSE below: it runs on a second stream so that the two sets of
        # single-CTA LUs share the GPU.  Its buffers come from the main stream and are freed after the join.
        mt = torch.empty((M, Nf, Nf), dtype=C128, device=dev)
        gamma_u = torch.empty((M, Nf, Nf), dtype=C128, device=dev)
        pivf = torch.empty((M, Nf), dtype=torch.int32, device=dev)
        self.f_status = torch.zeros(M, dtype=torch.int32, device=dev)
        colsf = _cols(Nf)
        self.f_rm = torch.empty((M, colsf, Nf), dtype=C128, device=dev)  # row c of F at [m][c][:]
        main = torch.cuda.current_stream()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            call("dga_local_fvertex_operands_c128", _p(self.gamma_cm), _p(self.uv), _p(self.chi0), n, self.niv,
                 self.niv_shell, W, beta, _p(mt), _p(gamma_u), _s())
            call("dga_lu_batched_c128", _p(mt), Nf, M, Nf * Nf, _p(pivf), _p(self.f_status), _s())
            call("dga_lu_solve_batched_c128", _p(mt), _p(pivf), Nf, M, Nf * Nf, _p(gamma_u), Nf * Nf, Nf, 1, Nf,
                 _p(self.f_rm), colsf * Nf, _p(self.f_status), _s())
        # auxiliary susceptibility's nu' sum: the ladder BSE at q = 0 with V = 0 (create_auxiliary_chi, create_vrg)
        work = torch.tensor([[ch, 0, w] for ch in range(2) for w in range(W)], dtype=torch.int32, device=dev)
        self.X = torch.empty((2, 1, W, N, n2), dtype=C128, device=dev)
        self.bse_status = torch.zeros(M, dtype=torch.int32, device=dev)
        nbytes = int(lib().dga_bse_scratch_bytes(N, n2, M))
        scratch = torch.empty(nbytes // 16 + 1, dtype=C128, device=dev)
        call("dga_bse_solve_sum_c128", n, self.niv, W, 1, 2, beta, 1.0 / beta**2, _p(self.gamma_cm),
             _p(self.chi0_inv), _p(self.uv), _p(work), M, _p(self.X), _p(self.bse_status), _p(scratch),
             scratch.numel() * 16, _s())
        del scratch
        # shell-corrected susceptibility and three-leg vertex (create_generalized_chi_with_shell_correction, create_vrg)
        self.chi_phys = torch.empty((2, 1, W, n2, n2), dtype=C128, device=dev)
        call("dga_chi_phys_c128", _p(self.X), _p(self.uv), _p(self.full_sum), _p(self.core_sum), n, self.niv, W, 1,
             2, beta, _p(self.chi_phys), _p(self.flags), _s())
        k_dc = torch.zeros((1, W, nv, n2, n2), dtype=C128, device=dev)
        k_out = torch.empty_like(k_dc)
        self.vrg = torch.empty((2, 1, W, nv, n2, n2), dtype=C128, device=dev)
        call("dga_kernel_assembly_c128", _p(self.chi0_inv), _p(self.X), _p(self.uv), _p(self.chi_phys), _p(k_dc), n,
             self.niv, W, 1, beta, _p(k_out), _p(self.vrg), _s())
        del k_dc, k_out
        # local self-energy (get_loc_self_energy_vrg)
        inner = torch.empty((W, nv, n2, n2), dtype=C128, device=dev)
        self.sigma = torch.empty((n, n, nv), dtype=C128, device=dev)
        call("dga_local_sigma_c128", _p(self.vrg), _p(self.chi_phys), _p(self.uv), _p(self.u), _p(self.g),
             _p(self.occ), n, self.niv, W, self.niv_g, beta, _p(inner), _p(self.sigma), _s())
        main.wait_stream(side)
        del mt, gamma_u, pivf
        self._ran = True
        return self

    def check(self) -> None:
        """Raises numpy.linalg.LinAlgError if any inversion met an exactly singular matrix (as np.linalg.inv)."""
        torch.cuda.current_stream().synchronize()
        singular = 1  # DGA_ITEM_SINGULAR
        for name in ("lu_status", "ucorr_status", "f_status", "bse_status"):
            if bool(((getattr(self, name) & singular) != 0).any()):
                raise np.linalg.LinAlgError("Singular matrix")

    # ------------------------------------------------------------------ upstream layouts
    def _copy(self, src: torch.Tensor, shape: tuple, strides: tuple, scale: float = 1.0) -> torch.Tensor:
        dst = torch.empty(shape, dtype=C128, device=self.dev)
        call("dga_strided_copy_c128", _p(src), _p(dst), len(shape), ll_array(shape), ll_array(strides),
             ll_array(list(dst.stride())), scale, _s())
        return dst

    def _four_point(self, src: torch.Tensor, nvb: int, ld: int, row_major: bool) -> torch.Tensor:
        """[a,b,c,d,w,nu,nu'] from compound matrices (p = (a,b), nu) x (s = (d,c), nu') spaced ``ld`` per w."""
        n, N = self.n, self.n2 * nvb
        shape = (n, n, n, n, self.W, nvb, nvb)
        if row_major:  # element (i, j) at i N + j
            st = (n * nvb * N, nvb * N, nvb, n * nvb, ld, N, 1)
        else:  # column-major: (i, j) at j N + i
            st = (n * nvb, nvb, nvb * N, n * nvb * N, ld, 1, N)
        return self._copy(src, shape, st)

    def gchi(self, ch: int) -> torch.Tensor:
        """gchi_r [a,b,c,d,w>=0,nu,nu'] (create_generalized_chi)."""
        return self._four_point(self.chi_cm[ch], self.nv, self.N * self.N, False)

    def gamma(self, ch: int) -> torch.Tensor:
        """Gamma_r [a,b,c,d,w>=0,nu,nu'] (create_gamma_r_with_shell_correction)."""
        return self._four_point(self.gamma_cm[ch], self.nv, self.N * self.N, False)

    def f(self, ch: int) -> torch.Tensor:
        """F_r [a,b,c,d,w>=0,nu,nu'] over the full box (create_full_vertex_from_gamma)."""
        return self._four_point(self.f_rm[ch * self.W], self.nvf, self.f_rm.shape[1] * self.Nf, True)

    def vrg_r(self, ch: int) -> torch.Tensor:
        """gamma_r [a,b,c,d,w>=0,nu] (create_vrg)."""
        n, n2, nv = self.n, self.n2, self.nv
        return self._copy(self.vrg[ch, 0], (n, n, n, n, self.W, nv), (n * n2, n2, 1, n, nv * n2 * n2, n2 * n2))

    def chi(self, ch: int) -> torch.Tensor:
        """chi_r [a,b,c,d,w>=0] (create_generalized_chi_with_shell_correction)."""
        n, n2 = self.n, self.n2
        return self._copy(self.chi_phys[ch, 0], (n, n, n, n, self.W), (n * n2, n2, 1, n, n2 * n2))

    def bubble(self) -> torch.Tensor:
        """chi0 [a,b,c,d,w>=0,nu] over the full box (BubbleGenerator.create_generalized_chi0 in the half w range)."""
        n, n2, nvf = self.n, self.n2, self.nvf
        return self._copy(self.chi0, (n, n, n, n, self.W, nvf), (n * n2, n2, 1, n, nvf * n2 * n2, n2 * n2))

    def sigma_loc(self) -> torch.Tensor:
        """Sigma_loc [1, 1, 1, n, n, 2 niv_core] (get_loc_self_energy_vrg)."""
        return self.sigma.reshape(1, 1, 1, self.n, self.n, self.nv)

    def f_dc(self) -> torch.Tensor:
        """2 F_magn permuted abcd -> cbad [a,b,c,d,w>=0,nu,nu'] over the full box, the double-counting vertex the
        nonlocal pass reads (nonlocal_sde.py:817-819), made on the device from F_magn in one strided copy."""
        n, nvf, Nf = self.n, self.nvf, self.Nf
        ld = self.f_rm.shape[1] * Nf
        # destination (i, j, k, l) takes F_magn[k, j, i, l]: row-major strides of (a, b, c, d) are
        # (n nvf Nf, nvf Nf, nvf, n nvf)
        st = (nvf, nvf * Nf, n * nvf * Nf, n * nvf, ld, Nf, 1)
        return self._copy(self.f_rm[self.W], (n, n, n, n, self.W, nvf, nvf), st, 2.0)

    def chi_loc_sum(self, ch: int) -> complex:
        """sum over orbitals and the full w range of chi_r / beta, the local sum the lambda-correction compares
        with (nonlocal_sde.py:383-392; w < 0 by conjugation, local_n_point.py:191-225)."""
        c = self.chi(ch).cpu().numpy()
        return complex((c.sum() + np.conj(c[..., 1:]).sum()) / self.beta)

    def nonlocal_inputs(self, base: dict) -> dict:
        """``base`` (an input dict of pipeline.LadderPass) with its local vertices replaced by this equation's
        results, kept on the device: gamma_dens / gamma_magn, f_dc and the local susceptibility sums (the
        upstream passes them through gamma_*_loc.npy, f_magn_loc.npy and chi_*_loc.npy, DGAmore.py:257-277)."""
        if not self._ran:
            self.run()
        self.check()
        if (base["niw"], base["niv_core"], base["niv_shell"]) != (self.niw, self.niv, self.niv_shell):
            raise ValueError("the nonlocal pass and the local equation must share the frequency boxes")
        out = dict(base)
        out["gamma_dens"], out["gamma_magn"] = self.gamma(0), self.gamma(1)
        out["f_dc"] = self.f_dc()
        out["chi_loc_sum_dens"], out["chi_loc_sum_magn"] = self.chi_loc_sum(0), self.chi_loc_sum(1)
        return out

    def results(self) -> tuple:
        """The upstream's 11 results as numpy arrays, in its order: gamma_d, gamma_m, chi_d, chi_m, vrg_d, vrg_m,
        f_d, f_m, gchi_d, gchi_m, sigma_loc."""
        if not self._ran:
            self.run()
        self.check()
        out = (self.gamma(0), self.gamma(1), self.chi(0), self.chi(1), self.vrg_r(0), self.vrg_r(1), self.f(0),
               self.f(1), self.gchi(0), self.gchi(1), self.sigma_loc())
        return tuple(x.cpu().numpy() for x in out)


def perform_local_schwinger_dyson(g, g2_dens, g2_magn, u, beta: float, niw_core: int, niv_core: int, niv_shell: int,
                                  occ) -> tuple:
    """Array form of local_sde.perform_local_schwinger_dyson (local_sde.py:175-217): the 11 results as numpy
    arrays in the upstream's order and layouts (half w range)."""
    return LocalSde(g, g2_dens, g2_magn, u, beta, niw_core, niv_core, niv_shell, occ).run().results()
