"""Device Eliashberg stage: full ladder vertex -> pairing vertices -> gap-equation operator -> leading eigenpairs.

Mirrors ``dgamore/eliashberg_solver.py``:

* ``solve`` (eliashberg_solver.py:584-752) without the optional local part (``include_local_part``, off in the
  upstream's shipped configuration): F_dens, F_magn in the pp box (niv_pp = min(niw//2, niv//2)), the singlet and
  triplet pairing vertices and the leading ``n_eig`` eigenpairs of each channel;
* ``solve_eliashberg_lanczos`` (eliashberg_solver.py:376-471): the upstream calls ``scipy.sparse.linalg.eigsh``
  on a complex operator, which SciPy routes to ARPACK's non-Hermitian Arnoldi (``eigs`` with which='LR') and
  returns the real parts; here the same eigenproblem is solved by a Krylov-Schur restarted Arnoldi iteration
  (G. W. Stewart, SIAM J. Matrix Anal. Appl. 23, 601 (2001)) with the operator applied by
  ``dga_eli_matvec_c128`` on the device, FP64 throughout, and the same start vector construction.

The full vertex comes from the pass itself when it was built with ``LadderPass(..., eliashberg_pp=niv_pp)``: its
FP64 BSE then solves the pp-box unit vectors with each item's own LU factors (``dga_bse_solve_sum_eli_c128``) and
this stage only adds the ladder term (``dga_eli_ladder_term_c128``), instead of factorising every (q, w < 2 niv_pp)
item a second time (``dga_eli_full_vertex_c128``, the path for passes built without it).

Every vertex and operator stage is a libdga_b200 kernel; torch provides device memory and the small vector
algebra of the Arnoldi basis.
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.linalg as sla
import torch

from ._lib import call, lib, ll_array
from .pipeline import LadderPass, _p, _s

C128 = torch.complex128


def default_niv_pp(niw: int, niv: int) -> int:
    """niv_pp = min(niw // 2, niv // 2) (eliashberg_solver.py:598)."""
    return min(niw // 2, niv // 2)


def initial_gap(nk: tuple, n_bands: int, niv_pp: int, channel: str, symmetry: str, irrk_ind, irrk_inv,
                rng: np.random.Generator | None = None) -> np.ndarray:
    """Start vector of the eigen-solve (eliashberg_solver.py:339-372, 405-410): d-wave / p-wave-x / p-wave-y
    with the channel's frequency parity, or random; stored as complex64 like the upstream, then symmetrised
    over the irreducible wedge.  Returns [kx, ky, kz, n, n, 2 niv_pp] complex128."""
    shape = (*nk, n_bands, n_bands, 2 * niv_pp)
    kx = np.linspace(0, 2 * np.pi, nk[0], endpoint=False)
    ky = np.linspace(0, 2 * np.pi, nk[1], endpoint=False)
    forms = {
        "d-wave": lambda: -np.cos(kx)[:, None, None] + np.cos(ky)[None, :, None],
        "p-wave-x": lambda: np.sin(kx)[:, None, None] + 0 * ky[None, :, None],
        "p-wave-y": lambda: np.sin(ky)[None, :, None] + 0 * kx[:, None, None],
    }
    gap = np.zeros(shape, dtype=np.complex64)
    if symmetry in forms:
        sym = forms[symmetry]()
        gap[..., niv_pp:] = np.repeat(sym[:, :, :, None, None, None], niv_pp, axis=-1)
        even = {"d-wave": channel == "sing", "p-wave-x": channel != "sing", "p-wave-y": channel != "sing"}[symmetry]
        gap[..., :niv_pp] = gap[..., niv_pp:] if even else -gap[..., niv_pp:]
    else:
        rng = rng if rng is not None else np.random.default_rng(0)
        gap = rng.random(shape)
    flat = gap.reshape(int(np.prod(nk)), *shape[3:])
    return flat[np.asarray(irrk_ind)][np.asarray(irrk_inv)].reshape(shape).astype(np.complex128)


class EliashbergSolver:
    """Pairing vertices and gap-equation operators of one request, resident on the device."""

    def __init__(self, lp: LadderPass, niv_pp: int | None = None, precision: str = "fp64"):
        """precision 'fp64': Gamma(R) in complex128; 'mixed': Gamma(R) stored in complex64 (half the bytes the
        operator streams), with FP64 products, sums, vectors and normalisation."""
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        self.precision = precision
        if lp.gamma3 is None:
            raise ValueError("the Eliashberg stage needs the three-leg vertex: build LadderPass(keep_intermediates=True)")
        self.lp = lp
        sh = lp.sh
        self.P = int(niv_pp if niv_pp is not None else default_niv_pp(sh.niw, sh.niv))
        if self.P <= 0 or 2 * self.P > sh.W:
            raise ValueError(f"niv_pp={self.P} needs 1 <= 2 niv_pp <= niw + 1")
        n, n2, P, Q = sh.n_orb, sh.n2, self.P, sh.n_q
        self.M = n2 * 2 * P
        M = self.M
        self.w_pp = 2 * P
        dev = lp.dev
        chi_r = lp.chi_lam if lp.do_lambda else lp.chi_phys
        work = [(ch, q, w) for w in range(self.w_pp) for ch in range(2) for q in range(Q)]
        self.work = torch.tensor(work, dtype=torch.int32, device=dev)
        n_items = len(work)
        self.fused = bool(getattr(lp, "f_pp_ready", False)) and lp.eli_P == P
        if self.fused:
            # the pass's FP64 BSE already wrote the chi* part of the vertex from its own LU factors: add the
            # ladder term in place (the buffer is consumed) instead of factorising every item again
            fph = lp.f_pp
            call("dga_eli_ladder_term_c128", _p(lp.uv), _p(lp.gamma3), _p(chi_r), n, sh.niv, sh.W, Q, P, self.w_pp,
                 _p(fph), _s())
            lp.f_pp_ready = False
            self.vertex_status = lp.bse_status.clone()
        else:
            self.vertex_status = torch.zeros(n_items, dtype=torch.int32, device=dev)
            sbytes = int(lib().dga_eli_vertex_scratch_bytes(n, sh.niv, P, n_items))
            scratch = torch.empty(sbytes // 16 + 1, dtype=C128, device=dev)
            fph = torch.empty((2, Q, self.w_pp, M, M), dtype=C128, device=dev)
            call("dga_eli_full_vertex_c128", n, sh.niv, sh.W, Q, P, self.w_pp, sh.beta, lp.inv_beta2,
                 _p(lp.gamma_cm), _p(lp.chi0_inv), _p(lp.uv), _p(lp.gamma3), _p(chi_r), _p(self.work), n_items,
                 _p(fph), _p(self.vertex_status), _p(scratch), scratch.numel() * 16, _s())
            del scratch
        self.gamma_pp_irr = torch.empty((2, Q, M, M), dtype=C128, device=dev)
        call("dga_eli_pairing_vertex_c128", _p(fph), n, P, Q, self.w_pp, _p(self.gamma_pp_irr), _s())
        if not self.fused:
            del fph
        # Gamma(R) = sign * FFT_q of the pairing vertex expanded to the full zone (eliashberg_solver.py:392-396)
        nx, ny, nz = sh.nk
        self.mat = torch.empty((2, sh.nk_tot, M, M), dtype=C128, device=dev)
        full = torch.empty((sh.nk_tot, M, M), dtype=C128, device=dev) if sh.rotated else None
        for st, sign in ((0, 1.0), (1, -1.0)):
            src, gather = self.gamma_pp_irr[st], lp.irrk_inv
            if sh.rotated:
                # auto-mode symmetries: each zone point's orbital rotation (U on the upstream positions o1, o3 =
                # rows a, b; U* on o2, o4 = columns c, d of Mat[(a,b,nu)][(c,d,nu')] = Gamma[a,c,b,d])
                P2 = 2 * P
                call("dga_fbz_rotate_c128", _p(src), _p(lp.irrk_inv), sh.nk_tot, _p(lp.rot_us), _p(lp.rot_sigmas),
                     _p(lp.rot_conjs), n, ll_array([n * P2 * M, n * P2, P2 * M, P2]), M, P2, 1, P2, M * M, _p(full),
                     _s())
                src, gather = full, lp.rot_ident
            call("dga_dft_planes_gather_c128", _p(src), 1, 0, M * M, _p(self.mat[st]), 1, 0, M * M,
                 1, M * M, nx, ny, nz, _p(lp.tw_fwd), sign, _p(gather), _s())
        del full
        if precision == "mixed":
            mat64 = torch.empty((2, sh.nk_tot, M, M), dtype=torch.complex64, device=dev)
            call("dga_narrow_c128_to_c64", _p(self.mat), _p(mat64), self.mat.numel(), _s())
            self.mat = mat64
        self.chi0pp = torch.empty((sh.nk_tot, 2 * P, n2, n2), dtype=C128, device=dev)
        call("dga_eli_chi0pp_c128", _p(lp.g_k), n, sh.niv_g, P, sh.nk_tot, _p(self.chi0pp), _s())
        self.mv_scratch = torch.empty(int(lib().dga_eli_matvec_scratch_bytes(n, P, sh.nk_tot)) // 16 + 1, dtype=C128,
                                      device=dev)
        self.dim = sh.nk_tot * M
        self.n_matvec = 0

    # --------------------------------------------------------------------------------------------
    def matvec(self, channel: str, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """out = A_channel x for a gap vector x [Nk * n2 * 2P] (layout [k][(a,b)][nu])."""
        sh = self.lp.sh
        st, sign = (0, 1.0) if channel == "sing" else (1, -1.0)
        x = x.contiguous()
        out = torch.empty_like(x) if out is None else out
        nx, ny, nz = sh.nk
        entry = "dga_eli_matvec_c64mat_c128" if self.precision == "mixed" else "dga_eli_matvec_c128"
        call(entry, _p(self.mat[st]), _p(self.chi0pp), _p(x), sh.n_orb, self.P, nx, ny, nz,
             _p(self.lp.tw_fwd), _p(self.lp.tw_inv), sh.beta, sign, _p(out), _p(self.mv_scratch),
             self.mv_scratch.numel() * 16, _s())
        self.n_matvec += 1
        return out

    def eigs(self, channel: str, n_eig: int = 4, tol: float = 1e-6, v0: np.ndarray | None = None,
             ncv: int | None = None, max_restarts: int = 1000):
        """Leading n_eig eigenpairs by largest real part of the channel's gap-equation operator.

        Returns (real parts of the eigenvalues in descending order, eigenvectors [n_eig, Nk*n2*2P], status 0 if
        converged to |residual| <= tol |theta| else DGA_ITEM_NOCONVERGE = 4)."""
        if v0 is None:
            v0 = np.random.default_rng(0).random(self.dim)
        x = torch.as_tensor(np.ascontiguousarray(v0, dtype=np.complex128).ravel(), device=self.lp.dev)
        out = torch.empty_like(x)
        return krylov_schur(lambda v: self.matvec(channel, v, out), x, n_eig, tol, ncv, max_restarts)

    # --------------------------------------------------------------------------------------------
    def solve(self, n_eig: int = 4, tol: float = 1e-6, symmetry: str = "random", seed: int = 0):
        """Leading eigenvalues and gap functions of the singlet and triplet channels (eliashberg_solver.py:584-752).

        Returns (lambdas_sing, lambdas_trip, gaps_sing, gaps_trip) with gaps [n_eig][kx,ky,kz,n,n,2 niv_pp]."""
        sh = self.lp.sh
        out = {}
        rng = np.random.default_rng(seed)
        for ch in ("sing", "trip"):
            g0 = initial_gap(sh.nk, sh.n_orb, self.P, ch, symmetry, self.irrk_ind_host, self.irrk_inv_host, rng)
            with torch.cuda.nvtx.range(f"dga.eliashberg.{ch}"):
                vals, vecs, status = self.eigs(ch, n_eig, tol, g0.ravel())
            gaps = [v.reshape(*sh.nk, sh.n_orb, sh.n_orb, 2 * self.P) for v in vecs]
            out[ch] = (vals, gaps, status)
        self.status = {ch: out[ch][2] for ch in out}
        return out["sing"][0], out["trip"][0], out["sing"][1], out["trip"][1]

    @property
    def irrk_ind_host(self):
        return np.asarray(self.lp.irrk_ind_host)

    @property
    def irrk_inv_host(self):
        return self.lp.irrk_inv.cpu().numpy()

    # conversions for tests -----------------------------------------------------------------------
    def pairing_vertex_ref_layout(self, st: int) -> np.ndarray:
        """[Q][(a,b,nu)][(c,d,nu')] -> upstream [q,a,b,c,d,nu,nu'] (with Mat = Gamma[a,c,b,d])."""
        sh = self.lp.sh
        n, nvp = sh.n_orb, 2 * self.P
        x = self.gamma_pp_irr[st].cpu().numpy().reshape(sh.n_q, n, n, nvp, n, n, nvp)  # q a b nu c d nu'
        # Gamma[o1,o2,o3,o4] = x[a=o1, b=o3, nu, c=o2, d=o4, nu']
        return x.transpose(0, 1, 4, 2, 5, 3, 6)


def krylov_schur(matvec, v0: torch.Tensor, k: int, tol: float = 1e-6, ncv: int | None = None,
                 max_restarts: int = 1000):
    """Eigenvalues of largest real part of a (possibly non-Hermitian) operator by the Krylov-Schur method
    (G. W. Stewart, SIAM J. Matrix Anal. Appl. 23, 601 (2001)): Arnoldi steps with classical Gram-Schmidt and
    one re-orthogonalisation (Daniel-Gragg-Kaufman-Stewart), a sorted Schur form of the projected matrix and
    thick restarts that keep the wanted Schur vectors.  Vectors live on v0's device; the small projected
    problems are solved on the host in FP64.  The same problem ARPACK's znaupd solves for eigs(which='LR').

    Returns (real parts of the k wanted eigenvalues, descending; eigenvectors [k, dim] as numpy; status 0 when
    every wanted Ritz pair has |residual| <= tol |theta|, else 4).
    """
    dim = v0.numel()
    m = int(ncv if ncv is not None else max(2 * k + 1, 20))
    m = max(min(m, dim), min(k + 1, dim))
    dev, dt = v0.device, v0.dtype
    V = torch.zeros((m + 1, dim), dtype=dt, device=dev)
    V[0] = v0 / torch.linalg.vector_norm(v0)
    H = np.zeros((m + 1, m), dtype=np.complex128)
    j0 = 0
    m_eff = m
    for _ in range(max_restarts):
        m_eff = m
        for j in range(j0, m):
            w = matvec(V[j]).clone()
            h = torch.mv(V[: j + 1].conj(), w)
            w -= torch.mv(V[: j + 1].T, h)
            h2 = torch.mv(V[: j + 1].conj(), w)
            w -= torch.mv(V[: j + 1].T, h2)
            H[: j + 1, j] = (h + h2).cpu().numpy()
            beta = float(torch.linalg.vector_norm(w).item())
            H[j + 1, j] = beta
            if beta <= 1e-300:  # invariant subspace: the projected matrix is exact
                m_eff = j + 1
                break
            V[j + 1] = w / beta
        Hm = H[:m_eff, :m_eff]
        ev_all = np.linalg.eigvals(Hm)
        kk = min(k, m_eff)
        cut = np.sort(ev_all.real)[::-1][kk - 1]
        T, Z, p = sla.schur(Hm, output="complex", sort=lambda z: z.real >= cut - 1e-14 * max(1.0, abs(cut)))
        p = int(max(min(p, m_eff - 1 if m_eff > kk else m_eff), kk))
        r = H[m_eff, m_eff - 1] * Z[m_eff - 1, :]  # coupling of the Schur vectors to the next Arnoldi vector
        ev, Y = np.linalg.eig(T[:p, :p])
        Y = Y / np.linalg.norm(Y, axis=0)
        res = np.abs(r[:p] @ Y)
        order = np.argsort(-ev.real)[:kk]
        converged = bool(np.all(res[order] <= tol * np.maximum(np.abs(ev[order]), 1e-300))) or m_eff < m
        if converged or _ == max_restarts - 1:
            coef = Z[:, :p] @ Y[:, order]  # [m_eff, kk]
            vecs = torch.as_tensor(coef.T.copy(), device=dev, dtype=dt) @ V[:m_eff]
            return ev.real[order], vecs.cpu().numpy(), 0 if converged else 4
        # thick restart with the p leading Schur vectors
        V[:p] = torch.as_tensor(Z[:, :p].T.copy(), device=dev, dtype=dt) @ V[:m_eff]
        V[p] = V[m_eff]
        H = np.zeros((m + 1, m), dtype=np.complex128)
        H[:p, :p] = T[:p, :p]
        H[p, :p] = r[:p]
        j0 = p
    raise RuntimeError("unreachable")
