"""Array-level mirror of the FourPoint BSE entry points (dgamore/four_point.py:590-684) on the device.

``invert_and_sum_over_last_vn(mat, beta)`` takes the explicit compound matrix of a FourPoint with two
fermionic frequency dimensions in the upstream layout ``[q, o1, o2, o3, o4, w, nu, nu']`` (half w range,
as the upstream converts with ``to_half_niw_range``) and returns ``[q, o1, o2, o3, o4, w, nu]`` =
``sum_nu' A^-1 / beta``, exactly what the upstream method stores in ``self.mat``.  The ``_v2`` name (the linear
solve against the n^2 selector right-hand sides, four_point.py:644-684) computes the same result and maps to
the same kernel.  Errors mirror the upstream: a wrong number of fermionic dimensions raises
``NotImplementedError`` (four_point.py:624-625); an exactly singular matrix raises ``numpy.linalg.LinAlgError``.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, lib


def _as_device(x) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=torch.complex128).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).cuda()


def invert_and_sum_over_last_vn(mat, beta: float, return_device: bool = False):
    """sum_nu' [A^-1]_{(o1,o2,nu),(o4,o3,nu')} / beta for every (q, w) (four_point.py:620-642)."""
    lib()
    if mat.ndim != 8:
        raise NotImplementedError("Method only implemented for objects with two fermionic frequency dimensions.")
    nq, nb, w_dim, nv = mat.shape[0], mat.shape[1], mat.shape[5], mat.shape[6]
    if mat.shape[1:5] != (nb,) * 4 or mat.shape[7] != nv or nv % 2:
        raise ValueError(f"unexpected FourPoint shape {tuple(mat.shape)}")
    n2, N = nb * nb, nb * nb * nv
    a = _as_device(mat)
    work = torch.tensor([(0, q, w) for q in range(nq) for w in range(w_dim)], dtype=torch.int32, device="cuda")
    n_items = work.shape[0]
    out = torch.empty((nq, w_dim, N, n2), dtype=torch.complex128, device="cuda")
    status = torch.zeros(n_items, dtype=torch.int32, device="cuda")
    sbytes = int(lib().dga_bse_scratch_bytes(N, n2, n_items))
    scratch = torch.empty(sbytes // 16 + 1, dtype=torch.complex128, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    call("dga_invert_sum_dense_c128", nb, nv // 2, w_dim, nq, float(beta), ctypes.c_void_p(a.data_ptr()),
         ctypes.c_void_p(work.data_ptr()), n_items, ctypes.c_void_p(out.data_ptr()),
         ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(scratch.data_ptr()), scratch.numel() * 16, stream)
    if int((status & 1).sum().item()):
        raise np.linalg.LinAlgError("Singular matrix")
    res = out.reshape(nq, w_dim, nb, nb, nv, nb, nb).permute(0, 2, 3, 6, 5, 1, 4)  # q o1 o2 o3 o4 w nu
    if return_device:
        return res.contiguous()
    return res.cpu().numpy()


invert_and_sum_over_last_vn_v2 = invert_and_sum_over_last_vn
