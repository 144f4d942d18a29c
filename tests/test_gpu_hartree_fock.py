"""Device Hartree-Fock term against the upstream get_hartree_fock (fixtures made by tests/golden/make_golden.py)."""

import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, load_golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ("t1", "t2", "t3"))
def test_hartree_fock_matches_upstream(name):
    from dgamore_b200 import _lib

    d = np.load(os.path.join(GOLDEN, "hartree_fock.npz"))
    nk = tuple(int(x) for x in d[f"{name}_nk"])
    n = d[f"{name}_u"].shape[0]
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).cuda()
    u, v, occ = up(d[f"{name}_u"]), up(d[f"{name}_v_q_full"]), up(d[f"{name}_occ"])
    occ_k = up(d[f"{name}_occ_k"].reshape(-1, n, n))
    h = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    f = torch.empty((int(np.prod(nk)), n, n), dtype=torch.complex128, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.call("dga_hartree_fock_c128", p(u), p(v), p(occ), p(occ_k), n, nk[0], nk[1], nk[2], p(h), p(f), None, 0,
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rel_err(h.cpu().numpy()[None, ..., None], d[f"{name}_hartree"]) < 1e-12
    assert rel_err(f.cpu().numpy()[..., None], d[f"{name}_fock"]) < 1e-12


def test_pass_adds_hartree_fock_to_sigma():
    from dgamore_b200 import synthetic
    from dgamore_b200.pipeline import LadderPass

    inp, _ = load_golden("t2")
    occ, occ_k = synthetic.make_occupations("t2")
    lp = LadderPass(inp, keep_intermediates=False)
    lp.run()
    torch.cuda.synchronize()
    bare = lp.sigma.cpu().numpy()
    lp.set_occupations(occ, occ_k, inp["v_q_full"], inp["u"])
    lp.run()
    torch.cuda.synchronize()
    hf = lp.hartree.cpu().numpy()[None, :, :, None] + lp.fock.cpu().numpy()[..., None]
    assert np.allclose(lp.sigma.cpu().numpy(), bare + hf, rtol=0, atol=1e-13)
