"""The block-form mixed BSE (kernel choice 4) at compound sizes that are not multiples of its 32 x 32 blocks.

The factorisation takes its steps in pairs (one K = 64 trailing product for two steps) wherever both blocks are full
and a trailing matrix follows them, and single K = 32 steps elsewhere: at the end of the matrix, before a ragged
last block and for an odd number of blocks.  These cases reach each of those forms:

* 1 orbital, niv = 50: N = 100 = 3 x 32 + 4 (one pair, then two single steps, the last 4 wide);
* 2 orbitals, niv = 33: N = 264 = 8 x 32 + 8 (four pairs, a single step before the ragged block);
* 3 orbitals, niv = 12: N = 216 = 6 x 32 + 24 (three pairs, the ragged block alone);
* 3 orbitals, niv = 16: N = 288 = 9 x 32 (four pairs and one single full step at the end).

Each mixed solve, refined to 1e-12, matches the FP64 drop-in BSE of the same inputs to 1e-10 relative.
"""

import dataclasses

import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu

CASES = [("c4_single", 50, 100), ("c4_bilayer", 33, 264), ("c3", 12, 216), ("c3", 16, 288)]


@pytest.mark.parametrize("name,niv,n_compound", CASES)
def test_block_kernel_matches_fp64(name, niv, n_compound):
    from dgamore_b200 import synthetic
    from dgamore_b200.pipeline import LadderPass

    cfg = dataclasses.replace(synthetic.CONFIGS[name], name=f"{name}_niv{niv}", nk=(4, 4, 1), niw=2, niv=niv)
    inp = synthetic.make_inputs(cfg)
    ref = LadderPass(inp, keep_intermediates=False)
    assert ref.sh.N == n_compound
    ref.pre_bse()
    ref.bse()
    torch.cuda.synchronize()
    x64 = [ref.x_ref_layout(ch) for ch in (0, 1)]
    assert int(ref.bse_status.abs().sum()) == 0
    del ref

    lp = LadderPass(inp, keep_intermediates=False, precision="mixed", refine_tol=1e-12)
    lp.pre_bse()
    lp.set_tuning((4, 0))
    lp.bse()
    torch.cuda.synchronize()
    assert int(lp.bse_status.abs().sum()) == 0
    for ch in (0, 1):
        assert rel_err(lp.x_ref_layout(ch), x64[ch]) < 1e-10, ch
