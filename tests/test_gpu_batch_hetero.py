"""Requests of different orbital counts in ONE persistent BSE launch, and the whole schedule in one CUDA graph.

``serving.BatchedPasses`` runs the pre-BSE stages of every request, one batch launch over all their BSE items
(the 128-thread kernels pick the right-hand-side count per item, so a 2-orbital and a 1-orbital request share
it), and the post-BSE stages.  Each item runs the same per-item code as in a single-request launch, so X and Sigma
must be BITWISE the single-request results, eagerly and replayed from the captured graph.
"""

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

MIXES = (("t4e", "t1b"), ("t2", "t5e", "t3"))  # 2 + 1 orbitals; 2 + 1 + 3 orbitals


def _single(name, precision):
    from dgamore_b200.pipeline import LadderPass

    inp, _ = load_golden(name)
    lp = LadderPass(inp, precision=precision, keep_intermediates=False)
    lp.run()
    torch.cuda.synchronize()
    return inp, lp.X.cpu().numpy(), lp.sigma.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mix", MIXES)
def test_mixed_orbital_batch_is_one_launch_and_bitwise(mix, precision):
    from dgamore_b200.pipeline import LadderPass
    from dgamore_b200.serving import BatchedPasses

    singles = {n: _single(n, precision) for n in mix}
    passes = [LadderPass(singles[n][0], precision=precision, keep_intermediates=False, own_bse_scratch=False)
              for n in mix]
    assert len({lp.sh.n_orb for lp in passes}) > 1
    bp = BatchedPasses(passes, precision)
    assert len(bp.batches) == 1  # one persistent launch over every request's items
    bp.run()
    torch.cuda.synchronize()
    for n, lp in zip(mix, passes):
        assert int(lp.bse_status.abs().sum()) == 0, n
        assert np.array_equal(lp.X.cpu().numpy(), singles[n][1]), n
        assert np.array_equal(lp.sigma.cpu().numpy(), singles[n][2]), n
    bp.capture()
    for lp in passes:
        lp.X.zero_()
        lp.sigma.zero_()
    bp.replay()
    torch.cuda.synchronize()
    for n, lp in zip(mix, passes):
        assert np.array_equal(lp.X.cpu().numpy(), singles[n][1]), n
        assert np.array_equal(lp.sigma.cpu().numpy(), singles[n][2]), n
