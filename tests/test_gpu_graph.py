"""A whole ladder pass captured in a CUDA graph replays to bitwise the eager result (FP64 and mixed)."""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ("t1", "t2", "t3"))
@pytest.mark.parametrize("precision", ("fp64", "mixed"))
def test_graph_replay_equals_eager(name, precision):
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(name)
    lp = LadderPass(inp, keep_intermediates=False, precision=precision)
    lp.run()
    torch.cuda.synchronize()
    eager = lp.sigma.cpu().numpy()
    lp.capture()
    lp.sigma.zero_()
    for _ in range(2):
        lp.replay()
    torch.cuda.synchronize()
    assert np.array_equal(lp.sigma.cpu().numpy(), eager)
    # end to end through the graph: host G(k) in, host Sigma out
    out = lp.run_e2e()
    assert np.array_equal(out, eager)
    assert rel_err(out, ref["sigma"]) < (1e-10 if precision == "fp64" else 1e-8)
