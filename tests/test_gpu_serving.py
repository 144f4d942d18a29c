"""Heterogeneous batching and the continuous-batching server on the GPU.

A batch launch solves each BSE item with the same device code as a single-request launch, so every result
must be BITWISE equal to the single-request result, whatever else shares the launch; the server's Sigma for
a request must be bitwise the same served alone and in a mix.  The footprint estimate used for admission must
equal the bytes a pass actually allocates.
"""

import numpy as np
import pytest
import torch

from conftest import GOLDEN_CONFIGS, load_golden, rel_err

pytestmark = pytest.mark.gpu

MIX = ("t1", "t1b", "t5e", "t2", "t4e", "t3")


def _single(name, precision):
    from dgamore_b200.pipeline import LadderPass

    inp, ref = load_golden(name)
    lp = LadderPass(inp, precision=precision, keep_intermediates=False)
    lp.run()
    torch.cuda.synchronize()
    return inp, ref, lp.X.cpu().numpy(), lp.sigma.cpu().numpy()


@pytest.fixture(scope="module", params=["fp64", "mixed"])
def singles(request):
    return request.param, {n: _single(n, request.param) for n in MIX}


def test_batch_launch_is_bitwise_the_single_launch(singles):
    from dgamore_b200.pipeline import LadderPass
    from dgamore_b200.serving import solve_bse_batch

    precision, ref = singles
    passes = [LadderPass(ref[n][0], precision=precision, keep_intermediates=False, own_bse_scratch=False) for n in MIX]
    for lp in passes:
        lp.pre_bse()
    solve_bse_batch(passes, precision)
    for lp in passes:
        lp.post_bse()
    torch.cuda.synchronize()
    for n, lp in zip(MIX, passes):
        assert int(lp.bse_status.abs().sum()) == 0, n
        assert np.array_equal(lp.X.cpu().numpy(), ref[n][2]), n
        assert np.array_equal(lp.sigma.cpu().numpy(), ref[n][3]), n
        # and the batch result is the upstream's
        sigma_ref = ref[n][1]["sigma"]
        tol = 1e-10 if precision == "fp64" else 1e-8
        assert rel_err(lp.sigma.cpu().numpy(), sigma_ref) < tol, n


def test_partial_batches_cover_each_item_once():
    """Items of one pass split over several launches (the server's chunking) give the same X."""
    from dgamore_b200.pipeline import LadderPass
    from dgamore_b200.serving import BseBatch

    inp, _, x_ref, _ = _single("t1b", "fp64")
    inp3, _, x3_ref, _ = _single("t5e", "fp64")
    a = LadderPass(inp, keep_intermediates=False, own_bse_scratch=False)
    b = LadderPass(inp3, keep_intermediates=False, own_bse_scratch=False)
    for lp in (a, b):
        lp.pre_bse()
        lp.X.zero_()
    scratch = torch.empty((64 << 20) // 16, dtype=torch.complex128, device="cuda")
    dev = a.dev
    for lo in range(0, max(a.n_items, b.n_items), 7):
        items = [(lp, torch.arange(lo, min(lo + 7, lp.n_items), device=dev)) for lp in (a, b) if lo < lp.n_items]
        BseBatch(items, "fp64").launch(scratch)
    torch.cuda.synchronize()
    assert np.array_equal(a.X.cpu().numpy(), x_ref)
    assert np.array_equal(b.X.cpu().numpy(), x3_ref)


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
@pytest.mark.parametrize("keep", [False, True])
def test_footprint_estimate_equals_allocations(name, keep):
    from dgamore_b200.pipeline import LadderPass, estimate_device_bytes

    inp, _ = load_golden(name)
    for precision in ("fp64", "mixed"):
        lp = LadderPass(inp, precision=precision, keep_intermediates=keep, own_bse_scratch=False)
        assert lp.device_bytes() == estimate_device_bytes(lp.sh, precision, keep), (name, precision)


def test_server_mix_is_bitwise_alone_and_respects_the_budget():
    from dgamore_b200.pipeline import PassShapes, estimate_device_bytes
    from dgamore_b200.serving import LadderServer, Request, poisson_arrivals

    names = ("t1b", "t2", "t1", "t3", "t5e", "t4e", "t1b", "t2")
    inputs = {n: load_golden(n)[0] for n in set(names)}
    feet = {n: estimate_device_bytes(PassShapes.from_inputs(inputs[n])) for n in inputs}
    budget = int(2.5 * max(feet.values()))
    arrivals = poisson_arrivals(len(names), rate_per_s=50.0, seed=7)
    reqs = [Request(inputs[n], arrival=float(t)) for n, t in zip(names, arrivals)]
    srv = LadderServer(hbm_budget=budget, scratch_bytes=128 << 20, items_per_request=5)
    stats = srv.serve(reqs, realtime=True)
    assert len(stats.completed) == len(names)
    assert stats.peak_admitted_bytes <= budget
    assert stats.iterations > 1
    summary = stats.summary()
    assert summary["p99_s"] >= summary["p50_s"] > 0
    alone = {}
    for n in inputs:
        solo = LadderServer(hbm_budget=budget, scratch_bytes=128 << 20, items_per_request=None)
        (r,) = solo.serve([Request(inputs[n])], realtime=False).completed
        alone[n] = r.sigma
        _, _, _, sigma_single = _single(n, "fp64")
        assert np.array_equal(r.sigma, sigma_single), n
    for n, r in zip(names, reqs):
        assert int(np.abs(r.bse_status).sum()) == 0
        assert np.array_equal(r.sigma, alone[n]), n


def test_server_mixed_precision_requests():
    from dgamore_b200.serving import LadderServer, Request

    names = ("t1b", "t5e", "t1")
    reqs = [Request(load_golden(n)[0], precision="mixed") for n in names]
    srv = LadderServer(hbm_budget=8 << 30, scratch_bytes=128 << 20, items_per_request=11)
    srv.serve(reqs, realtime=False)
    for n, r in zip(names, reqs):
        _, ref, _, sigma_single = _single(n, "mixed")
        assert np.array_equal(r.sigma, sigma_single), n
        assert rel_err(r.sigma, ref["sigma"]) < 1e-8
