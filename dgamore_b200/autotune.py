"""Autotuner for the BSE launch choices (``dga_bse_tuning``: kernel and CTAs per SM).

The best launch depends on the compound size N and the number of work items: the shared-memory-panel kernel
(one 512-thread CTA per SM, mixed form only) wins for the 3-orbital sizes, while for small N the 128-thread
kernel with several CTAs per SM keeps more items in flight.  ``tune_bse`` times every candidate the library
accepts for a pass's shape on a sample of its real work items (CUDA events on the pass's stream, best of
``repeats`` after one warm-up launch), keeps the fastest, and caches the choice per (device, shape,
precision) in memory and, if given, in a JSON file, so that later passes of the same shape skip the search.
Every candidate computes the same solves, so the choice affects speed only.
"""

from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass

import torch

from ._lib import BseTuning, call, lib

C128 = torch.complex128

# (kernel, ctas_per_sm): kernel 1 = shared-memory panel (mixed only), 2 = 128-thread kernel, 3 = shared-memory
# panel with tensor-core trailing tiles (mixed only), 4 = block form with pivoting inside 32 x 32 diagonal blocks
# and every update on the tensor cores (mixed only)
CANDIDATES = {
    "mixed": [(4, 0), (3, 0), (1, 0), (2, 0), (2, 2), (2, 1)],
    "fp64": [(2, 0), (2, 2), (2, 1)],
}

_CACHE: dict[str, tuple[int, int]] = {}


@dataclass
class TuneResult:
    key: str
    choice: tuple
    times_ms: dict
    sample_items: int


def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _s() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def shape_key(lp, precision: str) -> str:
    sh = lp.sh
    name = torch.cuda.get_device_name(lp.dev)
    return f"{name}|n_orb={sh.n_orb}|niv={sh.niv}|W={sh.W}|Q={sh.n_q}|{precision}"


def tuning_struct(choice) -> BseTuning:
    return BseTuning(kernel=int(choice[0]), ctas_per_sm=int(choice[1]))


def scratch_bytes(lp, n_items: int, mixed: int, choice) -> int:
    sh = lp.sh
    t = tuning_struct(choice)
    return int(lib().dga_bse_tuned_scratch_bytes(sh.N, sh.n2, n_items, mixed, ctypes.byref(t)))


def launch(lp, work: torch.Tensor, n_items: int, mixed: int, choice, scratch: torch.Tensor,
           status: torch.Tensor, iters: torch.Tensor) -> None:
    sh = lp.sh
    t = tuning_struct(choice)
    call("dga_bse_solve_sum_tuned_c128", sh.n_orb, sh.niv, sh.W, sh.n_q, 2, sh.beta, lp.inv_beta2, _p(lp.gamma_cm),
         _p(lp.chi0_inv), _p(lp.uv), _p(work), n_items, mixed, lp.refine_max_iter, lp.refine_tol, _p(lp.X),
         _p(status), _p(iters), ctypes.byref(t), _p(scratch), scratch.numel() * 16, _s())


def load_cache(path: str | None) -> None:
    if path and os.path.exists(path):
        with open(path) as f:
            for k, v in json.load(f).items():
                _CACHE[k] = tuple(v)


def save_cache(path: str | None) -> None:
    if not path:
        return
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump({k: list(v) for k, v in _CACHE.items()}, f, indent=1, sort_keys=True)


def tune_bse(lp, precision: str | None = None, sample_items: int | None = None, repeats: int = 2,
             cache_path: str | None = None, force: bool = False) -> TuneResult:
    """Chooses the BSE launch for ``lp`` (a LadderPass whose chi0^-1 is computed: run ``lp.pre_bse()`` first)
    and installs it with ``lp.set_tuning``.  Overwrites ``lp.X`` for the sampled items."""
    precision = precision or lp.precision
    mixed = 1 if precision == "mixed" else 0
    key = shape_key(lp, precision)
    load_cache(cache_path)
    if not force and key in _CACHE:
        lp.set_tuning(_CACHE[key])
        return TuneResult(key, _CACHE[key], {}, 0)
    sms = torch.cuda.get_device_properties(lp.dev).multi_processor_count
    n = lp.n_items if sample_items is None else min(lp.n_items, sample_items)
    if sample_items is None:
        n = min(lp.n_items, 6 * sms)
    work = lp.work[:n].contiguous()
    status = torch.zeros(n, dtype=torch.int32, device=lp.dev)
    iters = torch.zeros(n, dtype=torch.int32, device=lp.dev)
    cands = [c for c in CANDIDATES[precision] if scratch_bytes(lp, n, mixed, c) > 0]
    need = max(scratch_bytes(lp, n, mixed, c) for c in cands)
    scratch = torch.empty(need // 16 + 1, dtype=C128, device=lp.dev)
    stream = torch.cuda.current_stream()
    times = {}
    for c in cands:
        launch(lp, work, n, mixed, c, scratch, status, iters)  # warm-up (also sets the kernel attributes)
        best = float("inf")
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            launch(lp, work, n, mixed, c, scratch, status, iters)
            b.record(stream)
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        clean = int(status.abs().sum()) == 0
        times[c] = (best, clean)
    del scratch
    # the fastest candidate whose sampled items all came back clean (a flagged item costs an FP64 re-solve)
    ok = {c: t for c, (t, clean) in times.items() if clean} or {c: t for c, (t, _) in times.items()}
    choice = min(ok, key=ok.get)
    times = {c: t for c, (t, _) in times.items()}
    _CACHE[key] = choice
    save_cache(cache_path)
    lp.set_tuning(choice)
    return TuneResult(key, choice, {f"{k[0]}/{k[1]}": v for k, v in times.items()}, n)


# wedge-Sigma launch choices: (GEMM output tile of dga_sigma_wedge_c128 (0 = 64 x 64, 1 = 128 x 32), bosonic chunks
# of the contraction as a multiple of the pass's default)
SIGMA_TILES = (0, 1)
SIGMA_CHUNK_FACTORS = (0.5, 1.0, 2.0)


def tune_sigma(lp, repeats: int = 2, cache_path: str | None = None, force: bool = False) -> TuneResult:
    """Chooses the GEMM tile and the number of bosonic chunks of the wedge Sigma contraction for ``lp`` (a
    LadderPass whose kernel K is computed: run a pass first) by timing ``lp.sigma_stage`` with each candidate (CUDA
    events, best of ``repeats`` after a warm-up), installs the fastest and caches it per (device, shape).  Every
    candidate computes the same Sigma up to the order of the bosonic partial sums.  Passes that do not take the
    wedge form (orbital rotations, grids without the inversion) keep their defaults."""
    from .pipeline import sigma_chunks_for

    sh = lp.sh
    if not sh.wedge:
        return TuneResult("", (0, lp.sigma_chunks), {}, 0)
    key = "sigma|" + shape_key(lp, "fp64")  # one choice per shape, shared by both forms of the pass
    load_cache(cache_path)
    if not force and key in _CACHE:
        lp.sigma_tile, lp.sigma_chunks = _CACHE[key]
        _ensure_sigma_scratch(lp)
        return TuneResult(key, tuple(_CACHE[key]), {}, 0)
    base = sigma_chunks_for(sh)
    nwf = 2 * sh.niw + 1
    chunks = sorted({max(1, min(nwf, int(round(base * f)))) for f in SIGMA_CHUNK_FACTORS})
    stream = torch.cuda.current_stream()
    times = {}
    for tile in SIGMA_TILES:
        for ch in chunks:
            lp.sigma_tile, lp.sigma_chunks = tile, ch
            _ensure_sigma_scratch(lp)
            lp.sigma_stage()  # warm-up
            best = float("inf")
            for _ in range(repeats):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                lp.sigma_stage()
                b.record(stream)
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            times[(tile, ch)] = best
    choice = min(times, key=times.get)
    lp.sigma_tile, lp.sigma_chunks = choice
    _ensure_sigma_scratch(lp)
    _CACHE[key] = choice
    save_cache(cache_path)
    return TuneResult(key, choice, {f"{k[0]}/{k[1]}": v for k, v in times.items()}, 0)


def _ensure_sigma_scratch(lp) -> None:
    sh = lp.sh
    need = int(lib().dga_sigma_wedge_scratch_bytes(sh.n_orb, sh.niv, sh.niw, sh.n_q, sh.nk_tot, lp.sigma_chunks))
    if lp.sigma_scratch.numel() * 16 < need:
        lp.sigma_scratch = torch.empty(need // 16 + 1, dtype=C128, device=lp.dev)
