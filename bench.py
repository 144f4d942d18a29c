"""Benchmark: (q, w) ladder solves per second of the nonlocal ladder-DGA pass on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c3] [--impl ours|reference]

One step is one full nonlocal pass over the resident inputs of the configuration (bubble -> double-counting
kernel -> chi0^-1 -> BSE in the density and magnetic channels -> shell-corrected chi -> lambda (single band)
-> kernel -> Sigma(k, nu)).  One (q, w) ladder solve = one irreducible q x one w >= 0 x one channel, so a step
of the 3-orbital t2g configuration (32x32, niv = niw = 40, N = 720) is 153 * 41 * 2 = 12,546 solves.

The metric is whole-job throughput over the timed steps (CUDA events on the launching stream, max over
ranks).  ``e2e`` is the same metric through the public API with host G(k) in and host Sigma out.  Multi-GPU
runs are independent replicas (the device schedule has no inter-GPU exchange): weak scaling.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def f_solve(N: int, n2: int) -> float:
    """Real flops of one complex LU with partial pivoting plus n2 right-hand-side solves: 8/3 N^3 + 8 n2 N^2."""
    return 8.0 / 3.0 * N**3 + 8.0 * n2 * N**2


def measured_peaks() -> dict:
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms in the background."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
        "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
        "clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        if self.index < 0:
            return self
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        smax = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, val in zip(names, s[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(self.samples),
        }


def dist_setup(n_gpus: int):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def gemm_peak_tflops(dtype_name: str = "float64", tf32: bool = False) -> float:
    """cuBLAS GEMM 8192^3 best of 5 on this GPU: FP64 (DMMA), FP32 without TF32 (CUDA cores) or FP32 with TF32
    allowed (the TF32 tensor-core rate) -- the denominators MEASURED_PEAKS.json does not hold (it has bf16 and
    HBM only)."""
    import torch

    torch.backends.cuda.matmul.allow_tf32 = bool(tf32)
    dtype = getattr(torch, dtype_name)
    n = 8192
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2.0 * n**3 / best / 1e12


def cpu_baseline_sample(inp: dict, n_items: int = 6) -> dict:
    """The oracle (NumPy restatement of the upstream path) timed on a bounded sample of BSE solves."""
    from oracle import ladder as oracle

    beta = inp["beta"]
    nb = inp["u"].shape[0]
    niv = inp["niv_core"]
    chi0 = oracle.chi0_q_fft(inp["g_k"], inp["niw"], niv + inp["niv_shell"], inp["irrk_ind"][:1], beta)
    c0i = oracle.chi0_inv(oracle.cut_niv(chi0, niv, 1))
    uv = oracle.u_as_channel(inp["u"], "magn")[None] + oracle.v_as_channel(inp["v_q_irr"][:1], "magn")
    t0 = time.perf_counter()
    done = 0
    for w in range(min(n_items, c0i.shape[5])):
        oracle.bse_sum(c0i[..., w : w + 1, :], inp["gamma_magn"][..., w : w + 1, :, :], uv, beta)
        done += 1
    dt = time.perf_counter() - t0
    return {
        "value": done / dt,
        "unit": "(q,w) ladder solves/s",
        "cores": os.cpu_count(),
        "kind": "port",
        "sample": f"{done} BSE solves (N={nb * nb * 2 * niv}) of the oracle (numpy inv + nu' sum, "
        f"four_point.py:620-642), one q, magn channel",
    }


def run_reference(args, rank: int, world: int):
    """--impl reference: the upstream CPU path (its NumPy restatement in oracle/) on the host cores."""
    if rank != 0:
        return
    from dgamore_b200 import synthetic
    from oracle import ladder as oracle

    cfg = synthetic.CONFIGS[args.config]
    inp = synthetic.make_inputs(cfg)
    nb, niv = cfg.n_bands, cfg.niv
    N = nb * nb * 2 * niv
    beta = cfg.beta
    chi0 = oracle.chi0_q_fft(inp["g_k"], cfg.niw, cfg.niv_full, inp["irrk_ind"][:1], beta)
    c0i = oracle.chi0_inv(oracle.cut_niv(chi0, niv, 1))
    uv = oracle.u_as_channel(inp["u"], "magn")[None] + oracle.v_as_channel(inp["v_q_irr"][:1], "magn")
    per_step = max(1, min(cfg.niw + 1, args.ref_items))
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for w in range(per_step):
            oracle.bse_sum(c0i[..., w : w + 1, :], inp["gamma_magn"][..., w : w + 1, :, :], uv, beta)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = float(np.sum(times))
    value = per_step * args.steps / t
    line = {
        "impl": "reference",
        "metric": "(q,w) ladder solves/s",
        "value": value,
        "unit": "(q,w) ladder solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex128",
        "data": "synthetic (seeded model inputs with the configuration's shapes)",
        "config": {"workload": f"{args.config}: {cfg.n_bands}-orbital {cfg.nk[0]}x{cfg.nk[1]} niv=niw={cfg.niv}, N={N}",
                   "sample_per_step": f"{per_step} BSE solves"},
        "cpu_baseline": {"value": value, "unit": "(q,w) ladder solves/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{per_step} BSE solves per step (numpy inv + nu' sum of the oracle)"},
        "e2e": {"value": value, "unit": "(q,w) ladder solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def time_pass(lp, args, world: int, local: int, sample_clocks: bool):
    """Warm-up, then K timed device passes replayed from one CUDA graph (CUDA events on the launching stream,
    max over ranks); one more eager pass times the BSE launch alone for the roofline."""
    import torch

    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        lp.run()
    torch.cuda.synchronize()
    status = int(lp.bse_status.abs().sum().item()) + int(lp.status.abs().sum().item())
    sh = lp.sh

    # BSE launch time (eager pass, events around the BSE on the same stream)
    bse_ms = []
    for _ in range(2):
        lp.pre_bse()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        lp.bse()
        b.record(stream)
        lp.post_bse()
        b.synchronize()
        bse_ms.append(a.elapsed_time(b))

    # timed region: device-resident inputs, K graph replays of the whole pass
    lp.capture()
    for _ in range(max(1, args.warmup)):
        lp.replay()
    barrier(world)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local if sample_clocks else -1)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with clocks:
        start.record(stream)
        marks[0].record(stream)
        for k in range(args.steps):
            lp.replay()
            marks[k + 1].record(stream)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(start.elapsed_time(end) / 1e3, world)
    value = world * sh.n_solves * args.steps / t
    per_step = np.array([marks[k].elapsed_time(marks[k + 1]) for k in range(args.steps)])
    step_ms = {"median": float(np.median(per_step)), "p10": float(np.percentile(per_step, 10)),
               "p90": float(np.percentile(per_step, 90))}
    return {"t": t, "value": value, "bse_ms": float(min(bse_ms)), "status": status, "clocks": clocks,
            "step_ms": step_ms}


# DRAM bytes per BSE item of each kernel, from `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum` of a
# single-wave launch of the same kernel on the 3-orbital case with the full N = 720 (4x4 grid, niw = 10,
# 132 items); traffic grows in proportion to the items, so a full launch's traffic is items x this.
DRAM_BYTES_PER_ITEM = {
    "bse_solve_sum_fp64_kernel": 22.89e9 / 132,
    "bse_panel_mixed_kernel": (5.670e9 + 4.917e9) / 132,
    "bse_panel_mixed_kernel<TC> (tcgen05 trailing tiles)": (6.093e9 + 4.978e9) / 132,
    "bse_solve_sum_mixed_kernel": 11.79e9 / 132,
    # same 132-item case, one item per CTA: ncu dram__bytes_read.sum + dram__bytes_write.sum
    "bse_block_mixed_kernel (tcgen05, pivoting inside 32x32 blocks)": (7.053e9 + 4.934e9) / 132,
}


def kernel_name(lp) -> str:
    if lp.precision == "fp64":
        return "bse_solve_sum_fp64_kernel"
    kernel = lp.tuning.kernel if lp.tuning is not None else (4 if lp.sh.N >= 320 else 2)
    if kernel == 2:
        return "bse_solve_sum_mixed_kernel"
    if kernel == 3:
        return "bse_panel_mixed_kernel<TC> (tcgen05 trailing tiles)"
    if kernel == 4:
        return "bse_block_mixed_kernel (tcgen05, pivoting inside 32x32 blocks)"
    return "bse_panel_mixed_kernel"


def serving_leg(precision: str, n_requests: int) -> dict:
    """Continuous-batching server on a seeded Poisson mix of requests (1-3 orbitals, several grids and boxes,
    beta ~ U[5,30], U ~ U[2,10]): p50 / p99 latency from arrival to Sigma on the host."""
    from dgamore_b200.serving import LadderServer, serving_workload

    reqs = serving_workload(n_requests, rate_per_s=20.0, seed=5, precision=precision)
    srv = LadderServer(hbm_budget=40 << 30, scratch_bytes=2 << 30, items_per_request=256)
    # warm-up outside the measurement: one request of every launch class loads the kernels and sets their
    # attributes, as a running service has done before its first timed request
    seen, warm = set(), []
    for r in reqs:
        key = (r.inp["u"].shape[0], r.inp["niv_core"])
        if key not in seen:
            seen.add(key)
            warm.append(type(r)(r.inp, precision=precision))
    srv.serve(warm, realtime=False)
    srv.stats = type(srv.stats)()
    stats = srv.serve(reqs, realtime=True)
    out = stats.summary()
    out["bse_status_nonzero"] = int(sum(int(np.abs(r.bse_status).sum()) for r in stats.completed))
    return out


def serving_c5_leg(n_requests: int, rate_per_s: float = 25.0, seed: int = 11) -> dict:
    """The continuous-batching server on a loaded stream of requests drawn from the mixed-request workload's shape
    sets (serving.C5_SERVE_SHAPES: orbitals 1-3, grids 16^2-64^2, niv = niw 20-60, without the shapes whose inputs
    take more than seconds to generate), beta ~ U[5,30], U ~ U[2,10], Poisson arrivals faster than the server
    completes them; both forms on the same requests."""
    from collections import Counter

    from dgamore_b200.serving import C5_SERVE_SHAPES, LadderServer, serving_workload

    base = serving_workload(n_requests, rate_per_s=rate_per_s, seed=seed, precision="fp64", shapes=C5_SERVE_SHAPES)
    shapes = Counter((int(r.inp["u"].shape[0]), int(r.inp["nk"][0]), int(r.inp["niv_core"])) for r in base)
    out = {"workload": f"{n_requests} requests from {len(C5_SERVE_SHAPES)} shapes (n_orb, nk, niv) of the mixed "
                       f"workload's sets, Poisson arrivals at {rate_per_s}/s (seed {seed})",
           "shapes_drawn": {f"{k[0]}orb_{k[1]}x{k[1]}_niv{k[2]}": v for k, v in sorted(shapes.items())}}
    for precision in ("mixed", "fp64"):
        reqs = [type(r)(r.inp, arrival=r.arrival, precision=precision) for r in base]
        srv = LadderServer(hbm_budget=60 << 30, scratch_bytes=4 << 30, items_per_request=256)
        seen, warm = set(), []
        for r in reqs:
            key = (r.inp["u"].shape[0], r.inp["niv_core"])
            if key not in seen:
                seen.add(key)
                warm.append(type(r)(r.inp, precision=precision))
        srv.serve(warm, realtime=False)
        srv.stats = type(srv.stats)()
        stats = srv.serve(reqs, realtime=True)
        res = stats.summary()
        res["bse_status_nonzero"] = int(sum(int(np.abs(r.bse_status).sum()) for r in stats.completed))
        out[precision] = res
    return out


def c4_batch_leg(precision: str, steps: int = 3) -> dict:
    """The 2-orbital bilayer (48x48, niv = niw = 30, N = 240) and the 1-orbital lattice (32x32, niv = niw = 50,
    N = 100) as one device schedule: both passes' stages and ONE persistent BSE launch over the items of both,
    replayed from one captured CUDA graph; each request's X is compared bitwise with its single-request pass."""
    import torch

    from dgamore_b200 import synthetic
    from dgamore_b200.pipeline import LadderPass
    from dgamore_b200.serving import BatchedPasses

    inps = [synthetic.make_inputs("c4_bilayer"), synthetic.make_inputs("c4_single")]
    alone = []
    for inp in inps:
        lp = LadderPass(inp, precision=precision, keep_intermediates=False)
        lp.run()
        torch.cuda.synchronize()
        alone.append(lp.X.cpu())
        del lp
    torch.cuda.empty_cache()
    passes = [LadderPass(inp, precision=precision, keep_intermediates=False, own_bse_scratch=False) for inp in inps]
    bp = BatchedPasses(passes, precision)
    bp.capture()
    for _ in range(2):
        bp.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        bp.replay()
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    bitwise = all(torch.equal(lp.X.cpu(), x) for lp, x in zip(passes, alone))
    status = sum(int(lp.bse_status.abs().sum()) for lp in passes)
    out = {
        "workload": "2-orbital bilayer 48x48 niv=niw=30 (N=240) + 1-orbital 32x32 niv=niw=50 (N=100), one graph",
        "precision": precision,
        "bse_launches_per_step": len(bp.batches),
        "solves_per_step": bp.n_solves,
        "ms_per_step": ms,
        "solves_per_s": bp.n_solves / (ms / 1e3),
        "x_bitwise_equal_to_single_requests": bool(bitwise),
        "bse_status_nonzero": status,
    }
    bp.graph = None
    del bp, passes
    torch.cuda.empty_cache()
    return out


def small_configs_leg(steps: int = 3, configs=("c1", "c2")) -> dict:
    """The single-band configurations at their stated sizes (C1: 16x16, niv = niw = 20, N = 40; C2: 64x64,
    niv = niw = 60, N = 120), both forms replayed from one CUDA graph each: solves/s, the mixed/FP64 ratio, the
    Sigma error of the mixed form against the FP64 form and the difference of the lambdas."""
    import torch

    from dgamore_b200 import synthetic
    from dgamore_b200.pipeline import LadderPass

    out = {}
    for name in configs:
        inp = synthetic.make_inputs(name)
        res = {}
        sig = {}
        lam = {}
        for precision in ("mixed", "fp64"):
            lp = LadderPass(inp, precision=precision, keep_intermediates=False)
            lp.capture()
            for _ in range(2):
                lp.replay()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(steps):
                lp.replay()
            b.record()
            b.synchronize()
            ms = a.elapsed_time(b) / steps
            res[precision] = {"ms_per_pass": ms, "solves_per_s": lp.sh.n_solves / (ms / 1e3),
                              "bse_status_nonzero": int((lp.bse_status != 0).sum().item())}
            sig[precision] = lp.sigma.cpu().numpy()
            lam[precision] = lp.lambdas.cpu().numpy()
            del lp
            torch.cuda.empty_cache()
        out[name] = {
            "workload": f"{name}: 1-orbital {inp['nk'][0]}x{inp['nk'][1]}, niv = niw = {inp['niw']}, "
                        f"N = {2 * inp['niv_core']}, {2 * len(inp['irrk_ind']) * (inp['niw'] + 1)} solves per pass",
            "mixed": res["mixed"], "fp64": res["fp64"],
            "mixed_vs_fp64": res["fp64"]["ms_per_pass"] / res["mixed"]["ms_per_pass"],
            "sigma_rel_err_vs_fp64": float(np.abs(sig["mixed"] - sig["fp64"]).max() / np.abs(sig["fp64"]).max()),
            "lambda_abs_diff_vs_fp64": float(np.abs(lam["mixed"] - lam["fp64"]).max()),
        }
    return out


def eliashberg_leg(config: str = "c4_bilayer") -> dict:
    """Linearised Eliashberg on the bilayer configuration: pairing vertices from the FP64 pass, the gap-equation
    matvec timed with CUDA events (HBM roofline: it streams Gamma(R) [Nk][M][M] once per application), and the
    four leading eigenpairs of both channels."""
    import torch

    from dgamore_b200 import synthetic
    from dgamore_b200.eliashberg_solver import EliashbergSolver
    from dgamore_b200.pipeline import LadderPass

    inp = synthetic.make_inputs(config)
    lp = LadderPass(inp, keep_intermediates=True)
    lp.run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    lp.run()
    b.record()
    b.synchronize()
    pass_ms = a.elapsed_time(b)
    a.record()
    es = EliashbergSolver(lp)
    b.record()
    b.synchronize()
    vertex_ms = a.elapsed_time(b)
    # the vertex fused into the FP64 BSE (the pass's own LU factors solve the pp box; the stage adds the ladder term)
    lpf = LadderPass(inp, keep_intermediates=True, eliashberg_pp=es.P)
    lpf.run()
    torch.cuda.synchronize()
    a.record()
    lpf.run()
    b.record()
    b.synchronize()
    fused_pass_ms = a.elapsed_time(b)
    a.record()
    esf = EliashbergSolver(lpf)
    b.record()
    b.synchronize()
    fused_vertex_ms = a.elapsed_time(b)
    lsf, ltf, _, _ = esf.solve(n_eig=4, tol=1e-6)
    del esf, lpf
    x = torch.randn(es.dim, dtype=torch.complex128, device=lp.dev)
    out = torch.empty_like(x)
    for _ in range(3):
        es.matvec("sing", x, out)
    reps = 20
    a.record()
    for _ in range(reps):
        es.matvec("sing", x, out)
    b.record()
    b.synchronize()
    mv_ms = a.elapsed_time(b) / reps
    bytes_mv = es.mat[0].numel() * 16 + 4 * es.dim * 16  # Gamma(R) once + vector transforms in and out
    es.n_matvec = 0
    a.record()
    ls, lt, _, _ = es.solve(n_eig=4, tol=1e-6)
    b.record()
    b.synchronize()
    solve_ms = a.elapsed_time(b)
    # the operator with Gamma(R) stored in complex64 (FP64 products, vectors and normalisation)
    es32 = EliashbergSolver(lp, precision="mixed")
    for _ in range(3):
        es32.matvec("sing", x, out)
    a.record()
    for _ in range(reps):
        es32.matvec("sing", x, out)
    b.record()
    b.synchronize()
    mv32_ms = a.elapsed_time(b) / reps
    ls32, lt32, _, _ = es32.solve(n_eig=4, tol=1e-9)
    del es32
    hbm = measured_peaks().get("hbm_gbs")
    gbs = bytes_mv / (mv_ms / 1e3) / 1e9
    return {
        "workload": f"{config}: {lp.sh.n_orb}-orbital {lp.sh.nk[0]}x{lp.sh.nk[1]}, niv_pp={es.P}, M={es.M}",
        "vertex_ms": vertex_ms,
        "fused_vertex": {
            "note": "pass + full vertex with the vertex fused into the FP64 BSE (LadderPass(eliashberg_pp=niv_pp)) "
                    "against the separate vertex kernel",
            "pass_ms": fused_pass_ms, "vertex_ms": fused_vertex_ms, "total_ms": fused_pass_ms + fused_vertex_ms,
            "separate_pass_ms": pass_ms, "separate_vertex_ms": vertex_ms, "separate_total_ms": pass_ms + vertex_ms,
            "lambda_sing": [float(v) for v in lsf], "lambda_trip": [float(v) for v in ltf],
        },
        "matvec_ms": mv_ms,
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                     "frac": gbs / hbm if hbm else None, "bytes_per_matvec": bytes_mv},
        "solve_ms": solve_ms,
        "matvecs_in_solve": es.n_matvec,
        "lambda_sing": [float(v) for v in ls],
        "lambda_trip": [float(v) for v in lt],
        "complex64_operator": {
            "matvec_ms": mv32_ms,
            "speedup_vs_fp64_matvec": mv_ms / mv32_ms,
            "lambda_max_sing": float(ls32[0]),
            "lambda_max_trip": float(lt32[0]),
            "lambda_max_abs_err_vs_fp64": max(abs(float(ls32[0]) - float(ls[0])), abs(float(lt32[0]) - float(lt[0]))),
        },
        "status": {k: int(v) for k, v in es.status.items()},
    }


def run_ours(args, rank: int, world: int, local: int):
    import torch

    from dgamore_b200 import autotune, synthetic
    from dgamore_b200.pipeline import LadderPass

    cfg = synthetic.CONFIGS[args.config]
    inp = synthetic.make_inputs(cfg)
    stream = torch.cuda.current_stream()
    cache = os.path.join(HERE, "_build", "tuning.json") if args.tune_cache else None

    # FP64 drop-in form first: the reference point of the mixed form and of its Sigma error
    lp64 = LadderPass(inp, keep_intermediates=False, precision="fp64")
    lp64.pre_bse()
    tune64 = autotune.tune_bse(lp64, cache_path=cache)
    lp64.run()
    tune_sig = autotune.tune_sigma(lp64, cache_path=cache)  # the Sigma stage's tile and chunks, shared by both forms
    r64 = time_pass(lp64, args, world, local, sample_clocks=False)
    sigma64 = lp64.sigma.clone()
    del lp64
    torch.cuda.empty_cache()

    lp = LadderPass(inp, keep_intermediates=False, precision=args.precision)
    sh = lp.sh
    lp.pre_bse()
    tune = autotune.tune_bse(lp, cache_path=cache)
    autotune.tune_sigma(lp, cache_path=cache)
    res = time_pass(lp, args, world, local, sample_clocks=True)
    t, value, bse_ms, status, clocks = res["t"], res["value"], res["bse_ms"], res["status"], res["clocks"]
    sig_err = float((lp.sigma - sigma64).abs().max().item() / sigma64.abs().max().item())
    iters = lp.bse_iters.cpu().numpy() if args.precision == "mixed" else None
    kname = kernel_name(lp)
    kernels_per_pass = lp.kernels_per_pass()

    # end to end through the public API: host G(k) -> device pass (graph replay) -> host Sigma
    lp.run_e2e()
    barrier(world)
    e_s, e_e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_s.record(stream)
    for _ in range(args.steps):
        lp.run_e2e()
    e_e.record(stream)
    e_e.synchronize()
    t_e2e = max_over_ranks(e_s.elapsed_time(e_e) / 1e3, world)
    e2e_value = world * sh.n_solves * args.steps / t_e2e
    del lp
    torch.cuda.empty_cache()

    fp64_peak = gemm_peak_tflops("float64") if rank == 0 else None
    fp32_peak = gemm_peak_tflops("float32") if rank == 0 else None
    tf32_peak = gemm_peak_tflops("float32", tf32=True) if rank == 0 else None
    tensor_kernel = args.precision == "mixed" and "TC" in kname or "tcgen05" in kname
    peak = (tf32_peak if tensor_kernel else fp32_peak) if args.precision == "mixed" else fp64_peak
    flops_launch = sh.n_solves * f_solve(sh.N, sh.n2)
    achieved = flops_launch / (bse_ms / 1e3) / 1e12
    per_item = DRAM_BYTES_PER_ITEM.get(kname)
    peaks = measured_peaks()
    algo_bytes = 2 * sh.W * sh.N * sh.N * 16 + sh.n_solves * (sh.nv * sh.n2 * sh.n2 + sh.N * sh.n2) * 16
    if args.precision == "mixed" and tensor_kernel:
        peak_source = ("cuBLAS FP32 GEMM 8192^3 with TF32 allowed (the TF32 tensor-core rate), measured in this run; "
                       "the kernel issues every trailing-update product as three TF32 MMAs (hi*hi + hi*lo + lo*hi), "
                       "so its tensor pipe does 3x the algorithmic flops of the update")
    elif args.precision == "mixed":
        peak_source = "cuBLAS FP32 SGEMM 8192^3 without TF32 (CUDA cores), measured in this run"
    else:
        peak_source = "cuBLAS FP64 DGEMM 8192^3, measured in this run"
    serving = {}
    if args.serve_requests > 0 and rank == 0:
        for prec in ("fp64", "mixed"):
            serving[prec] = serving_leg(prec, args.serve_requests)
    eliashberg = eliashberg_leg() if (args.eliashberg and rank == 0) else None
    small = small_configs_leg() if (args.small and rank == 0) else None
    serving_c5 = serving_c5_leg(args.serve_c5) if (args.serve_c5 and rank == 0) else None
    c4 = {}
    if args.c4 and rank == 0:
        for prec in ("fp64", "mixed"):
            c4[prec] = c4_batch_leg(prec)
    line = {
        "metric": "(q,w) ladder solves/s",
        "value": value,
        "unit": "(q,w) ladder solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps,
        "step_ms": res["step_ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex64 LU + complex128 refinement" if args.precision == "mixed" else "complex128",
        "data": "synthetic (seeded model inputs with the configuration's shapes; see dgamore_b200/synthetic.py)",
        "config": {
            "workload": f"{args.config}: {cfg.n_bands}-orbital {cfg.nk[0]}x{cfg.nk[1]} square lattice, "
            f"niv=niw={cfg.niv}, N={sh.N}, {sh.n_q} irreducible q, {sh.n_solves} solves per pass",
            "precision": "mixed (FP32 LU, FP64 refinement)" if args.precision == "mixed" else "fp64 drop-in",
            "step": "one full nonlocal pass (bubble, dc kernel, chi0^-1, BSE dens+magn, chi_phys, lambda, kernel, "
            "Sigma) replayed from one CUDA graph",
            "l2": "inputs larger than L2 (Gamma_r alone is %.0f MB)" % (2 * sh.W * sh.N * sh.N * 16 / 1e6),
            "parallelism": f"{world} independent replica(s)",
            "bse_launch": {"kernel": kname, "tuning": list(tune.choice), "tuning_times_ms": tune.times_ms},
            "sigma_launch": {"tuning_tile_chunks": list(tune_sig.choice), "tuning_times_ms": tune_sig.times_ms},
        },
        "gpu_launches": kernels_per_pass * args.steps,
        "e2e": {
            "value": e2e_value,
            "unit": "(q,w) ladder solves/s",
            "h2d_bytes_per_step": inp["g_k"].size * 16,
            "d2h_bytes_per_step": sh.nk_tot * sh.n2 * 2 * sh.niv * 16,
        },
        "fp64_dropin": {
            "value": r64["value"],
            "ms_per_step": 1e3 * r64["t"] / args.steps,
            "bse_ms_per_launch": r64["bse_ms"],
            "bse_tflops": flops_launch / (r64["bse_ms"] / 1e3) / 1e12,
            "bse_frac_of_fp64_peak": (flops_launch / (r64["bse_ms"] / 1e3) / 1e12 / fp64_peak) if fp64_peak else None,
            "tuning": list(tune64.choice),
        },
        "mixed_vs_fp64": value / r64["value"],
        "sigma_rel_err_vs_fp64": sig_err,
        "refinement_iters": None if iters is None else {"mean": float(iters.mean()), "max": int(iters.max())},
        "roofline": {
            "bound": "tensor",
            "kernel": kname,
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None,
            "frac_note": "achieved = flops_per_launch / bse_ms_per_launch (algorithmic complex-LU flops, "
            "8/3 N^3 + 8 n2 N^2 per solve); frac = achieved / peak",
            "peak_source": peak_source,
            "peaks_measured_tflops": {"tf32_tensor": tf32_peak, "fp32_cuda_core": fp32_peak, "fp64": fp64_peak,
                                      "bf16_sustained (MEASURED_PEAKS.json)": peaks.get("bf16_tflops_sustained")},
            "frac_of_bf16_sustained": (achieved / peaks["bf16_tflops_sustained"])
            if peaks.get("bf16_tflops_sustained") else None,
            "flops_per_launch": flops_launch,
            "bse_ms_per_launch": bse_ms,
            "traffic": None if per_item is None else per_item * sh.n_solves,
            "traffic_note": "ncu DRAM bytes per item of a single-wave launch of the same kernel, times the items",
            "algorithmic_bytes": algo_bytes,
            "traffic_over_algorithmic": None if per_item is None else per_item * sh.n_solves / algo_bytes,
        },
        "bse_status_nonzero": status,
        "clocks": clocks.summary(),
        "serving": serving,
        "eliashberg": eliashberg,
        "small_configs": small,
        "serving_c5": serving_c5,
        "c4_batch": c4,
    }
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline_sample(inp, args.cpu_items)
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-items", type=int, default=4)
    ap.add_argument("--ref-items", type=int, default=3)
    ap.add_argument("--serve-requests", type=int, default=24, help="requests of the serving leg (0: skip)")
    ap.add_argument("--tune-cache", action="store_true", help="keep autotuner choices in _build/tuning.json")
    ap.add_argument("--eliashberg", type=int, default=1, help="run the Eliashberg leg (0: skip)")
    ap.add_argument("--c4", type=int, default=1, help="run the uneven-orbital batch leg under one graph (0: skip)")
    ap.add_argument("--small", type=int, default=1, help="run the C1/C2 mixed-vs-FP64 leg (0: skip)")
    ap.add_argument("--serve-c5", type=int, default=0,
                    help="requests of the loaded serving leg on the mixed-request workload's shapes (0: skip)")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
