"""Continuous batching of ladder passes on one B200.

The upstream runs one nonlocal pass per job (``nonlocal_sde.calculate_self_energy_q``,
dgamore/nonlocal_sde.py:786-879) and its BSE as one ``create_auxiliary_chi_r_q_sum`` call per job
(nonlocal_sde.py:85-156).  Serving many independent requests -- different lattices, frequency boxes,
temperatures, interactions -- on one GPU is done here the way LLM servers batch decode steps:

* **Admission by HBM footprint.**  A request is admitted when the device bytes of its pass
  (``pipeline.estimate_device_bytes``, computed from its shapes before anything is allocated) fit the
  server's budget next to the requests already running; otherwise it waits in FIFO order.
* **One persistent launch per iteration.**  Every iteration gathers BSE work items (request, channel, q, w)
  from all running requests of the same launch class (orbital count; in the mixed form also the side of
  the compound size takes) into one ``dga_bse_solve_sum_batch_c128`` launch.
  Items are taken round-robin, a bounded number per request per iteration (``items_per_request``), so a
  small request that arrives while a large one runs finishes in a few iterations instead of waiting for
  the large one to drain (the chunked scheduling of long prompts in LLM serving).
* **Per-request stages around it.**  Admission runs a request's pre-BSE stages (G(R), bubble, K_dc,
  chi0^-1); the iteration in which its last BSE item completes runs its post-BSE stages (chi_r, lambda,
  kernel assembly, Sigma) and copies Sigma to pinned host memory.

Each BSE item is solved by the same device code as in a single-request launch, and the other stages are
per request, so a request's Sigma is bitwise the same whether it is served alone or in a mix.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import BseProblem, call, lib
from .pipeline import LadderPass, PassShapes, estimate_device_bytes

_MODES = {"fp64": 0, "mixed": 1}
_RESOLVE = 2


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# Compound size from which the mixed form runs the shared-memory-panel kernel when alone (the library's default
# rule); a batch launch serves requests on one side of it only, so each gets the kernel it gets alone.
def launch_class(lp: LadderPass, precision: str) -> tuple:
    """Requests of one class share a batch launch: the same kernel as each would take alone
    (dga_bse_default_kernel), so that a request's results are bitwise the same in a batch and alone.  The
    128-thread kernels and the mixed form's block kernel for 1 to 3 orbitals choose the right-hand-side count per
    item, so their requests share one launch whatever their orbital counts; the shared-memory-panel kernels and
    the 4-orbital block kernel are compiled per orbital count, so there the class also holds n_orb."""
    mixed = precision == "mixed"
    kernel = int(lib().dga_bse_default_kernel(lp.sh.n_orb, lp.sh.niv, 1 if mixed else 0))
    per_orbital = kernel in (1, 3) or (kernel == 4 and lp.sh.n_orb > 3)
    return (precision, kernel, lp.sh.n_orb if per_orbital else 0)


def item_cost(sh: PassShapes) -> float:
    """Relative cost of one BSE item: the LU of an N x N matrix."""
    return float(sh.N) ** 3


def _descriptor(lp: LadderPass) -> BseProblem:
    sh = lp.sh
    return BseProblem(
        gamma_cm=lp.gamma_cm.data_ptr(), chi0_inv=lp.chi0_inv.data_ptr(), uv=lp.uv.data_ptr(), out=lp.X.data_ptr(),
        n_orb=sh.n_orb, niv=sh.niv, niw_half=sh.W, n_q=sh.n_q, beta=sh.beta, inv_beta2=lp.inv_beta2,
    )


class BseBatch:
    """One launch over BSE items of several passes of the same launch class (``launch_class``).

    ``items`` is a list of (pass, item indices into ``pass.work``).  The launch writes each item's X into its
    own pass and its status word into ``pass.bse_status``; in mixed precision the items whose refinement did
    not converge are re-solved in FP64 by a second launch (mode 2) that skips every other item."""

    def __init__(self, items: list[tuple[LadderPass, torch.Tensor]], precision: str = "fp64",
                 refine_max_iter: int = 6, refine_tol: float = 1e-10):
        if precision not in _MODES:
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        passes = []
        index = {}
        for lp, _ in items:
            if id(lp) not in index:
                index[id(lp)] = len(passes)
                passes.append(lp)
        if len({launch_class(lp, precision) for lp in passes}) != 1:
            raise ValueError("a batch launch needs passes of one launch class (launch_class); split the batch")
        self.passes = passes
        self.precision = precision
        self.refine_max_iter = int(refine_max_iter)
        self.refine_tol = float(refine_tol)
        dev = passes[0].dev
        self.probs_host = (BseProblem * len(passes))(*[_descriptor(lp) for lp in passes])
        raw = torch.frombuffer(bytearray(bytes(self.probs_host)), dtype=torch.uint8)
        self.probs_dev = raw.to(dev)
        # work rows (request, ch, q, w), most expensive items first so that the static round-robin of the
        # persistent grid gives every CTA a similar load
        rows, owners, local = [], [], []
        for lp, idx in items:
            p = index[id(lp)]
            idx = torch.as_tensor(idx, dtype=torch.long, device=dev)
            w = lp.work.index_select(0, idx).to(torch.int32)
            rows.append(torch.cat([torch.full((len(idx), 1), p, dtype=torch.int32, device=dev), w], dim=1))
            owners.append(torch.full((len(idx),), p, dtype=torch.long))
            local.append(idx)
        cost = torch.cat([torch.full((len(o),), item_cost(passes[int(o[0])].sh) if len(o) else 0.0, dtype=torch.float64)
                          for o in owners])
        order = torch.argsort(cost, descending=True, stable=True)
        self.work = torch.cat(rows).index_select(0, order.to(dev)).contiguous()
        self.owner = torch.cat(owners).index_select(0, order)
        self.local = torch.cat(local).index_select(0, order.to(dev))
        # per pass, the batch positions of its items (device index lists, so that launch() copies nothing from the
        # host and can be captured in a CUDA graph)
        self.sel = [(self.owner == p).nonzero().squeeze(1).to(dev) for p in range(len(passes))]
        self.n_items = int(self.work.shape[0])
        self.status = torch.zeros(self.n_items, dtype=torch.int32, device=dev)
        self.iters = torch.zeros(self.n_items, dtype=torch.int32, device=dev)

    def scratch_bytes(self, mode: int | None = None) -> int:
        mode = _MODES[self.precision] if mode is None else mode
        return int(lib().dga_bse_batch_scratch_bytes(self.probs_host, len(self.passes), self.n_items, mode))

    def launch(self, scratch: torch.Tensor) -> None:
        """Enqueues the batch on the current stream (no synchronisation)."""
        nbytes = scratch.numel() * scratch.element_size()
        mode = _MODES[self.precision]
        call("dga_bse_solve_sum_batch_c128", self.probs_host, _ptr(self.probs_dev), len(self.passes), _ptr(self.work),
             self.n_items, mode, self.refine_max_iter, self.refine_tol, _ptr(self.status), _ptr(self.iters),
             _ptr(scratch), nbytes, _stream())
        if mode == 1:
            call("dga_bse_solve_sum_batch_c128", self.probs_host, _ptr(self.probs_dev), len(self.passes),
                 _ptr(self.work), self.n_items, _RESOLVE, self.refine_max_iter, self.refine_tol, _ptr(self.status),
                 _ptr(self.iters), _ptr(scratch), nbytes, _stream())
        # scatter the status words back to the passes
        for p, lp in enumerate(self.passes):
            sel = self.sel[p]
            lp.bse_status.index_copy_(0, self.local.index_select(0, sel), self.status.index_select(0, sel))
            lp.bse_iters.index_copy_(0, self.local.index_select(0, sel), self.iters.index_select(0, sel))


def solve_bse_batch(passes: list[LadderPass], precision: str = "fp64", scratch: torch.Tensor | None = None,
                    **kw) -> None:
    """BSE of several whole passes (all their items), one launch per launch class (``launch_class``)."""
    groups: dict[tuple, list[LadderPass]] = {}
    for lp in passes:
        groups.setdefault(launch_class(lp, precision), []).append(lp)
    for group in groups.values():
        dev = group[0].dev
        batch = BseBatch([(lp, torch.arange(lp.n_items, device=dev)) for lp in group], precision, **kw)
        sc = scratch
        if sc is None:
            need = max(batch.scratch_bytes(), batch.scratch_bytes(_RESOLVE) if precision == "mixed" else 0)
            sc = torch.empty(need // 16 + 1, dtype=torch.complex128, device=dev)
        batch.launch(sc)


class BatchedPasses:
    """Whole nonlocal passes of several requests as one device schedule: every pass's pre-BSE stages, one batch
    launch per launch class over all their BSE items (requests of different orbital counts -- the 2-orbital
    bilayer next to a 1-orbital lattice, say -- share a single launch), every pass's post-BSE stages.
    ``capture()`` records the whole schedule in one CUDA graph; ``replay()`` runs it again on refreshed inputs
    (the passes' resident G(k) and vertices are read in place)."""

    def __init__(self, passes: list[LadderPass], precision: str = "fp64", **kw):
        if any(lp.own_bse_scratch for lp in passes):
            raise ValueError("build the passes with own_bse_scratch=False: the batch launch brings the scratch")
        self.passes = passes
        self.precision = precision
        groups: dict[tuple, list[LadderPass]] = {}
        for lp in passes:
            groups.setdefault(launch_class(lp, precision), []).append(lp)
        dev = passes[0].dev
        self.batches = [BseBatch([(lp, torch.arange(lp.n_items, device=dev)) for lp in g], precision, **kw)
                        for g in groups.values()]
        need = max(max(b.scratch_bytes(), b.scratch_bytes(_RESOLVE) if precision == "mixed" else 0)
                   for b in self.batches)
        self.scratch = torch.empty(need // 16 + 1, dtype=torch.complex128, device=dev)
        self.graph = None

    @property
    def n_solves(self) -> int:
        return sum(lp.sh.n_solves for lp in self.passes)

    def run(self) -> None:
        for lp in self.passes:
            lp.pre_bse()
        for b in self.batches:
            b.launch(self.scratch)
        for lp in self.passes:
            lp.post_bse()

    def capture(self) -> "torch.cuda.CUDAGraph":
        self.run()  # module loading and kernel attributes outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            self.run()
        torch.cuda.synchronize()
        self.graph = g
        return g

    def replay(self) -> None:
        self.graph.replay()


# ------------------------------------------------------------------------------------------------------------
# continuous-batching server
# ------------------------------------------------------------------------------------------------------------
@dataclass
class Request:
    """One nonlocal-pass request: the inputs of ``LadderPass`` and an arrival time (seconds after start)."""

    inp: dict
    arrival: float = 0.0
    precision: str = "fp64"
    rid: int = -1
    # filled in by the server
    footprint: int = 0
    t_admit: float = float("nan")
    t_done: float = float("nan")
    sigma: np.ndarray | None = None
    lambdas: np.ndarray | None = None
    bse_status: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


@dataclass
class _Running:
    req: Request
    lp: LadderPass
    cursor: int = 0
    sigma_host: torch.Tensor | None = None


@dataclass
class ServerStats:
    iterations: int = 0
    launches: int = 0
    items: int = 0
    peak_admitted_bytes: int = 0
    completed: list = field(default_factory=list)

    def latencies(self) -> np.ndarray:
        return np.array([r.latency for r in self.completed])

    def summary(self) -> dict:
        lat = self.latencies()
        if len(lat) == 0:
            return {"requests": 0}
        span = max(r.t_done for r in self.completed) - min(r.arrival for r in self.completed)
        solves = sum(2 * PassShapes.from_inputs(r.inp).n_q * (int(r.inp["niw"]) + 1) for r in self.completed)
        return {
            "requests": len(lat),
            "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()),
            "span_s": float(span),
            "requests_per_s": len(lat) / span if span > 0 else float("nan"),
            "solves_per_s": solves / span if span > 0 else float("nan"),
            "iterations": self.iterations,
            "launches": self.launches,
            "peak_admitted_bytes": self.peak_admitted_bytes,
        }


class LadderServer:
    """Admits requests by HBM footprint and advances all running requests' BSE items in shared launches.

    hbm_budget: bytes the running passes may hold together (their resident inputs and work buffers);
    scratch_bytes: the BSE launch scratch, shared by every iteration and counted separately;
    items_per_request: BSE items each running request contributes to one iteration (None: all of them)."""

    def __init__(self, hbm_budget: int, scratch_bytes: int = 4 << 30, items_per_request: int | None = 256,
                 device: str = "cuda", refine_max_iter: int = 6, refine_tol: float = 1e-10,
                 reserve_bytes: int | None = None):
        self.dev = torch.device(device)
        with torch.cuda.device(self.dev):
            call("dga_bse_preload")  # the BSE kernels' code is loaded at start-up, not inside a request
        # the requests' buffers are carved from one segment of the caching allocator reserved now (a block freed
        # here stays cached and is split for later allocations), so that admitting a request does not pay a
        # device-synchronising cudaMalloc
        reserve = min(int(hbm_budget), 16 << 30) if reserve_bytes is None else int(reserve_bytes)
        if reserve > 0:
            block = torch.empty(reserve, dtype=torch.uint8, device=self.dev)
            del block
        self.hbm_budget = int(hbm_budget)
        self.items_per_request = items_per_request
        self.refine_max_iter = refine_max_iter
        self.refine_tol = refine_tol
        self.scratch = torch.empty(int(scratch_bytes) // 16, dtype=torch.complex128, device=self.dev)
        self.waiting: list[Request] = []
        self.running: list[_Running] = []
        self.admitted_bytes = 0
        self.stats = ServerStats()
        self._t0 = time.perf_counter()
        self._next_rid = 0

    # -------------------------------------------------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request) -> Request:
        if req.rid < 0:
            req.rid = self._next_rid
            self._next_rid += 1
        req.footprint = estimate_device_bytes(PassShapes.from_inputs(req.inp), req.precision)
        if req.footprint > self.hbm_budget:
            raise ValueError(f"request {req.rid} needs {req.footprint} B, above the server budget {self.hbm_budget} B")
        self.waiting.append(req)
        return req

    def _admit(self) -> None:
        while self.waiting and self.admitted_bytes + self.waiting[0].footprint <= self.hbm_budget:
            req = self.waiting.pop(0)
            lp = LadderPass(req.inp, device=str(self.dev), precision=req.precision, keep_intermediates=False,
                            own_bse_scratch=False, refine_max_iter=self.refine_max_iter, refine_tol=self.refine_tol)
            lp.g_k.copy_(lp.g_k_host, non_blocking=True)
            lp.pre_bse()
            req.t_admit = self.now()
            self.admitted_bytes += req.footprint
            self.stats.peak_admitted_bytes = max(self.stats.peak_admitted_bytes, self.admitted_bytes)
            self.running.append(_Running(req, lp))

    def step(self) -> list[Request]:
        """One iteration: admit, one batch launch per launch class (``launch_class``), finish completed requests.
        Synchronises the stream once at the end; returns the requests completed in this iteration."""
        self._admit()
        if not self.running:
            return []
        groups: dict[tuple, list] = {}
        for r in self.running:
            left = r.lp.n_items - r.cursor
            take = left if self.items_per_request is None else min(left, self.items_per_request)
            if take > 0:
                groups.setdefault(launch_class(r.lp, r.req.precision), []).append((r, take))
        for (precision, _, _), members in groups.items():
            items = []
            for r, take in members:
                items.append((r.lp, torch.arange(r.cursor, r.cursor + take, device=self.dev)))
                r.cursor += take
            batch = BseBatch(items, precision, self.refine_max_iter, self.refine_tol)
            batch.launch(self.scratch)
            self.stats.launches += 1 + (precision == "mixed")
            self.stats.items += batch.n_items
        done = [r for r in self.running if r.cursor >= r.lp.n_items]
        for r in done:
            r.lp.post_bse()
            r.sigma_host = torch.empty(r.lp.sigma.shape, dtype=r.lp.sigma.dtype).pin_memory()
            r.sigma_host.copy_(r.lp.sigma, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        t = self.now()
        self.stats.iterations += 1
        finished = []
        for r in done:
            req = r.req
            req.t_done = t
            req.sigma = r.sigma_host.numpy()
            req.lambdas = r.lp.lambdas.cpu().numpy() if r.lp.do_lambda else None
            req.bse_status = r.lp.bse_status.cpu().numpy()
            self.running.remove(r)
            self.admitted_bytes -= req.footprint
            self.stats.completed.append(req)
            finished.append(req)
        return finished

    def serve(self, requests: list[Request], realtime: bool = True) -> ServerStats:
        """Runs until every request is done.  With ``realtime`` a request is submitted once the clock passes
        its arrival time (an open-loop arrival process); otherwise all are submitted at once."""
        pending = sorted(requests, key=lambda r: r.arrival)
        self._t0 = time.perf_counter()
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        while pending or self.waiting or self.running:
            now = self.now()
            while pending and pending[0].arrival <= now:
                self.submit(pending.pop(0))
            if not self.waiting and not self.running:
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                continue
            self.step()
        return self.stats


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0) -> np.ndarray:
    """Arrival times of an open-loop Poisson process (exponential gaps), starting at 0."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=n)
    gaps[0] = 0.0
    return np.cumsum(gaps)


# (n_orb, nk, niv = niw) shapes of the serving mix: orbitals 1-3, small and mid momentum grids and boxes
SERVE_SHAPES = ((1, 16, 10), (1, 16, 20), (2, 8, 10), (2, 16, 10), (3, 8, 8), (3, 8, 12))
# The mixed-request workload's shape sets (orbitals {1, 2, 3} x grids {16^2, 32^2, 64^2} x boxes niv = niw
# {20, 40, 60}) without the shapes whose seeded inputs take more than seconds to generate on the host (two
# orbitals at niv = 60, three orbitals at niv >= 40): (n_orb, nk, niv).
C5_SERVE_SHAPES = tuple((n, nk, niv) for n in (1, 2, 3) for nk in (16, 32, 64) for niv in (20, 40, 60)
                        if not (n == 2 and niv == 60) and not (n == 3 and niv >= 40))


def serving_workload(n_requests: int = 24, rate_per_s: float = 20.0, seed: int = 5, precision: str = "fp64",
                     shapes=SERVE_SHAPES) -> list[Request]:
    """Seeded serving mix: each request draws a shape (orbitals, grid, frequency box), a temperature
    beta ~ U[5, 30] and an interaction U ~ U[2, 10] and gets its own synthetic inputs; arrivals are Poisson."""
    import dataclasses

    from . import synthetic

    rng = np.random.default_rng(seed)
    arrivals = poisson_arrivals(n_requests, rate_per_s, seed=seed)
    reqs = []
    for i in range(n_requests):
        n_orb, nk, niv = shapes[int(rng.integers(len(shapes)))]
        beta = float(rng.uniform(5.0, 30.0))
        u = float(rng.uniform(2.0, 10.0))
        base = {1: "c1", 2: "c4_bilayer", 3: "c3"}[n_orb]
        cfg = dataclasses.replace(synthetic.CONFIGS[base], name=f"serve{i}", nk=(nk, nk, 1), niw=niv, niv=niv,
                                  niv_shell=0, beta=beta, u=u, seed=1000 + i)
        reqs.append(Request(synthetic.make_inputs(cfg), arrival=float(arrivals[i]), precision=precision))
    return reqs

