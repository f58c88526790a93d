"""A serving loop over resident H-matrices: continuous batching of products and
kernel-ridge solves, construction of new point sets under an HBM budget, and
per-request latency.

No reference counterpart (hmglib is a library of blocking calls on one H-matrix).
The loop keeps compressed H-matrices resident on the device, each with its own CUDA
stream so that work on different H-matrices overlaps on the GPU, and admits requests
as they arrive:

* ``Matvec(mid, x)``: requests queued on the same H-matrix are packed, up to 32 at a
  time, into one ``hmg_matvec_multi`` call (the stored H-matrix is read once for the
  whole batch).  A request that arrives while a batch is on the GPU joins the next.
* ``Solve(mid, B, shift)``: kernel-ridge CG on (H + shift I) X = B for the columns of
  B (at most MAX_SOLVES per H-matrix at a time, the others wait), run by the
  library's block CG (``hmg_cg_multi_*``): one multi-vector product per iteration for
  all columns, FP64 vector updates and inner products on the H-matrix's stream,
  residual norms read back asynchronously (no host synchronisation), converged
  columns frozen, and FP64-product refinement of the true residual, so the result
  solves the stored operator to ``tol``.  Each poll of the loop enqueues at most one
  iteration, so solve iterations and product batches on the same H-matrix
  interleave.
* ``Build(points, ...)``: a new point set compressed on a worker thread with its own
  stream, admitted only when the budget holds its estimated bytes (idle H-matrices
  built by earlier requests are evicted, least recently used first).

``run(requests)`` replays an arrival timeline (seconds from the start) and returns
the requests with their completion times; latency = completion - arrival, measured
on the host clock when the result's CUDA event has completed.

Latency targets (``Server(slo_s={"matvec": ..., "solve": ...})``): a product or solve
is admitted only if its predicted completion fits its class's target; otherwise it is
refused at once (``rejected`` set, no result).  The prediction: the work queued and
running on its own H-matrix's stream plus its own runs in order (A seconds); the other
H-matrices' streams interleave with it on the GPU, adding at most their outstanding
work and at most (busy streams - 1) x A.  Work is counted in GPU seconds of a product
batch and of a solve iteration per resident H-matrix (exponential averages of CUDA-event
timings, seeded from the stored bytes at HBM speed) and the mean iterations per solve.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .hmatrix import HMatrix

MAX_BATCH = 32       # vectors per product pass
MAX_SOLVES = 2       # solves advancing at once per H-matrix (their vectors live on the device)
HBM_BYTES_PER_S = 5.0e12   # seed of the service-time estimates: stored bytes read at this rate
EWMA = 0.25          # weight of a new timing in the service-time estimates


@dataclass
class Matvec:
    mid: int
    x: np.ndarray
    arrival: float = 0.0
    y: np.ndarray | None = None
    done: float | None = None
    batch: int = 0
    rejected: str | None = None


@dataclass
class Solve:
    mid: int
    B: np.ndarray            # (k, n) right-hand sides
    shift: float
    tol: float = 1e-5
    maxit: int = 2000
    arrival: float = 0.0
    X: np.ndarray | None = None
    iters: int = 0
    relres: np.ndarray | None = None
    done: float | None = None
    rejected: str | None = None


@dataclass
class Build:
    points: np.ndarray       # (dim, n)
    kind: int
    param: float
    eps: float
    precision: int
    arrival: float = 0.0
    mid: int | None = None
    done: float | None = None
    rejected: str | None = None


@dataclass
class _Resident:
    H: HMatrix
    stream: object
    nbytes: int
    pinned: bool
    last_use: float = 0.0
    matvecs: collections.deque = field(default_factory=collections.deque)
    waiting_solves: collections.deque = field(default_factory=collections.deque)
    solves: list = field(default_factory=list)
    inflight: list = field(default_factory=list)   # (event, finisher)
    batch_s: float = 0.0     # GPU seconds of one product batch (estimate)
    iter_s: float = 0.0      # GPU seconds of one solve iteration (estimate)


def outstanding_seconds(queued_batches, running_batches, solve_iters_left, batch_s, iter_s):
    """GPU seconds of the work queued and running, per resident H-matrix: its product
    batches (queued and in flight) times the batch estimate plus the solve iterations
    still to run times the iteration estimate."""
    return [(q + r) * b + it * i for q, r, it, b, i in
            zip(queued_batches, running_batches, solve_iters_left, batch_s, iter_s)]


def predict_latency(own_queue_s: float, own_s: float, others_s: float, busy_streams: int) -> float:
    """Completion of a request: its stream's work and its own in order (A), plus the
    other streams' work interleaved with it: at most all of it and at most
    (busy streams - 1) x A."""
    a = own_queue_s + own_s
    return a + min(others_s, max(0, busy_streams - 1) * a)


def admit(predicted_s: float, target_s: float | None) -> bool:
    """A request is admitted when its predicted completion fits its latency target."""
    return target_s is None or predicted_s <= target_s


def ewma(old: float, new: float, w: float = EWMA) -> float:
    return new if old <= 0.0 else (1.0 - w) * old + w * new


def build_hmatrix(points, kind, param, eps, precision, stream=None, max_rank=64, eta=1.5, leaf=None):
    # leaf: 64 (2D) / 128 (3D) unless given
    """Set up and compress one H-matrix (synchronous on `stream`)."""
    dim, n = points.shape
    H = HMatrix(n, n, dim, stream=stream)
    H.set_points(0, points)
    H.set_points(1, points)
    H.setup(eta, leaf or (64 if dim == 2 else 128), rule=L.ADMISSIBLE_MIN)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(max_rank, eps, precision)
    H.precompute_dense(L.PREC_FP32 if precision == L.PREC_MIXED else precision)
    H.synchronize()
    return H


def resident_bytes(H: HMatrix) -> int:
    i = H.info()
    return int(i["near_bytes"] + i["far_bytes"] + 8 * 4 * (i["n1"] + i["n2"]))


class Server:
    def __init__(self, budget_bytes: float, device: int = 0, slo_s: dict | None = None):
        import torch
        self.torch = torch
        self.device = device
        self.budget = int(budget_bytes)
        self.slo = dict(slo_s or {})   # class name ("matvec", "solve") -> latency target, seconds
        self.iters_per_solve = 30.0    # estimate, updated as solves finish
        self.res: dict[int, _Resident] = {}
        self.next_id = 0
        self.builds: collections.deque = collections.deque()
        self.build_thread: threading.Thread | None = None
        self.build_result = None
        self.bytes_per_point = None

    # -- residency -------------------------------------------------------------
    def used_bytes(self) -> int:
        return sum(r.nbytes for r in self.res.values())

    def add(self, H: HMatrix, stream, pinned: bool = True) -> int:
        mid = self.next_id
        self.next_id += 1
        nb = resident_bytes(H)
        # seeds: one read of the stored bytes per batch; a solve iteration reads them once
        # for all its vectors plus the vector updates
        self.res[mid] = _Resident(H, stream, nb, pinned, batch_s=nb / HBM_BYTES_PER_S,
                                  iter_s=1.5 * nb / HBM_BYTES_PER_S)
        bpp = self.res[mid].nbytes / max(1, H.n1)
        self.bytes_per_point = bpp if self.bytes_per_point is None else max(self.bytes_per_point, bpp)
        return mid

    def _evict_for(self, need: int) -> bool:
        while self.used_bytes() + need > self.budget:
            idle = [(r.last_use, mid) for mid, r in self.res.items()
                    if not r.pinned and not r.matvecs and not r.solves and not r.waiting_solves
                    and not r.inflight]
            if not idle:
                return False
            _, mid = min(idle)
            self.res.pop(mid).H.close()
        return True

    # -- request intake ----------------------------------------------------------
    def outstanding(self) -> dict:
        mids = list(self.res)
        rs = [self.res[m] for m in mids]
        left = [sum(max(1.0, self.iters_per_solve - st["it"]) for st in r.solves if st["final"] is None)
                + self.iters_per_solve * len(r.waiting_solves) for r in rs]
        w = outstanding_seconds([-(-len(r.matvecs) // MAX_BATCH) for r in rs], [len(r.inflight) for r in rs],
                                left, [r.batch_s for r in rs], [r.iter_s for r in rs])
        return dict(zip(mids, w))

    def submit(self, req, now: float):
        if isinstance(req, (Matvec, Solve)):
            r = self.res[req.mid]
            own = r.batch_s if isinstance(req, Matvec) else self.iters_per_solve * r.iter_s
            cls = "matvec" if isinstance(req, Matvec) else "solve"
            w = self.outstanding()
            busy = 1 + sum(1 for m, v in w.items() if m != req.mid and v > 0)
            pred = predict_latency(w[req.mid], own, sum(v for m, v in w.items() if m != req.mid), busy)
            if not admit(pred, self.slo.get(cls)):
                req.rejected = f"predicted {pred:.2f} s > {cls} target {self.slo[cls]:.2f} s"
                req.done = time.perf_counter()
                return
            (r.matvecs if isinstance(req, Matvec) else r.waiting_solves).append(req)
        else:
            self.builds.append(req)

    # -- products ----------------------------------------------------------------
    def _launch_matvecs(self, r: _Resident, now: float):
        torch = self.torch
        batch = [r.matvecs.popleft() for _ in range(min(MAX_BATCH, len(r.matvecs)))]
        with torch.cuda.stream(r.stream):
            e_start = torch.cuda.Event(enable_timing=True)
            e_start.record(r.stream)
            X = torch.from_numpy(np.stack([q.x for q in batch])).pin_memory().cuda(non_blocking=True)
            Y = torch.empty(len(batch), r.H.n1, dtype=torch.float64, device="cuda")
            if len(batch) == 1:
                r.H.matvec(X[0], Y[0])
            else:
                r.H.matvec_multi(X, Y)
            Yh = torch.empty(Y.shape, dtype=torch.float64, pin_memory=True)
            Yh.copy_(Y, non_blocking=True)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(r.stream)

        def finish(t):
            for j, q in enumerate(batch):
                q.y = Yh[j].numpy().copy()
                q.done = t
                q.batch = len(batch)
            r.batch_s = ewma(r.batch_s, e_start.elapsed_time(ev) * 1e-3)
        r.inflight.append((ev, finish, (X, Y)))
        r.last_use = now

    # -- block CG on the library (hmg_cg_multi_*: one multi-vector product per iteration) --
    def _start_solve(self, req: Solve):
        torch = self.torch
        r = self.res[req.mid]
        with torch.cuda.stream(r.stream):
            B = torch.from_numpy(np.ascontiguousarray(req.B)).pin_memory().cuda(non_blocking=True)
            X = torch.zeros_like(B)
        cg = r.H.cg_multi(B, X, req.shift, tol=req.tol, maxit=req.maxit, refine=True)
        return {"req": req, "B": B, "X": X, "cg": cg, "final": None, "events": collections.deque(), "it": 0}

    def _step_solve(self, r: _Resident, st, now: float):
        """Advance one solve by at most one enqueued iteration; True once its result
        has reached the host.  The library keeps the recurrence on the device and
        decides convergence from residual norms read back asynchronously."""
        torch = self.torch
        req = st["req"]
        if st["final"] is not None:
            ev, Xh, rel, it = st["final"]
            if not ev.query():
                return False
            req.X, req.iters, req.relres, req.done = Xh.numpy().copy(), it, rel, time.perf_counter()
            self.iters_per_solve = ewma(self.iters_per_solve, float(it))
            st["cg"].close()
            return True
        # iteration timings: consecutive recorded events that have completed
        evs = st["events"]
        while len(evs) >= 2 and evs[1].query():
            r.iter_s = ewma(r.iter_s, evs[0].elapsed_time(evs[1]) * 1e-3)
            evs.popleft()
        cg = st["cg"]
        done, it, rel = cg.poll()
        st["it"] = it
        if done:
            with torch.cuda.stream(r.stream):
                Xh = torch.empty(st["X"].shape, dtype=torch.float64, pin_memory=True)
                Xh.copy_(st["X"], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(r.stream)
            st["final"] = (ev, Xh, rel, it)
            return False
        if cg.advance():
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(r.stream)
            evs.append(ev)
        r.last_use = now
        return False

    # -- construction on a worker thread -----------------------------------------------
    def _poll_builds(self, now: float):
        torch = self.torch
        if self.build_thread is not None:
            if self.build_thread.is_alive():
                return
            self.build_thread.join()
            req, H, stream, err = self.build_result
            self.build_thread = None
            if err is not None:
                req.rejected = err
            else:
                req.mid = self.add(H, stream, pinned=False)
            req.done = time.perf_counter()
        if not self.builds:
            return
        req = self.builds[0]
        est = int((self.bytes_per_point or 0) * req.points.shape[1] * 1.5)
        pinned = sum(r.nbytes for r in self.res.values() if r.pinned)
        if pinned + est > self.budget:
            # can never fit beside the pinned H-matrices: refuse it now
            self.builds.popleft()
            req.rejected = f"needs ~{est / 1e9:.1f} GB beside {pinned / 1e9:.1f} GB pinned (budget {self.budget / 1e9:.1f} GB)"
            req.done = time.perf_counter()
            return
        if not self._evict_for(est):
            return  # wait for resident work to drain
        self.builds.popleft()
        stream = torch.cuda.Stream()

        def work():
            torch.cuda.set_device(self.device)
            try:
                H = build_hmatrix(req.points, req.kind, req.param, req.eps, req.precision,
                                  stream=stream.cuda_stream)
                self.build_result = (req, H, stream, None)
            except Exception as e:  # the request fails, the server goes on
                self.build_result = (req, None, stream, str(e))
        self.build_thread = threading.Thread(target=work, daemon=True)
        self.build_thread.start()

    # -- the loop --------------------------------------------------------------------------
    def _poll(self, now: float) -> bool:
        busy = False
        for r in list(self.res.values()):
            keep = []
            for ev, finish, hold in r.inflight:
                if ev.query():
                    finish(time.perf_counter())
                else:
                    keep.append((ev, finish, hold))
            r.inflight = keep
            # one product batch in flight per H-matrix; solves advance between batches
            if r.matvecs and not r.inflight:
                self._launch_matvecs(r, now)
            while r.waiting_solves and len(r.solves) < MAX_SOLVES:
                r.solves.append(self._start_solve(r.waiting_solves.popleft()))
            still = []
            for st in r.solves:
                if not self._step_solve(r, st, now):
                    still.append(st)
            r.solves = still
            busy |= bool(r.matvecs or r.inflight or r.solves or r.waiting_solves)
        self._poll_builds(now)
        busy |= bool(self.builds or self.build_thread is not None)
        return busy

    def run(self, requests, time_limit: float = 600.0):
        """Replay `requests` (each with .arrival in seconds from the start)."""
        order = sorted(requests, key=lambda q: q.arrival)
        t0 = time.perf_counter()
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < len(order) and order[i].arrival <= now:
                self.submit(order[i], now)
                i += 1
            busy = self._poll(now)
            if i >= len(order) and not busy:
                break
            if now > time_limit:
                left = collections.Counter(type(q).__name__ for q in order if q.done is None)
                raise TimeoutError(f"serving run exceeded its time limit; unfinished: {dict(left)}")
            if not busy and i < len(order):
                time.sleep(max(0.0, min(order[i].arrival - now, 1e-3)))
        for q in order:
            if q.done is not None:
                q.done -= t0
        return order, time.perf_counter() - t0


def latency_summary(reqs):
    """p50 / p99 / max latency per request class over the requests that completed
    (refused ones are counted apart)."""
    out = {}
    for name, cls in (("matvec", Matvec), ("solve", Solve), ("build", Build), ("all", object)):
        mine = [q for q in reqs if isinstance(q, cls)]
        lat = np.array([q.done - q.arrival for q in mine if q.done is not None and getattr(q, "rejected", None) is None])
        refused = sum(1 for q in mine if getattr(q, "rejected", None) is not None)
        if lat.size or refused:
            out[name] = {"count": int(lat.size), "refused": int(refused)}
            if lat.size:
                out[name].update({"p50_ms": float(np.percentile(lat, 50) * 1e3),
                                  "p99_ms": float(np.percentile(lat, 99) * 1e3), "max_ms": float(lat.max() * 1e3)})
    return out


def poisson_requests(n_requests: int, rate: float, sizes, seed: int = 4, mix=(0.80, 0.15, 0.05),
                     solve_rhs: int = 8, build_lo: float = 14.0, build_hi: float = 18.0,
                     kind: int = L.KERNEL_MATERN32, param: float = 0.2, eps: float = 1e-5,
                     precision: int = L.PREC_MIXED, shift_per_point: float = 1e-4, tol: float = 1e-5):
    """The serving mix: Poisson arrivals at `rate` per second (SplitMix64 stream
    `seed`); each request is a single-vector product (mix[0]), a `solve_rhs`-vector
    kernel-ridge solve (mix[1]) or a new uniform 3D point set of 2^U[build_lo,
    build_hi] points (mix[2]).  Products and solves pick one of the resident
    H-matrices (`sizes[i]` points each) uniformly; vectors are U[-1, 1]."""
    from . import synth
    u = synth.uniform01(seed, 4 * n_requests)
    t = np.cumsum(-np.log1p(-u[:n_requests]) / rate)
    out = []
    for i in range(n_requests):
        a, b = u[n_requests + i], u[2 * n_requests + i]
        mid = min(int(b * len(sizes)), len(sizes) - 1)
        vseed = (seed << 24) + i
        if a < mix[0]:
            out.append(Matvec(mid, synth.uniform01(vseed, sizes[mid]) * 2.0 - 1.0, arrival=float(t[i])))
        elif a < mix[0] + mix[1]:
            B = (synth.uniform01(vseed, solve_rhs * sizes[mid]) * 2.0 - 1.0).reshape(solve_rhs, sizes[mid])
            out.append(Solve(mid, B, shift_per_point * sizes[mid], tol=tol, maxit=300, arrival=float(t[i])))
        else:
            n = int(round(2.0 ** (build_lo + (build_hi - build_lo) * u[3 * n_requests + i])))
            out.append(Build(synth.uniform_points(n, 3, vseed), kind, param, eps, precision, arrival=float(t[i])))
    return out
