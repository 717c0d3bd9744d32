"""Serving mode: a request loop over the island solve with continuous
batching.

A request is one field cutout with its source list and PSF model -- the
keyword set of ``island_fit`` (``bandnames``, ``data_minus_bg``, ``invvar``,
``psfs``, ``island_set``, ``buckets``, source arrays, ...).  Requests arrive
at any time (:meth:`Server.submit` returns a future).  ``workers`` threads
take them in arrival order; each plans its request on the host, estimates
the device memory the solve will hold (:func:`solver.estimate_device_bytes`)
and waits until that fits the HBM budget next to the requests already on the
device (requests that do not fit wait on the host: queued spill).  Admitted
requests solve concurrently, each on its worker's own library context
(resident field and PSF buffers, its own streams), so their kernels overlap
on the device while the host of another worker plans or unpacks; the solve
releases the interpreter lock while it runs.

A request's result does not depend on what else is in flight: every request
owns its device buffers and every kernel is deterministic, so a result in
the mix is bitwise the result alone.

Budget accounting: a worker's context keeps its padded field stacks between
requests (reused, and regrown when a larger cutout arrives), so those bytes
stay charged to the budget after the request that allocated them: a request
is charged its transient bytes (chunk buffers and the rest, released when
it finishes) plus the growth of its worker's resident field.  Freed chunk
buffers stay cached in the stream-ordered memory pool, but the pool never
holds more than the largest admitted total, so device memory stays within
the budget.

Latency of a request = time from its submission to its result (queueing,
planning, upload, solve, download and unpack).
"""

from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np


@dataclass
class RequestStats:
    """Timestamps (``time.perf_counter`` seconds) and sizes of one request."""
    rid: int
    submitted: float
    admitted: float = 0.0
    finished: float = 0.0
    device_bytes: int = 0
    n_islands: int = 0
    pixels: int = 0                # n_bands * H * W
    worker: int = -1

    @property
    def latency(self) -> float:
        return self.finished - self.submitted


@dataclass
class _Item:
    rid: int
    kwargs: dict
    future: Future
    stats: RequestStats


class Server:
    """Continuous-batching request server for one GPU.

    ``solve_fn(worker_state, kwargs, plan) -> result`` and
    ``plan_fn(kwargs) -> (plan, device_bytes, n_islands[, field_bytes])``
    default to the CUDA solver (:func:`default_plan`, :func:`default_solve`);
    ``field_bytes`` (part of ``device_bytes``, 0 when omitted) is what the
    worker keeps resident after the request.  Tests may pass host-only
    stand-ins to exercise admission without a GPU.
    """

    def __init__(self, device: int = 0, workers: int = 4,
                 hbm_budget_bytes: float = 160e9, precision: str = "mixed",
                 plan_fn: Optional[Callable] = None,
                 solve_fn: Optional[Callable] = None,
                 worker_init: Optional[Callable] = None):
        if workers < 1:
            raise ValueError("workers must be >= 1")
        self.device = int(device)
        self.precision = precision
        self.budget = float(hbm_budget_bytes)
        self.in_use = 0.0
        self.peak_in_use = 0.0
        self._plan = plan_fn or default_plan
        self._solve = solve_fn or default_solve
        self._init = worker_init or (lambda i: {"device": self.device,
                                                "precision": self.precision})
        self._q: "queue.Queue[Optional[_Item]]" = queue.Queue()
        self._cv = threading.Condition()
        self._next = 0
        self._lock = threading.Lock()
        self.stats: list[RequestStats] = []
        # bytes each worker keeps resident between requests (field stacks)
        self.resident = [0.0] * workers
        self._threads = [threading.Thread(target=self._run, args=(i,), daemon=True)
                         for i in range(workers)]
        self._closed = False
        for t in self._threads:
            t.start()

    # ------------------------------------------------------------------ API
    def submit(self, kwargs: dict) -> Future:
        """Queue one request (``island_fit`` keywords); returns a future of
        its ``IslandFitResult``."""
        if self._closed:
            raise RuntimeError("server is closed")
        with self._lock:
            rid = self._next
            self._next += 1
        st = RequestStats(rid, time.perf_counter())
        fut: Future = Future()
        self._q.put(_Item(rid, kwargs, fut, st))
        return fut

    def close(self):
        """Finish every queued request, then stop the workers."""
        if self._closed:
            return
        self._closed = True
        for _ in self._threads:
            self._q.put(None)
        for t in self._threads:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ internals
    def _acquire(self, nbytes: float):
        nbytes = min(float(nbytes), self.budget)   # a request larger than the budget runs alone
        with self._cv:
            while self.in_use + nbytes > self.budget:
                self._cv.wait()
            self.in_use += nbytes
            self.peak_in_use = max(self.peak_in_use, self.in_use)
        return nbytes

    def _release(self, nbytes: float):
        with self._cv:
            self.in_use -= nbytes
            self._cv.notify_all()

    def _run(self, wi: int):
        state = self._init(wi)
        while True:
            item = self._q.get()
            if item is None:
                break
            st = item.stats
            st.worker = wi
            held = 0.0
            try:
                planned = self._plan(item.kwargs)
                plan, nbytes, n_isl = planned[:3]
                field_bytes = float(planned[3]) if len(planned) > 3 else 0.0
                st.device_bytes, st.n_islands = int(nbytes), int(n_isl)
                d = item.kwargs.get("data_minus_bg")
                st.pixels = int(np.prod(np.shape(d))) if d is not None else 0
                # transient bytes plus the growth of this worker's resident
                # field; the resident part stays charged after the request
                growth = max(0.0, field_bytes - self.resident[wi])
                held = self._acquire(nbytes - field_bytes + growth)
                if growth:
                    keep = min(growth, held)
                    held -= keep
                    self.resident[wi] += keep
                st.admitted = time.perf_counter()
                res = self._solve(state, item.kwargs, plan)
                st.finished = time.perf_counter()
                item.future.set_result(res)
            except BaseException as e:  # noqa: BLE001 -- reported through the future
                st.finished = time.perf_counter()
                item.future.set_exception(e)
            finally:
                if held:
                    self._release(held)
                with self._lock:
                    self.stats.append(st)


def default_plan(kwargs: dict):
    """Host planning of one request: (plan, device bytes, fitted islands);
    plan None when every island takes the giant path (nothing to fit)."""
    from .solver import estimate_device_bytes, plan_field
    try:
        fp = plan_field(**kwargs)
    except ValueError as e:
        if "no buckets selected" not in str(e):
            raise
        return None, 0, 0          # every island takes the giant path
    nb, H, W = np.shape(kwargs["data_minus_bg"])
    nbytes = estimate_device_bytes(fp, nb, H, W,
                                   precision=kwargs.get("precision", "mixed"))
    field_bytes = 2 * 4 * nb * (H + 2 * fp.PAD) * (W + 2 * fp.PAD)
    return fp, nbytes, sum(p.n_islands for p, _ in fp.classes), field_bytes


def default_solve(state: dict, kwargs: dict, plan):
    """Solve one request on the worker's context (created on first use and
    kept: its field and PSF buffers are reused and regrown as needed)."""
    from . import _lib
    from .solver import DeviceField, IslandFitJob, giant_only_result
    if plan is None:
        return giant_only_result(**kwargs)
    if "ctx" not in state:
        state["ctx"] = _lib.Context(state["device"])
    kw = dict(kwargs)
    kw.setdefault("precision", state["precision"])
    fld = DeviceField.from_unpadded(kw["data_minus_bg"], kw["invvar"], plan.PAD,
                                    device=state["device"], context=state["ctx"])
    job = IslandFitJob(**kw, device=state["device"], field=fld, plan=plan)
    try:
        job.solve()
        return job.result()
    finally:
        job.close()


def latency_summary(stats: list[RequestStats]) -> dict:
    """p50/p95/p99 latency (ms), islands/s and pixels/s over a request set
    (throughput over the span from the first submission to the last
    result)."""
    ok = [s for s in stats if s.finished > 0]
    if not ok:
        return {}
    lat = np.array([s.latency for s in ok]) * 1e3
    span = max(s.finished for s in ok) - min(s.submitted for s in ok)
    return {"requests": len(ok),
            "p50_ms": float(np.percentile(lat, 50)),
            "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()),
            "islands_per_s": float(sum(s.n_islands for s in ok) / span),
            "pixels_per_s": float(sum(s.pixels for s in ok) / span),
            "span_s": float(span)}


def poisson_stream(server: Server, requests: list[dict], rate_hz: float,
                   seed: int = 0) -> list:
    """Submit ``requests`` with exponential inter-arrival times of mean
    1 / rate_hz; returns the futures (in submission order)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, len(requests))
    t0 = time.perf_counter()
    due = t0
    futs = []
    for kw, g in zip(requests, gaps):
        due += g
        wait = due - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        futs.append(server.submit(kw))
    return futs
