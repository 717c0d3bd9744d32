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

:class:`PackedServer` packs instead: the requests admitted while the device
is busy are solved together as ONE library job holding every request's
chunks (each chunk bound to its own request's field and PSF on the device),
so their islands of every size run through the same LM-loop kernels -- with
the "queue" engine, one persistent work-queue kernel per kernel kind and LM
phase over the islands of all packed requests, converged islands retired on
the device.  Results are again bitwise those of each request alone: a
chunk's islands are computed the same whatever else the job holds.

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
    pack: int = -1                 # PackedServer: the pack it was solved in
    pack_size: int = 0

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
        try:
            state, init_error = self._init(wi), None
        except BaseException as e:  # noqa: BLE001 -- reported to every request it takes
            state, init_error = None, e
        while True:
            item = self._q.get()
            if item is None:
                break
            st = item.stats
            st.worker = wi
            held = 0.0
            try:
                if init_error is not None:
                    raise init_error
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


@dataclass
class _Admitted:
    item: _Item
    plan: object
    charged: float                 # budget bytes held while in flight
    field_bytes: float
    key: object                    # requests of one pack share it


class PackedServer:
    """Continuous-batching server that packs requests into one solve.

    ``planners`` host threads take requests in arrival order, plan them and
    admit them by the HBM budget (a request waits on the host until its
    device bytes fit next to those in flight).  ``engines`` device threads,
    each with its own library context, take every admitted request not yet
    taken (up to ``max_pack``, sharing the first one's LM step limit) as one
    pack: upload each request's field and PSF, add all their chunks to one
    job, solve it once (``engine``/``lanes`` as ``uph_job_set_engine``) and
    unpack each request's result.  Requests that arrive while a pack is on
    the device are admitted meanwhile and form the next pack; with several
    engines, packs upload and unpack while others solve (four planners and
    four engines gave the highest islands/s on the serving request pool).

    ``pack_fn(engine_state, [(kwargs, plan), ...]) -> [result or exception]``
    and ``plan_fn`` (as :class:`Server`) default to the CUDA solver
    (:func:`default_pack`, :func:`default_plan`); tests pass host stand-ins.
    A request fails alone: an exception in its planning, upload or unpacking
    reaches its own future only.
    """

    def __init__(self, device: int = 0, planners: int = 4, engines: int = 4,
                 hbm_budget_bytes: float = 160e9, precision: str = "mixed",
                 max_pack: int = 64, engine: str = "chunks", lanes: int = 0,
                 plan_fn: Optional[Callable] = None,
                 pack_fn: Optional[Callable] = None,
                 engine_init: Optional[Callable] = None,
                 key_fn: Optional[Callable] = None):
        if planners < 1 or engines < 1 or max_pack < 1:
            raise ValueError("planners, engines and max_pack must be >= 1")
        self.device = int(device)
        self.precision = precision
        self.budget = float(hbm_budget_bytes)
        self.max_pack = int(max_pack)
        self.in_use = 0.0
        self.peak_in_use = 0.0
        self._plan = plan_fn or default_plan
        self._pack = pack_fn or default_pack
        self._key = key_fn or (lambda kw: kw.get("max_steps"))
        self._init = engine_init or (lambda i: {"device": self.device,
                                                "precision": self.precision,
                                                "engine": engine, "lanes": int(lanes)})
        self._q: "queue.Queue[Optional[_Item]]" = queue.Queue()
        self._cv = threading.Condition()            # budget
        self._rcv = threading.Condition()           # admitted requests
        self._ready: list[_Admitted] = []
        self._planning = int(planners)
        self._next = 0
        self._npack = 0
        self._lock = threading.Lock()
        self.stats: list[RequestStats] = []
        self.packs: list[int] = []                  # size of every pack solved
        self.resident = [0.0] * engines             # field bytes kept per engine
        self._planners = [threading.Thread(target=self._plan_loop, daemon=True)
                          for _ in range(planners)]
        self._engines = [threading.Thread(target=self._engine_loop, args=(i,), daemon=True)
                         for i in range(engines)]
        self._closed = False
        for t in self._planners + self._engines:
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
        """Finish every queued request, then stop the threads."""
        if self._closed:
            return
        self._closed = True
        for _ in self._planners:
            self._q.put(None)
        for t in self._planners:
            t.join()
        for t in self._engines:
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

    def _finish(self, item: _Item, result=None, error=None):
        item.stats.finished = time.perf_counter()
        with self._lock:
            self.stats.append(item.stats)
        if error is not None:
            item.future.set_exception(error)
        else:
            item.future.set_result(result)

    def _plan_loop(self):
        while True:
            item = self._q.get()
            if item is None:
                break
            st = item.stats
            try:
                planned = self._plan(item.kwargs)
                plan, nbytes, n_isl = planned[:3]
                fb = float(planned[3]) if len(planned) > 3 else 0.0
                st.device_bytes, st.n_islands = int(nbytes), int(n_isl)
                d = item.kwargs.get("data_minus_bg")
                st.pixels = int(np.prod(np.shape(d))) if d is not None else 0
                key = self._key(item.kwargs)
            except BaseException as e:  # noqa: BLE001 -- reported through the future
                self._finish(item, error=e)
                continue
            held = self._acquire(nbytes)
            st.admitted = time.perf_counter()
            with self._rcv:
                self._ready.append(_Admitted(item, plan, held, fb, key))
                self._rcv.notify()
        with self._rcv:
            self._planning -= 1
            self._rcv.notify_all()

    def _take(self) -> list:
        """Every admitted request sharing the oldest one's key, oldest first
        (called with the ready lock held)."""
        key = self._ready[0].key
        pack, rest = [], []
        for a in self._ready:
            if a.key == key and len(pack) < self.max_pack:
                pack.append(a)
            else:
                rest.append(a)
        self._ready = rest
        return pack

    def _engine_loop(self, ei: int):
        try:
            state, init_error = self._init(ei), None
        except BaseException as e:  # noqa: BLE001 -- reported to every request it takes
            state, init_error = None, e
        while True:
            with self._rcv:
                while not self._ready and self._planning > 0:
                    self._rcv.wait()
                if not self._ready:
                    break
                pack = self._take()
            with self._lock:
                pid = self._npack
                self._npack += 1
                self.packs.append(len(pack))
            for a in pack:
                a.item.stats.worker, a.item.stats.pack = ei, pid
                a.item.stats.pack_size = len(pack)
            try:
                if init_error is not None:
                    raise init_error
                outs = list(self._pack(state, [(a.item.kwargs, a.plan) for a in pack]))
                if len(outs) != len(pack):
                    raise RuntimeError(f"pack_fn returned {len(outs)} results for "
                                       f"{len(pack)} requests")
            except BaseException as e:  # noqa: BLE001 -- every request of the pack
                outs = [e] * len(pack)
            # the context keeps the last uploaded field between packs: at
            # most the largest field seen stays charged to the budget
            new_res = max([self.resident[ei]] +
                          ([a.field_bytes for a in pack] if init_error is None else []))
            growth = new_res - self.resident[ei]
            self.resident[ei] = new_res
            with self._cv:
                self.in_use -= sum(a.charged for a in pack) - growth
                self._cv.notify_all()
            for a, r in zip(pack, outs):
                if isinstance(r, BaseException):
                    self._finish(a.item, error=r)
                else:
                    self._finish(a.item, result=r)


def default_pack(state: dict, reqs: list) -> list:
    """Solve planned requests as one job on the engine's context: every
    request's field and PSF uploaded (a field bound by the job's chunks stays
    allocated while later fields are uploaded), all chunks added to one job,
    one solve, then each request's rows unpacked.  Returns one result or
    exception per request.  If the packed solve itself fails, each request
    is solved alone so that one bad request does not fail the others."""
    from . import _lib
    from .solver import DeviceField, IslandFitJob, giant_only_result
    if "ctx" not in state:
        state["ctx"] = _lib.Context(state["device"])
    ctx = state["ctx"]
    out: list = [None] * len(reqs)
    fits = []
    job = _lib.Job(ctx)
    try:
        job.set_engine(state.get("engine", "chunks"), int(state.get("lanes", 0)))
        for i, (kw, plan) in enumerate(reqs):
            try:
                if plan is None:
                    out[i] = giant_only_result(**kw)
                    continue
                kw = dict(kw)
                kw.setdefault("precision", state["precision"])
                fld = DeviceField.from_unpadded(kw["data_minus_bg"], kw["invvar"], plan.PAD,
                                                device=state["device"], context=ctx)
                fits.append((i, IslandFitJob(**kw, device=state["device"], field=fld,
                                             plan=plan, job=job)))
            except BaseException as e:  # noqa: BLE001 -- this request only
                out[i] = e
        if fits:
            try:
                job.solve(max(f.max_steps for _, f in fits))
            except BaseException:  # noqa: BLE001 -- retried one by one below
                fits_alone, fits = fits, []
                job.close()
                for i, _ in fits_alone:
                    try:
                        out[i] = default_solve(state, reqs[i][0], reqs[i][1])
                    except BaseException as e:  # noqa: BLE001
                        out[i] = e
            for i, f in fits:
                try:
                    out[i] = f.result()
                except BaseException as e:  # noqa: BLE001
                    out[i] = e
    finally:
        job.close()
    return out


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
