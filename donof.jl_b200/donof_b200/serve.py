"""Continuous batching of GNOF energy jobs on one GPU.

Requests (core Hamiltonian, RI tensor b, starting orbitals and occupations,
parameters, precision) are admitted while their device footprint fits the
memory budget; each admitted job runs the energy loop of ``optimize.energy``
(or the mixed-precision form with closing FP64 iterations) on its own library
context, i.e. its own CUDA stream, so the device work of all jobs in flight
overlaps on the GPU.  A job that arrives while others run is admitted as soon
as a slot and enough memory are free; results are returned per ticket.

Admission policy (``Admission``): first fit over the queue in arrival order,
bounded by ``max_inflight`` slots and the memory budget; the head of the queue
is never passed over more than ``max_bypass`` times, so a large job cannot be
starved by a stream of small ones.  The policy is separate from the executor so
that it can be exercised without a GPU.

The device footprint of a job is its RI tensor (FP64, plus the bf16 split in the
mixed form) and the per-call scratch of the transforms (tmp, b_pq, W), the
orbital state and the partial sums (see ``footprint``).
"""
from __future__ import annotations

import copy
import functools
import itertools
import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional

import numpy as np

from .param import Param

PRECISIONS = ("fp64", "mixed", "mixed_refined", "auto")

# "auto": the mixed form with closing FP64 iterations where its bulk contractions
# pay off, the FP64 form for small jobs, whose steps are bound by launch and
# synchronisation latency rather than by the contractions (the mixed phase would
# only add iterations there).  Threshold on nbf * nbf5 * naux, the size of the
# three-index transform.
AUTO_MIXED_MIN_WORK = 2.0e7


# The FP64 form's first contraction runs on the tensor cores from int8 digit
# slices of b (ozaki.cu) for jobs of at least this many basis functions: there
# it is faster than the DMMA GEMM (nbf = 202: 450 against 746 us per call,
# nbf = 256: 130 against 290 us); below, the contraction is a few microseconds
# either way and the slices would only cost memory.
FP64_TC_MIN_NBF = 128


def use_fp64_tc(fp64_tc: Optional[bool], nbf: int) -> bool:
    return nbf >= FP64_TC_MIN_NBF if fp64_tc is None else bool(fp64_tc)


def resolve_precision(precision: str, nbf: int, nbf5: int, naux: int) -> str:
    if precision != "auto":
        return precision
    return "mixed_refined" if nbf * nbf5 * naux >= AUTO_MIXED_MIN_WORK else "fp64"


@dataclass
class Request:
    """One energy job.  b is the host RI tensor b[m, n, P] (nbf x nbf x naux,
    column-major); C the starting orbitals; gamma the starting occupation
    parameters (the reference's guess when None)."""
    H: np.ndarray
    b: np.ndarray
    C: np.ndarray
    p: Param
    gamma: Optional[np.ndarray] = None
    precision: str = "fp64"
    E_nuc: float = 0.0
    maxit: Optional[int] = None
    tag: object = None
    fp64_tc: Optional[bool] = None  # FP64 contraction on the tensor cores (None: nbf >= FP64_TC_MIN_NBF)


@dataclass
class Result:
    ticket: int
    E_elec: float = float("nan")
    E_tot: float = float("nan")
    converged: bool = False
    iterations: int = 0
    C: Optional[np.ndarray] = None
    n: Optional[np.ndarray] = None
    error: Optional[str] = None
    t_submit: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0
    footprint: int = 0
    tag: object = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


def footprint(nbf: int, naux: int, nbf5: int, precision: str, fp64_tc: bool = False) -> int:
    """Device bytes a job holds while it runs (upper estimate)."""
    b = 8 * nbf * nbf * naux
    if fp64_tc:  # b's int8 digit slices (7 per element, rows padded to 16 bytes) and row scales
        b += 7 * nbf * (-(-nbf // 16) * 16) * naux + 8 * nbf * naux
    nb = (nbf + 63) // 64
    split = 4 * 64 * nb * nbf * naux if precision != "fp64" else 0
    # FP64 transforms: tmp (nbf nbf5 naux), b_pq and W (nbf5^2 naux each)
    scratch = 8 * (nbf * nbf5 * naux + 2 * nbf5 * nbf5 * naux)
    if precision != "fp64" and (nbf > 256 or nbf5 > 64):
        # general-shape mixed pipeline: tmp split, FP32 b_pq, W split, Y partials
        ldm, ldq = -(-nbf // 8) * 8, -(-nbf5 // 8) * 8
        scratch += 4 * (ldm * nbf5 * naux + nbf5 * nbf5 * naux + ldq * nbf5 * naux + 148 * nbf * nbf5)
    small = 8 * (4 * nbf * nbf + 16 * nbf * nbf5) + (32 << 20)
    return b + split + scratch + small


class Admission:
    """First-fit admission by memory budget and slots (no GPU involved)."""

    def __init__(self, budget_bytes: int, max_inflight: int = 8, max_bypass: int = 4):
        self.budget = int(budget_bytes)
        self.max_inflight = max_inflight
        self.max_bypass = max_bypass
        self.used = 0
        self.inflight = 0
        self.queue: Deque[tuple] = deque()  # (ticket, bytes)
        self._head_bypassed = 0

    def push(self, ticket: int, nbytes: int) -> None:
        if nbytes > self.budget:
            raise ValueError(f"job needs {nbytes} bytes, more than the whole budget of {self.budget}")
        self.queue.append((ticket, nbytes))

    def take(self) -> List[tuple]:
        """Tickets (with their bytes) to start now, in the order they start."""
        started = []
        while self.inflight < self.max_inflight and self.queue:
            pick = None
            for i, (t, nb) in enumerate(self.queue):
                if self.used + nb <= self.budget:
                    if i > 0 and self._head_bypassed >= self.max_bypass:
                        break  # the head waits for memory; nobody passes it any more
                    pick = i
                    break
            if pick is None:
                break
            t, nb = self.queue[pick]
            del self.queue[pick]
            if pick > 0:
                self._head_bypassed += 1
            else:
                self._head_bypassed = 0
            self.used += nb
            self.inflight += 1
            started.append((t, nb))
        return started

    def release(self, nbytes: int) -> None:
        self.used -= nbytes
        self.inflight -= 1

    def remove(self, ticket: int) -> bool:
        """Drops a queued ticket (a cancelled job); False if it is not queued."""
        for i, (t, _) in enumerate(self.queue):
            if t == ticket:
                del self.queue[i]
                if i == 0:
                    self._head_bypassed = 0
                return True
        return False

    def take_group(self, eligible: Callable[[int], bool], max_group: int, min_group: int = 2,
                   scale: float = 2.0) -> List[tuple]:
        """Queued tickets to run together as one group on one slot: when the head
        of the queue is eligible, the eligible tickets in arrival order (at most
        max_group) whose bytes, times ``scale`` (a group holds each job's scratch
        twice: the grouped loop's and the per-job steps'), fit the free budget.
        Fewer than min_group: nothing (the single-job path takes them)."""
        if self.inflight >= self.max_inflight or not self.queue or not eligible(self.queue[0][0]):
            return []
        head = self.queue[0][0]
        room = self.budget - self.used
        group = []
        for t, nb in self.queue:
            if len(group) >= max_group:
                break
            need = int(scale * nb)
            if eligible(t) and need <= room:
                group.append((t, need))
                room -= need
        if len(group) < min_group:
            return []
        picked = {t for t, _ in group}
        if head in picked:
            self._head_bypassed = 0
        else:  # the head does not fit: the group passes it over, as take() counts it
            if self._head_bypassed >= self.max_bypass:
                return []
            self._head_bypassed += 1
        self.queue = deque(q for q in self.queue if q[0] not in picked)
        self.used += sum(nb for _, nb in group)
        self.inflight += 1
        return group

    def release_group(self, nbytes_total: int) -> None:
        self.release(nbytes_total)


def run_energy(req: Request, device: int, cta_limit: int = 0) -> Result:
    """Executor: the energy loop of one request on its own context and stream;
    cta_limit caps the CTAs of a small job's persistent kernels (0: one per SM).
    Large jobs (those auto runs in the mixed form) keep every SM: their
    contractions fill the GPU, the small jobs' steps are latency-bound."""
    from . import api
    from .optimize import energy, energy_mixed_refined

    ctx = api.Context(device, torch_stream=False)
    p = req.p
    if cta_limit and p.nbf * p.nbf5 * p.nbfaux < AUTO_MIXED_MIN_WORK:
        ctx.set_cta_limit(cta_limit)
    b = None
    try:
        prec = resolve_precision(req.precision, req.p.nbf, req.p.nbf5, req.p.nbfaux)
        up = "fp64" if prec == "fp64" else "mixed"
        b = api.eris_to_gpu(req.b, up, ctx)
        if use_fp64_tc(req.fp64_tc, p.nbf):
            b.set_fp64_tc(True)
        if prec == "mixed_refined":
            r, _ = energy_mixed_refined(req.H, b, req.p, req.C, req.gamma, E_nuc=req.E_nuc, maxit=req.maxit)
        else:
            r = energy(req.H, b, req.p, req.C, req.gamma, E_nuc=req.E_nuc, maxit=req.maxit)
        return Result(ticket=-1, E_elec=r.E_elec, E_tot=r.E_tot, converged=r.converged, iterations=r.iterations,
                      C=r.C, n=r.n)
    finally:
        if b is not None:
            b.free()
        ctx.close()


def run_energy_group(reqs: List[Request], device: int) -> List[Result]:
    """Executor of a group: the energy loops of several FP64 jobs on one context
    as one batch (``api.Batch.energy``, donof_batch_energy): each outer
    iteration optimises the orbitals of every job still running with grouped
    launches, one per stage of a gradient step.  Every job's result is
    bit-for-bit what ``run_energy`` gives it alone."""
    import copy

    from . import api, gnof

    ctx = api.Context(device, torch_stream=False)
    bts = []
    batch = None
    try:
        ps = []
        for r in reqs:
            p = copy.copy(r.p)
            if r.maxit is not None:
                p.maxit = int(r.maxit)
            ps.append(p)
            bts.append(api.eris_to_gpu(r.b, "fp64", ctx))
        batch = api.Batch(bts, ps, ctx)
        gammas = [gnof.guess_gamma(p) if r.gamma is None else r.gamma for r, p in zip(reqs, ps)]
        out = batch.energy([r.H for r in reqs], [r.C for r in reqs], gammas)
        res = []
        for r, p, (C, gamma, n, f) in zip(reqs, ps, out):
            r.p.alpha, r.p.maxloop = p.alpha, p.maxloop
            res.append(Result(ticket=-1, E_elec=f["E_elec"], E_tot=f["E_elec"] + r.E_nuc,
                              converged=bool(f["converged"]), iterations=f["iterations"], C=C, n=n))
        return res
    finally:
        if batch is not None:
            batch.free()
        for b in bts:
            b.free()
        ctx.close()


def cta_share(max_inflight: int, sm_count: int = 148) -> int:
    """CTAs per job for a server with max_inflight slots: all SMs for one job,
    else about two jobs per SM, at least 16."""
    if max_inflight <= 1:
        return 0
    return max(16, -(-2 * sm_count // max_inflight))


def cta_share_for(max_inflight: int, device: int = 0) -> int:
    import torch
    return cta_share(max_inflight, torch.cuda.get_device_properties(device).multi_processor_count)


class Server:
    """Accepts requests at any time; runs admitted jobs concurrently, each on
    its own stream.  ``executor(request, device) -> Result`` does the work
    (``run_energy`` by default).

    With ``group_max > 1``, the FP64 jobs waiting in the queue when a slot frees
    (those ``auto`` runs in FP64: the small ones) start together as one group
    on that slot, through ``group_executor(requests, device) -> [Result]``
    (``run_energy_group``: one batch whose gradient steps advance every job of
    the group with grouped launches); the other jobs start one per slot as
    before."""

    def __init__(self, device: int = 0, budget_bytes: Optional[int] = None, max_inflight: int = 8,
                 max_bypass: int = 4, executor: Callable[[Request, int], Result] = run_energy,
                 cta_share: Optional[int] = None, group_max: int = 0,
                 group_executor: Callable[[List[Request], int], List[Result]] = run_energy_group,
                 continuous_slots: int = 0):
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            budget_bytes = int(0.85 * free)
        self.device = device
        self.admission = Admission(budget_bytes, max_inflight, max_bypass)
        if executor is run_energy:
            # each in-flight job's persistent kernels get a share of the SMs (about
            # two jobs' worth of overlap per SM), so that the jobs run side by side
            share = cta_share if cta_share is not None else cta_share_for(max_inflight, device)
            executor = functools.partial(run_energy, cta_limit=share)
        self.executor = executor
        self.group_max = int(group_max)
        self.group_executor = group_executor
        self._lock = threading.Condition()
        self._tickets = itertools.count(1)
        self._pending: Dict[int, Request] = {}
        self._results: Dict[int, Result] = {}
        self._submit_t: Dict[int, float] = {}
        self._bytes: Dict[int, int] = {}
        self._threads: List[threading.Thread] = []
        self._closed = False
        # continuous batching (continuous_slots > 0): the FP64 jobs go to one batch
        # per shape, `continuous_slots` slots each, served by donof_batch_serve
        self.continuous_slots = int(continuous_slots)
        self._buckets: Dict[tuple, "_Bucket"] = {}

    # ---- client side
    def submit(self, req: Request) -> int:
        if req.precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}")
        nbf, naux = req.p.nbf, req.p.nbfaux
        nb = footprint(nbf, naux, req.p.nbf5, resolve_precision(req.precision, nbf, req.p.nbf5, naux),
                       use_fp64_tc(req.fp64_tc, nbf))
        with self._lock:
            if self._closed:
                raise RuntimeError("server is shut down")
            t = next(self._tickets)
            if self.continuous_slots > 0 and resolve_precision(req.precision, nbf, req.p.nbf5, naux) == "fp64":
                self._submit_t[t] = time.perf_counter()
                self._bucket_locked(req).submit(t, req)
                return t
            self.admission.push(t, nb)
            self._pending[t] = req
            self._submit_t[t] = time.perf_counter()
            self._bytes[t] = nb
            self._admit_locked()
        return t

    def poll(self, ticket: int) -> Optional[Result]:
        with self._lock:
            return self._results.get(ticket)

    def wait(self, ticket: int, timeout: Optional[float] = None) -> Result:
        end = None if timeout is None else time.perf_counter() + timeout
        with self._lock:
            while ticket not in self._results:
                rem = None if end is None else end - time.perf_counter()
                if rem is not None and rem <= 0:
                    raise TimeoutError(f"ticket {ticket} not done")
                self._lock.wait(rem)
            return self._results[ticket]

    def cancel(self, ticket: int) -> bool:
        """Cancels a job that has not started: its result (error "cancelled")
        is available at once.  A job already running or done is left alone
        (False)."""
        with self._lock:
            if not self.admission.remove(ticket):
                return False
            req = self._pending.pop(ticket)
            now = time.perf_counter()
            self._bytes.pop(ticket)
            self._results[ticket] = Result(ticket=ticket, error="cancelled", t_submit=self._submit_t.pop(ticket),
                                           t_start=now, t_done=now, tag=req.tag)
            self._admit_locked()
            self._lock.notify_all()
            return True

    def shutdown(self, wait: bool = True) -> None:
        with self._lock:
            self._closed = True
            buckets = list(self._buckets.values())
        for bk in buckets:
            bk.close()
        if wait:
            for th in list(self._threads):
                th.join()
            for bk in buckets:
                bk.join()

    def _bucket_locked(self, req: Request) -> "_Bucket":
        p = req.p
        key = (p.nbf, p.nbfaux, p.nbf5, p.nalpha, p.nbeta, p.orb_method)
        bk = self._buckets.get(key)
        if bk is None:
            bk = self._buckets[key] = _Bucket(self, self.continuous_slots)
        return bk

    def _finish(self, t: int, r: Result) -> None:
        with self._lock:
            r.ticket = t
            r.t_submit = self._submit_t.pop(t)
            self._results[t] = r
            self._lock.notify_all()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.shutdown()

    # ---- scheduling
    def _groupable(self, t: int) -> bool:
        p = self._pending[t].p
        return resolve_precision(self._pending[t].precision, p.nbf, p.nbf5, p.nbfaux) == "fp64"

    def _admit_locked(self) -> None:
        while self.group_max > 1:
            group = self.admission.take_group(self._groupable, self.group_max)
            if not group:
                break
            reqs = [self._pending.pop(t) for t, _ in group]
            th = threading.Thread(target=self._run_group, args=(group, reqs), daemon=True)
            self._threads.append(th)
            th.start()
        for t, nb in self.admission.take():
            req = self._pending.pop(t)
            th = threading.Thread(target=self._run, args=(t, req, nb), daemon=True)
            self._threads.append(th)
            th.start()

    def _run_group(self, group: List[tuple], reqs: List[Request]) -> None:
        t0 = time.perf_counter()
        try:
            out = self.group_executor(reqs, self.device)
        except Exception as e:  # every job of the group fails, the server goes on
            out = [Result(ticket=-1, error=f"{type(e).__name__}: {e}") for _ in reqs]
        t1 = time.perf_counter()
        with self._lock:
            for (t, nb), req, r in zip(group, reqs, out):
                r.ticket, r.t_start, r.t_done, r.footprint, r.tag = t, t0, t1, nb, req.tag
                r.t_submit = self._submit_t.pop(t)
                self._bytes.pop(t)
                self._results[t] = r
            self.admission.release_group(sum(nb for _, nb in group))
            self._admit_locked()
            self._lock.notify_all()

    def _run(self, t: int, req: Request, nb: int) -> None:
        t0 = time.perf_counter()
        try:
            r = self.executor(req, self.device)
        except Exception as e:  # the job fails, the server goes on
            r = Result(ticket=t, error=f"{type(e).__name__}: {e}")
        r.ticket = t
        r.t_start = t0
        r.t_done = time.perf_counter()
        r.footprint = nb
        r.tag = req.tag
        with self._lock:
            r.t_submit = self._submit_t.pop(t)
            self._results[t] = r
            self.admission.release(self._bytes.pop(t))
            self._admit_locked()
            self._lock.notify_all()


class _Bucket:
    """The FP64 jobs of one shape under continuous batching: a batch of `slots`
    slots on its own context (stream) serves a queue (donof_batch_serve); each
    request uploads its RI tensor on a context of its own, pushes itself and
    waits for its result, so no context is used by two threads at once."""

    def __init__(self, server: "Server", slots: int):
        from . import api
        self.server, self.slots = server, slots
        self.ctx = api.Context(server.device, torch_stream=False)
        # no CTA share: a shape's grouped launches carry every job of the shape (with
        # the share of a single served job the benchmark stream served 2.2 against
        # 4.2 energies/s)
        self.queue = api.BatchQueue()
        self.batch = None
        self.ready = threading.Event()   # the batch exists (made from the first request)
        self.lock = threading.Lock()
        self.thread = None

    def submit(self, t: int, req: Request) -> None:
        th = threading.Thread(target=self._request, args=(t, req), daemon=True)
        self.server._threads.append(th)
        th.start()

    def _request(self, t: int, req: Request) -> None:
        from . import api, gnof
        t0 = time.perf_counter()
        ctx = b = None
        try:
            ctx = api.Context(self.server.device, torch_stream=False)
            b = api.eris_to_gpu(req.b, "fp64", ctx)
            p = copy.copy(req.p)
            gamma = gnof.guess_gamma(p) if req.gamma is None else req.gamma
            with self.lock:
                if self.batch is None:  # every slot starts bound to the first request's tensor
                    self.batch = api.Batch([b] * self.slots, [p] * self.slots, self.ctx)
                    self.thread = threading.Thread(target=self.batch.serve, args=(self.queue,), daemon=True)
                    self.thread.start()
            ticket = self.queue.push(b, req.H, req.C, gamma, p, maxit=req.maxit)
            C, g, n, f = self.queue.wait(ticket)
            r = Result(ticket=t, E_elec=f["E_elec"], E_tot=f["E_elec"] + req.E_nuc, converged=bool(f["converged"]),
                       iterations=f["iterations"], C=C, n=n)
        except Exception as e:  # the job fails, the server goes on
            r = Result(ticket=t, error=f"{type(e).__name__}: {e}")
        finally:
            if b is not None:
                b.free()
            if ctx is not None:
                ctx.close()
        r.t_start, r.t_done, r.tag = t0, time.perf_counter(), req.tag
        self.server._finish(t, r)

    def close(self) -> None:
        self.queue.close()

    def join(self) -> None:
        if self.thread is not None:
            self.thread.join()
        if self.batch is not None:
            self.batch.free()
        self.ctx.close()


def percentiles(values, qs=(50, 99)) -> dict:
    v = np.asarray(values, dtype=np.float64)
    return {f"p{q}": float(np.percentile(v, q)) for q in qs} if v.size else {f"p{q}": None for q in qs}


# ---------------------------------------------------------------- native server
class NativeServer:
    """The library's own server (donof_server_*): the same admission policy,
    SM shares and energy loop in native code, behind a thread-safe queue.  The
    request's arrays are kept alive here until the job is collected."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_inflight: int = 8):
        import ctypes as ct
        from . import _lib
        self._ct = ct
        self.lib = _lib.load()
        h = ct.c_void_p()
        _lib.check(self.lib.donof_server_create(int(device), int(budget_bytes), int(max_inflight), ct.byref(h)))
        self.handle = h
        self._keep: Dict[int, tuple] = {}

    def submit(self, req: Request) -> int:
        import ctypes as ct
        from . import _lib, api, gnof
        p = req.p
        H, b, C = api._f64(req.H), api._f64(req.b), api._f64(req.C)
        gamma = np.ascontiguousarray(gnof.guess_gamma(p) if req.gamma is None else req.gamma, dtype=np.float64)
        prm = api._EnergyParams(api._occ_params(p), _lib.ORB_METHODS[p.orb_method], int(req.maxit or p.maxit),
                                int(p.maxloop), float(p.alpha), float(p.threshgorb), float(p.threshgocc),
                                float(p.threshen), int(p.ipnof > 4), 0, 0.0,
                                int(bool(getattr(p, "occ_device", False))))
        prec = {"fp64": 0, "mixed": 1, "mixed_refined": 1, "auto": 2}[req.precision]
        r = _NativeRequest(H.ctypes.data, b.ctypes.data, C.ctypes.data, gamma.ctypes.data, p.nbf, p.nbfaux, prm,
                           prec, float(req.E_nuc))
        C_out = np.zeros((p.nbf, p.nbf), order="F")
        n_out = np.zeros(p.nbf5)
        t = ct.c_ulonglong()
        _lib.check(self.lib.donof_server_submit(self.handle, ct.byref(r), C_out.ctypes.data, n_out.ctypes.data,
                                                ct.byref(t)))
        self._keep[t.value] = (H, b, C, gamma, r, C_out, n_out, req.tag)
        return t.value

    def _result(self, ticket: int, res) -> Result:
        H, b, C, gamma, r, C_out, n_out, tag = self._keep.pop(ticket)
        err = (res.error.decode() or f"status {res.status}") if res.status != 0 else None
        return Result(ticket=ticket, E_elec=res.E_elec, E_tot=res.E_tot, converged=bool(res.converged),
                      iterations=res.iterations, C=C_out, n=n_out, error=err, t_submit=0.0,
                      t_start=res.queue_s, t_done=res.latency_s, tag=tag)

    def wait(self, ticket: int) -> Result:
        from . import _lib
        res = _NativeResult()
        _lib.check(self.lib.donof_server_wait(self.handle, self._ct.c_ulonglong(ticket), self._ct.byref(res)))
        return self._result(ticket, res)

    def poll(self, ticket: int) -> Optional[Result]:
        """The result if the job has ended (it is then collected), else None."""
        from . import _lib
        res = _NativeResult()
        done = self._ct.c_int()
        _lib.check(self.lib.donof_server_poll(self.handle, self._ct.c_ulonglong(ticket), self._ct.byref(res),
                                              self._ct.byref(done)))
        return self._result(ticket, res) if done.value else None

    def cancel(self, ticket: int) -> None:
        """Cancels a job: a queued one ends at once, a running one at its next
        outer iteration; its result then carries the error "cancelled"."""
        from . import _lib
        _lib.check(self.lib.donof_server_cancel(self.handle, self._ct.c_ulonglong(ticket)))

    def close(self) -> None:
        if self.handle:
            self.lib.donof_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _native_types():
    import ctypes as ct
    from . import api

    class Req(ct.Structure):
        _fields_ = [("H", ct.c_void_p), ("b", ct.c_void_p), ("C", ct.c_void_p), ("gamma", ct.c_void_p),
                    ("nbf", ct.c_int), ("naux", ct.c_int), ("params", api._EnergyParams), ("precision", ct.c_int),
                    ("E_nuc", ct.c_double)]

    class Res(ct.Structure):
        _fields_ = [("status", ct.c_int), ("E_elec", ct.c_double), ("E_tot", ct.c_double),
                    ("iterations", ct.c_int), ("converged", ct.c_int), ("precision", ct.c_int),
                    ("queue_s", ct.c_double), ("latency_s", ct.c_double), ("error", ct.c_char * 256)]

    return Req, Res


_NativeRequest, _NativeResult = _native_types()
