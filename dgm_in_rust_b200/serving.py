"""Continuous-batching solve server: a host scheduler over device-resident batched solves.

No counterpart in the reference, which runs one configured solve per process.  Requests (an
O-grid size, flow condition and polynomial order) arrive over time.  The loop

* prepares each request's mesh in a pool of worker processes (or threads) as soon as it arrives;
  the initial state is projected on the device at admission;
* admits prepared requests in arrival order while the device footprint of the active solves
  plus theirs fits the HBM budget (a request that does not fit waits, and so does every prepared
  request behind it, until running solves retire and free their memory; a request still being
  prepared does not hold back those behind it);
* packs the requests it admits together into cohorts -- one :class:`Batch` context per
  polynomial order, so that every launch of a step covers all of a cohort's meshes -- and runs
  each cohort on its own CUDA stream, so cohorts admitted at different times overlap on the
  GPU.  Each member occupies a slot with room for a mesh ``headroom`` times its own
  (dgm_create_batch_slots);
* polls every cohort without blocking; when a cohort's chunk of steps is done it reads the
  density-residual norm of each member that has reached its next check, retires the members
  that have converged (residual dropped by ``tol`` relative to the first step's) or reached
  ``max_steps``, and hands each freed slot to the first waiting request of the cohort's order
  whose mesh fits it (dgm_instance_replace: the new solve joins the cohort's launches at once,
  without a new context) -- continuous batching at the granularity of a slot.  A slot nobody
  takes is switched off (later launches skip its elements); the cohort's memory returns to the
  budget when all its slots are free and no waiting request fits one;
* advances each cohort by the steps until its earliest member check, every member stopping at
  its own check (its loop bound), so members that joined at different times keep their own
  schedule.

Each member of a cohort is computed exactly as it would be alone (instances of a batch are
disconnected meshes with their own time step and clock, padding slots are skipped, and every
reduction is per instance and deterministic), and convergence is tested at the same step counts
(step 1, then every ``chunk_steps``), so a request's result does not depend on what else was
running or which slot it ran in; the tests check this bitwise.
"""
from __future__ import annotations

import dataclasses
import math
import multiprocessing
import queue
import threading
import time
from concurrent.futures import ProcessPoolExecutor, ThreadPoolExecutor

import numpy as np

from .basis_function import default_rules
from ._native import DgmError
from .solver import Batch, build_solver, slot_capacity
from .workloads import HCR, Instance, instance_mesh

__all__ = ["Request", "Result", "ServingLoop", "footprint_bytes", "latency_summary", "requests_from_stream",
           "solve_alone", "one_at_a_time"]

CFL = 0.1
NEQ = 4


@dataclasses.dataclass
class Request:
    rid: int
    arrival_s: float
    instance: Instance


@dataclasses.dataclass
class Result:
    rid: int
    arrival_s: float
    admitted_s: float
    finished_s: float
    steps: int
    time: float
    residual_drop: float
    converged: bool
    status: int
    dofs: int
    state: np.ndarray | None = None
    ready_s: float | None = None     # host preparation finished (serving loop only)

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


def requests_from_stream(stream: list) -> list:
    """[(arrival_s, Instance)] as produced by workloads.request_stream -> [Request]."""
    return [Request(i, float(t), inst) for i, (t, inst) in enumerate(stream)]


def footprint_bytes(meshes: list, order: int, precision: str, limiter: bool = True, capacities=None) -> int:
    """Device bytes a batch context of ``meshes`` allocates: the sum of the requested sizes of
    its allocations (what dgm_device_bytes reports), following dgm_create's allocation list.
    ``capacities``: the slot rooms of dgm_create_batch_slots (default: the meshes' own sizes)."""
    nb = (order + 1) * (order + 2) // 2
    ng = default_rules(order)[1]
    eb = 8 if precision == "fp64" else 4
    n = len(meshes)
    own = [slot_capacity(m) for m in meshes]
    caps = own if capacities is None else [tuple(int(x) for x in c) for c in capacities]
    padded = any(tuple(c) != tuple(o) for c, o in zip(caps, own))
    ne = sum(c[0] for c in caps) + (1 if padded else 0)
    ld = (ne + 31) // 32 * 32
    n_int = sum(c[1] for c in caps)
    n_bnd = sum(c[2] for c in caps)
    n_patch = sum(c[3] for c in caps)
    max_ne = max(c[0] for c in caps)

    def arr(count, size):             # dev_alloc: at least one element
        return max(count, 1) * size

    control = 1280 + (n + 1) * 72                                    # Control, InstCtl[n + 1]
    geometry = 3 * ne * 8 + 4 * ld * 8 + 2 * 3 * ld * 4 + ne * 4 + ld // 32 * 4  # jac, hmin, h15, dinv, face, nbr,
    #                                                                              inst, batch order
    edges = (arr(n_int, 8) + arr(n_int, 4) + arr(n_int, 32) + arr(n_bnd, 4) + arr(n_bnd, 4) + arr(n_bnd, 32)
             + max(n_patch, 1) * 32 + (n_int + n_bnd) * 8)          # internal, boundary, patches, slot_ref
    offsets = 2 * (2 * n) * 4                                        # instance ranges
    state = 4 * NEQ * nb * ld * eb                                   # U, U1, U2, R
    flux = (n_int + n_bnd) * ng * 4 * eb                             # F
    stage = max_ne * NEQ * nb * 8                                    # FP64 staging
    limiter_bytes = ne * (1 + 4 + 4 + 32 + 4)                        # t0, status, work, wl1 entries, pend
    diag = n * 8 * 8
    gram = nb * (nb + 1) // 2 * ld * 8 if limiter else 0              # WENO Gram matrices
    return int(control + geometry + edges + offsets + state + flux + stage + limiter_bytes + diag + gram)


def _prepare_request(req: Request):
    """Host preparation of one request (runs in a worker): the processed O-grid and its
    free-stream initial condition."""
    if req.instance.order not in (1, 2, 3):
        raise ValueError(f"unsupported polynomial order {req.instance.order}")
    mesh, init = instance_mesh(req.instance)
    return req, mesh, init


def _warm():
    return 0


class _Member:
    def __init__(self, req: Request, index: int, ready_s: float, elements: int, admitted_s: float):
        self.req = req
        self.index = index
        self.elements = elements
        self.ready_s = ready_s
        self.admitted_s = admitted_s
        self.r0 = None
        self.drop = 1.0
        self.next_check = 1  # the first check is after one step: its residual is the reference
        self.done = False


def _room(cap, headroom: float) -> tuple:
    """A slot's room for a mesh of counts ``cap``: each count times ``headroom``, rounded up."""
    return tuple(int(math.ceil(c * headroom)) for c in cap)


def _fits(need, room) -> bool:
    return all(n <= r for n, r in zip(need, room))


class _Cohort:
    def __init__(self, items: list, order: int, precision: str, device: int, max_steps: int, now: float,
                 headroom: float):
        meshes = [it[1] for it in items]
        n = len(items)
        self.order = order
        self.max_steps = max_steps
        self.rooms = [_room(slot_capacity(m), headroom) for m in meshes]
        self.batch = Batch(meshes, order, HCR, [CFL] * n, [1.0e30] * n, [1] * n, limiter=True,
                           device=device, precision=precision, capacities=self.rooms)
        for i, it in enumerate(items):
            self.batch.set_initial(i, it[2])
        self.slots = [_Member(it[0], i, it[3], it[1].n_elements, now) for i, it in enumerate(items)]
        self.bytes = self.batch.device_bytes()
        self.checks = 0
        self.advance()

    def members(self):
        return [m for m in self.slots if m is not None and not m.done]

    def free_slots(self):
        return [i for i, m in enumerate(self.slots) if m is None or m.done]

    def advance(self) -> bool:
        """Enqueue the steps up to the earliest member check (each member stops at its own check);
        False if no member is running."""
        live = self.members()
        if not live:
            return False
        steps = {m.index: self.batch.state(m.index)[1] for m in live}
        n = min(min(m.next_check, self.max_steps) - steps[m.index] for m in live)
        self.batch.advance(max(n, 1), with_residual=True)
        self.batch.enqueue_diagnostics(use_residual=True)  # read at the check, no device work there
        return True

    def take(self, i: int, item, now: float) -> None:
        """Slot i takes a waiting request (the cohort's stream is idle)."""
        req, mesh, init, ready_s = item
        self.batch.replace(i, mesh, CFL, 1.0e30, 1)
        self.batch.set_initial(i, init)
        self.slots[i] = _Member(req, i, ready_s, mesh.n_elements, now)

    def close(self):
        self.batch.close()


class ServingLoop:
    """Serve solve requests with continuous batching under an HBM budget.

    ``precision`` is the batched contexts' precision ("fp32": FP32 bulk arithmetic with the
    limiter, positivity checks, time step and diagnostics in FP64; "fp64": the reference's
    arithmetic).  ``window_s`` is how long a new arrival may wait for others to share its
    cohort while the GPU is busy (an idle GPU admits at once).  ``max_active_elements`` caps the
    work in flight: a request is admitted only while the elements of the running (not yet retired)
    requests plus its own stay within the cap (a request larger than the cap runs alone).  Enough
    elements to keep the GPU's launches full run at once; later arrivals wait in arrival order
    instead of sharing the GPU with everything admitted before them, so early requests finish
    early (first come, first served at the granularity of the cap).  ``prep`` selects worker
    threads ("thread", the default: the mesh is built by the library's native code, which runs
    outside the interpreter lock, and nothing is copied back) or worker processes ("process",
    started with spawn before the clock starts, like a server's standing pool; each prepared mesh
    is pickled back to the serving process) for mesh preparation.  ``headroom`` sizes every slot
    for a mesh that many times its first occupant's counts, and a freed slot takes a waiting
    request of its cohort's order whose mesh fits it and is no smaller than the slot's room divided
    by ``max_slot_waste`` (``headroom`` 1 gives exact-size slots that only an equal or smaller mesh
    reuses)."""

    def __init__(self, hbm_budget_bytes: int = 40 << 30, device: int = 0, precision: str = "fp32",
                 chunk_steps: int = 32, tol: float = 1e-6, max_steps: int = 5000, window_s: float = 0.002,
                 max_cohort_elements: int = 4 << 20, max_active_elements: int = 2 << 20, prep_workers: int = 4,
                 prep: str = "thread", keep_states: bool = False, headroom: float = 1.5,
                 max_slot_waste: float = 4.0):
        if chunk_steps < 1 or max_steps < 1:
            raise ValueError("chunk_steps and max_steps must be positive")
        self.budget = int(hbm_budget_bytes)
        self.device = int(device)
        self.precision = precision
        self.chunk = int(chunk_steps)
        self.tol = float(tol)
        self.max_steps = int(max_steps)
        self.window = float(window_s)
        self.max_cohort_elements = int(max_cohort_elements)
        self.max_active_elements = int(max_active_elements)
        if prep not in ("process", "thread"):
            raise ValueError("prep must be 'process' or 'thread'")
        self.prep_workers = max(1, int(prep_workers))
        self.prep = prep
        self.keep_states = keep_states
        if headroom < 1.0 or max_slot_waste < 1.0:
            raise ValueError("headroom and max_slot_waste must be >= 1")
        self.headroom = float(headroom)
        self.max_slot_waste = float(max_slot_waste)
        self.slot_reuses = 0
        self.peak_bytes = 0
        self.cohorts_formed = 0
        self.max_concurrent = 0
        self.stats = {}
        self._realtime = True

    def run(self, requests: list, realtime: bool = True) -> list:
        """Serve ``requests`` (list of Request).  With ``realtime`` each request becomes visible
        at its arrival time on the wall clock (latency is measured from it); otherwise all are
        visible at once (latency from the start of the run).  Returns the Results ordered by
        request id."""
        reqs = sorted(requests, key=lambda r: (r.arrival_s, r.rid))
        if not reqs:
            return []
        ready: "queue.Queue" = queue.Queue()
        self._realtime = bool(realtime)
        if self.prep == "process":
            pool = ProcessPoolExecutor(max_workers=self.prep_workers, mp_context=multiprocessing.get_context("spawn"))
            for f in [pool.submit(_warm) for _ in range(self.prep_workers)]:
                f.result()
        else:
            pool = ThreadPoolExecutor(max_workers=self.prep_workers)
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        def done(fut, r):
            exc = fut.exception()
            ready.put((r, None, exc) if exc is not None else fut.result())

        def feeder():
            for r in reqs:
                if realtime:
                    wait = r.arrival_s - now()
                    if wait > 0:
                        time.sleep(wait)
                pool.submit(_prepare_request, r).add_done_callback(lambda f, r=r: done(f, r))

        self.stats = {"create_s": 0.0, "check_s": 0.0, "replace_s": 0.0, "idle_s": 0.0, "chunks": 0}
        self.slot_reuses = 0
        feed = threading.Thread(target=feeder, daemon=True)
        feed.start()
        waiting: list = []       # prepared, not admitted: (req, mesh, initial, ready_s), in arrival order
        active: list = []        # cohorts
        results: list = []
        used = 0
        try:
            while len(results) < len(reqs):
                got = False
                while True:
                    try:
                        item = ready.get_nowait()
                    except queue.Empty:
                        break
                    if item[1] is None:
                        raise RuntimeError(f"preparing request {item[0].rid} failed") from item[2]
                    waiting.append(item + (now(),))
                    got = True
                if got:
                    waiting.sort(key=lambda it: (it[0].arrival_s, it[0].rid))
                used = self._admit(waiting, active, used, now)
                progressed = False
                for co in list(active):
                    st = co.batch.query()
                    if st is None:
                        continue
                    progressed = True
                    tc = time.perf_counter()
                    finished = self._check(co, results, waiting, active, now)
                    self.stats["check_s"] += time.perf_counter() - tc
                    self.stats["chunks"] += 1
                    if finished:
                        active.remove(co)
                        used -= co.bytes
                        co.close()
                if not progressed and not got:
                    ti = time.perf_counter()
                    time.sleep(0.0002)
                    self.stats["idle_s"] += time.perf_counter() - ti
        finally:
            feed.join()
            pool.shutdown(wait=True)
            for co in active:
                co.close()
        return sorted(results, key=lambda r: r.rid)

    def _admit(self, waiting: list, active: list, used: int, now) -> int:
        if not waiting:
            return used
        if active and (now() - min(it[3] for it in waiting)) < self.window:
            return used
        take: list = []
        need_total = 0
        running = sum(m.elements for co in active for m in co.members())
        for item in waiting:
            need = footprint_bytes([item[1]], item[0].instance.order, self.precision,
                                   capacities=[_room(slot_capacity(item[1]), self.headroom)])
            if (active or take) and used + need_total + need > self.budget:
                break           # first-come first-served: nothing overtakes a request that waits for memory
            if (running or take) and running + item[1].n_elements > self.max_active_elements:
                break           # enough work in flight: later requests wait, in arrival order
            take.append(item)
            need_total += need
            running += item[1].n_elements
        if not take:
            return used
        del waiting[:len(take)]
        groups: dict = {}
        for item in take:
            groups.setdefault(item[0].instance.order, []).append(item)
        for order, items in sorted(groups.items()):
            chunk: list = []
            ne = 0
            for item in items + [None]:
                if item is None or (chunk and ne + item[1].n_elements > self.max_cohort_elements):
                    tc = time.perf_counter()
                    co = _Cohort(chunk, order, self.precision, self.device, self.max_steps, now(), self.headroom)
                    self.stats["create_s"] += time.perf_counter() - tc
                    active.append(co)
                    used += co.bytes
                    self.cohorts_formed += 1
                    chunk, ne = [], 0
                if item is not None:
                    chunk.append(item)
                    ne += item[1].n_elements
        self.peak_bytes = max(self.peak_bytes, used)
        self.max_concurrent = max(self.max_concurrent, sum(len(c.members()) for c in active))
        return used

    def _check(self, co: _Cohort, results: list, waiting: list, active: list, now) -> bool:
        """Convergence test of the members at their check step; retires members, hands freed slots
        to waiting requests, enqueues the next steps.  Returns True when the cohort can close (no
        member running)."""
        b = co.batch
        diag = b.collected_diagnostics()
        co.checks += 1
        for m in co.members():
            t, step, status, _ = b.state(m.index)
            if status == 0 and step < min(m.next_check, self.max_steps):
                continue  # not at its check yet
            r = math.sqrt(max(float(diag[m.index, 6]), 0.0))
            if m.r0 is None:
                m.r0 = r if r > 0.0 else 1.0
            m.drop = r / m.r0
            converged = step > 1 and m.drop <= self.tol
            if status != 0 or converged or step >= self.max_steps:
                state = b.download(m.index) if self.keep_states else None
                arrival = m.req.arrival_s if self._realtime else 0.0
                results.append(Result(m.req.rid, arrival, m.admitted_s, now(), step, t, m.drop, converged,
                                      status, m.req.instance.dofs, state, m.ready_s))
                b.set_instance(m.index, t, step, 1.0e30, step)   # switched off from the next launch on
                m.done = True
            else:
                m.next_check = step + self.chunk
                b.set_instance(m.index, t, step, 1.0e30, min(m.next_check, self.max_steps))
        self._fill_slots(co, waiting, active, now)
        return not co.advance()

    def _fill_slots(self, co: _Cohort, waiting: list, active: list, now) -> None:
        """Hand the cohort's free slots to the waiting requests at the head of the queue, in arrival
        order, while the work-in-flight cap allows: each takes the smallest free slot that fits it
        (and is not more than max_slot_waste times too large).  The first request that cannot take
        a slot here (another order, too large, or no room in flight) stops the scan: first come,
        first served, nothing overtakes a request that waits."""
        free = co.free_slots()
        if not free or not waiting:
            return
        running = sum(m.elements for c in active for m in c.members())
        k = 0
        while k < len(waiting) and free:
            item = waiting[k]
            if item[0].instance.order != co.order:
                break
            need = slot_capacity(item[1])
            fit = [i for i in free if _fits(need, co.rooms[i]) and co.rooms[i][0] <= self.max_slot_waste * need[0]]
            if not fit:
                break
            if running and running + item[1].n_elements > self.max_active_elements:
                break
            i = min(fit, key=lambda j: co.rooms[j][0])
            tr = time.perf_counter()
            co.take(i, item, now())
            self.stats["replace_s"] += time.perf_counter() - tr
            self.slot_reuses += 1
            free.remove(i)
            del waiting[k]
            running += item[1].n_elements
        self.max_concurrent = max(self.max_concurrent, sum(len(c.members()) for c in active))


def solve_alone(req: Request, precision: str = "fp64", device: int = 0, chunk_steps: int = 32, tol: float = 1e-6,
                max_steps: int = 5000, keep_state: bool = False) -> tuple:
    """One request on a plain single-mesh context (the reference-shaped Solver path), with the
    serving loop's convergence schedule (step 1, then every ``chunk_steps``).  Returns
    (Result with finished_s = service time, service time in s, of which host preparation in s)."""
    t0 = time.perf_counter()
    _, mesh, init = _prepare_request(req)
    prep = time.perf_counter() - t0
    solver = build_solver(mesh, req.instance.order, HCR, CFL, 1.0e30, max_steps, limiter=True, device=device,
                          precision=precision)
    try:
        td, sd = solver.temporal_disc, solver.spatial_disc
        td.set_initial_on_device(init)
        r0, drop, converged, status = None, 1.0, False, 0
        n = 1
        while True:
            td.advance(n, with_residual=True)
            sd.enqueue_diagnostics(use_residual=True)
            try:
                td.synchronize()
            except DgmError as e:
                status = e.status
            step = td.current_step
            r = math.sqrt(max(float(sd.collected_diagnostics()[6]), 0.0))
            if r0 is None:
                r0 = r if r > 0.0 else 1.0
            drop = r / r0
            converged = step > 1 and drop <= tol
            if status != 0 or converged or step >= max_steps:
                break
            n = chunk_steps
        state = None
        if keep_state:
            state = sd.new_state()
            td.download(state)
        service = time.perf_counter() - t0
        return Result(req.rid, 0.0, 0.0, service, step, td.current_time, drop, converged, status, req.instance.dofs,
                      state), service, prep
    finally:
        solver.close()


def one_at_a_time(requests: list, precision: str = "fp64", device: int = 0, chunk_steps: int = 32, tol: float = 1e-6,
                  max_steps: int = 5000) -> tuple:
    """A first-come first-served server that runs one request at a time on the plain context.
    Each request is solved back to back (service times measured); its latency is then that of
    the FIFO queue under the requests' arrival times: finish_i = max(arrival_i, finish_{i-1}) +
    service_i.  Returns (Results, total service time in s, of which host preparation in s)."""
    out = []
    busy = 0.0
    prep_total = 0.0
    finish = 0.0
    for req in sorted(requests, key=lambda r: (r.arrival_s, r.rid)):
        res, service, prep = solve_alone(req, precision, device, chunk_steps, tol, max_steps)
        busy += service
        prep_total += prep
        start = max(req.arrival_s, finish)
        finish = start + service
        res.arrival_s, res.admitted_s, res.finished_s = req.arrival_s, start, finish
        out.append(res)
    return sorted(out, key=lambda r: r.rid), busy, prep_total


def latency_summary(results: list, wall_s: float) -> dict:
    """p50/p99/mean latency (arrival to retirement) and throughput in DOF-stage updates/s."""
    lat = np.array([r.latency_s for r in results])
    dof_stages = sum(r.dofs * 3 * r.steps for r in results)
    out = {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
           "mean_s": float(lat.mean()), "wall_s": wall_s, "dof_stage_updates_per_s": dof_stages / wall_s,
           "converged": int(sum(r.converged for r in results)), "failed": int(sum(r.status != 0 for r in results))}
    if all(r.ready_s is not None for r in results):
        out["mean_prep_s"] = float(np.mean([r.ready_s - r.arrival_s for r in results]))
        out["mean_queue_s"] = float(np.mean([r.admitted_s - r.ready_s for r in results]))
        out["mean_run_s"] = float(np.mean([r.finished_s - r.admitted_s for r in results]))
    return out
